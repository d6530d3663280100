"""Shared test helpers: build the oracle twin of a bfx configuration."""
from __future__ import annotations

import numpy as np

import bfx._lib as L
import oracle as O

GEOMETRY_NAMES = {L.GEOMETRY_NONE: None, L.GEOMETRY_BIRD: "bird", L.GEOMETRY_ELLIPSOID: "ellipsoid",
                  L.GEOMETRY_MESH: "mesh", L.GEOMETRY_FLAPPING_WING: "wing"}


def oracle_params(cfg: L.Config) -> O.Params:
    p = O.make_params(
        cfg.nx, cfg.ny, cfg.nz, dx=cfg.cell_size, origin=tuple(cfg.origin), dt=cfg.time_step,
        v2l=cfg.velocity_to_lattice, f2p=cfg.force_to_physical, omega_p=cfg.omega_plus, omega_m=cfg.omega_minus,
        sponge_strength=cfg.sponge_strength, sponge_width=cfg.sponge_width, far=tuple(cfg.far_field),
        gravity=tuple(cfg.gravity), accumulate_loads=bool(cfg.accumulate_loads),
        interpolated=cfg.wall_rule == L.WALL_INTERPOLATED, collision=cfg.collision,
        load_component=cfg.load_component, force_mode=cfg.force_estimator, selected_part=cfg.selected_part,
        free_flight=bool(cfg.free_flight), face_bc=tuple(cfg.face_bc),
        face_velocity=[tuple(cfg.face_velocity[i]) for i in range(6)], substeps=cfg.body_substeps,
        local_density=bool(cfg.moving_wall_local_density))
    return p


def oracle_wing(wing: L.FlappingWing) -> O.Wing:
    w = O.Wing()
    for name, _ in O.Wing._fields_:
        getattr(w, name).v[:] = list(getattr(wing, name).v)
    w.kinematics1.v[3] = 0.0  # the library drops the reference speed (not part of the geometry)
    return w


def oracle_twin(cfg: L.Config, bird_rows=None, body=None, mesh=None, wing=None) -> O.OracleSim:
    p = oracle_params(cfg)
    geometry = GEOMETRY_NAMES[cfg.geometry]
    bird = O.bird_from_dict(dict(zip(L.BIRD_FIELDS, bird_rows))) if bird_rows is not None else None
    shear = None
    if cfg.init in (L.INIT_SHEAR_WAVE_Y, L.INIT_SHEAR_WAVE_Z):
        shear = (cfg.init_amplitude, 1 if cfg.init == L.INIT_SHEAR_WAVE_Y else 2)
    om = None
    if mesh is not None:
        om = dict(mesh)
        om["local"] = np.ascontiguousarray(mesh["local"], np.float32).ravel()
        om["local"] = om["local"].reshape(-1, 3)
        om["half_thickness"] = cfg.mesh_half_thickness
        if mesh.get("kf_times") is not None:
            om["kf_times"] = np.ascontiguousarray(mesh["kf_times"], np.float32)
            om["kf_points"] = np.ascontiguousarray(mesh["kf_points"], np.float32).ravel()
    return O.OracleSim(p, geometry=geometry, bird=bird, body=body, mesh=om,
                       link_rule="linear" if cfg.link_rule == L.LINK_LINEAR else "ray", shear=shear,
                       wing=oracle_wing(wing) if wing is not None else None)


def body_struct_from_tuple(body):
    s = L.BodyState()
    if body is None:
        s.orientation[:] = [0, 0, 0, 1]
        return s
    pos, orient, vel, omega = body
    s.position[:] = list(pos)
    s.orientation[:] = list(orient)
    s.velocity[:] = list(vel)
    s.omega_body[:] = list(omega)
    return s


def rel_diff(a, b, floor=1e-30):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))
