"""Workload builders: the lattice configurations the library is measured and
tested on, each as (bfx config, bird rows, body state, mesh).

All sizes are in lattice units (dx = dt = 1) unless a case says otherwise.
  shear_wave            periodic TRT shear-wave decay (64^3, nu 0.01, magic 1/4)
  ellipsoid_channel     RR3 channel past a stationary ellipsoid, velocity inlet,
                        zero-gradient outlet, periodic y/z, interpolated links
  flapping_plates       two rectangular flat-plate wings as a triangle mesh,
                        stroke 60 deg sin, pitch 45 deg cos, links rebuilt each step
  compact_bird          the reference's compact analytic bird on 48^3
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L
from .config import BirdParameters, LatticeScaling, SimulationConfiguration, GridSize, WingKinematics, f32
from .simulation import default_config


def _trt_rates(viscosity: float, magic: float):
    s = LatticeScaling.lattice_only(viscosity, magic)
    return s.omega_plus, s.omega_minus


def zero_bird_rows():
    return [(0.0, 0.0, 0.0, 0.0)] * 13


def shear_wave(n=64, viscosity=0.01, amplitude=0.01, magic=0.25, axis="z", storage=L.STORAGE_F32,
               collision=L.COLLISION_TRT, nx=None, ny=None, nz=None):
    op, om = _trt_rates(viscosity, magic)
    cfg = default_config(nx or n, ny or n, nz or n, omega_plus=op, omega_minus=om, face_bc=[L.BC_PERIODIC] * 6,
                         init=L.INIT_SHEAR_WAVE_Z if axis == "z" else L.INIT_SHEAR_WAVE_Y,
                         init_amplitude=amplitude, storage=storage, collision=collision, accumulate_loads=0)
    return cfg, None, None, None


def ellipsoid_bird_rows(radii, mass=1.0, inertia=(1.0, 1.0, 1.0)):
    rows = zero_bird_rows()
    rows[0] = (radii[0], radii[1], radii[2], mass)
    rows[1] = (inertia[0], inertia[1], inertia[2], 0.0)
    rows[8] = (0.0, 0.15, 0.0, 0.0)
    return rows


def ellipsoid_channel(nx=256, ny=128, nz=128, radii=(24.0, 12.0, 12.0), center=None, inflow=0.05,
                      viscosity=0.005, magic=3.0 / 16.0, collision=L.COLLISION_RR3, storage=L.STORAGE_F32,
                      wall_rule=L.WALL_INTERPOLATED, static=True):
    op, om = _trt_rates(viscosity, magic)
    if center is None:
        center = (nx / 4.0, ny / 2.0, nz / 2.0)
    faces = [L.BC_VELOCITY, L.BC_OUTFLOW, L.BC_PERIODIC, L.BC_PERIODIC, L.BC_PERIODIC, L.BC_PERIODIC]
    fv = [(inflow, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5
    cfg = default_config(nx, ny, nz, omega_plus=op, omega_minus=om, face_bc=faces, face_velocity=fv,
                         far_field=[inflow, 0.0, 0.0, 1.0], geometry=L.GEOMETRY_ELLIPSOID, wall_rule=wall_rule,
                         collision=collision, storage=storage, static_geometry=int(static), sponge_strength=0.0)
    body = (tuple(center), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return cfg, ellipsoid_bird_rows(radii), body, None


def plate_mesh(span=64.0, chord=12.0, n_chord=32, n_span=128, chord_offset=-3.0, span_offset=0.0):
    """Two triangulated flat rectangles in their wing frames (chord, span, normal):
    2 * n_chord * n_span triangles per wing, part 2 = left, 3 = right."""
    cs = np.linspace(0.0, chord, n_chord + 1, dtype=np.float64) + chord_offset
    ss = np.linspace(0.0, span, n_span + 1, dtype=np.float64) + span_offset
    C, S = np.meshgrid(cs, ss, indexing="xy")  # rows along span, columns along chord
    local_one = np.stack([C.ravel(), S.ravel(), np.zeros(C.size)], axis=1).astype(np.float32)
    nv = local_one.shape[0]
    tris = []
    w = n_chord + 1
    for j in range(n_span):
        for i in range(n_chord):
            a = j * w + i
            b = a + 1
            c = a + w
            d = c + 1
            tris.append((a, b, c))
            tris.append((d, c, b))
    tris = np.asarray(tris, np.uint32)
    local = np.concatenate([local_one, local_one])
    segment = np.concatenate([np.full(nv, 1, np.uint8), np.full(nv, 2, np.uint8)])
    tris2 = np.concatenate([tris, tris + nv])
    part = np.concatenate([np.full(len(tris), 2, np.uint8), np.full(len(tris), 3, np.uint8)])
    return {"local": local, "segment": segment, "tris": tris2, "tri_part": part}


def flapping_plates(nx=512, ny=256, nz=256, span=64.0, chord=12.0, thickness=2.0, n_chord=32, n_span=128,
                    period=4000.0, stroke_deg=60.0, pitch_deg=45.0, viscosity=0.004, magic=3.0 / 16.0,
                    storage=L.STORAGE_F32, collision=L.COLLISION_TRT, link_rule=L.LINK_RAY_ROOT,
                    wall_rule=L.WALL_INTERPOLATED, sponge_width=16.0, sponge_strength=0.05, deviation_deg=0.0,
                    pitch_phase_offset_deg=0.0):
    op, om = _trt_rates(viscosity, magic)
    rows = zero_bird_rows()
    rows[0] = (4.0, 4.0, 4.0, 1.0)
    rows[1] = (1.0, 1.0, 1.0, 0.0)
    rows[2] = (span, chord, chord, thickness)
    rows[3] = (0.0, 0.0, 0.0, 0.0)
    freq = 1.0 / period
    rows[5] = (freq, float(f32(math.radians(stroke_deg))), 0.0, 0.0)
    rows[6] = (float(f32(math.radians(pitch_deg))), float(f32(math.pi / 2.0 + math.radians(pitch_phase_offset_deg))),
               float(f32(math.radians(deviation_deg))), 0.0)
    rows[8] = (0.0, 0.15, 0.0, 0.0)
    cfg = default_config(nx, ny, nz, omega_plus=op, omega_minus=om, face_bc=[L.BC_FARFIELD] * 6,
                         geometry=L.GEOMETRY_MESH, wall_rule=wall_rule, collision=collision, storage=storage,
                         link_rule=link_rule, mesh_half_thickness=0.5 * thickness, sponge_width=sponge_width,
                         sponge_strength=sponge_strength)
    body = ((nx / 2.0, ny / 2.0, nz / 2.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return cfg, rows, body, plate_mesh(span, chord, n_chord, n_span)


def compact_bird(free_flight=False, storage=L.STORAGE_F32, n=48):
    """compactMetalTestCase (Tests/BirdFlowMetalTests/MetalExecutionTests.swift:411-470)."""
    bird = BirdParameters(
        body_radii_meters=(0.015, 0.011, 0.012), mass_kilograms=0.025,
        principal_inertia_kilogram_meters_squared=(0.000004, 0.000007, 0.000008),
        wing_span_meters=0.025, wing_root_chord_meters=0.020, wing_tip_chord_meters=0.012,
        wing_thickness_meters=0.008, wing_sweep_meters=0.004, wing_root_offset_meters=(0.0, 0.010, 0.003),
        tail_length_meters=0.020, tail_half_width_meters=0.014, tail_thickness_meters=0.008,
        wing_kinematics=WingKinematics(3.0, 0.25, 0.0, 0.0, 0.15, 0.4))
    scaling = LatticeScaling.make(bird.wing_root_chord_meters, 8, 1.0, 100.0, 1.225, 0.03)
    config = SimulationConfiguration(
        grid=GridSize(n, n, n), domain_origin_meters=(0.0, 0.0, 0.0), scaling=scaling,
        far_field_velocity_meters_per_second=(0.0, 0.0, 0.0) if free_flight else (-1.0, 0.0, 0.0),
        sponge_width_cells=4, sponge_strength=0.04, free_flight=free_flight,
        gravity_meters_per_second_squared=(0.0, 0.0, 0.0))
    half = tuple(0.5 * d for d in config.domain_size_meters)
    from .config import BirdBodyState
    state = BirdBodyState(position_meters=half,
                          linear_velocity_meters_per_second=(1.0, 0.0, 0.0) if free_flight else (0.0, 0.0, 0.0))
    return config, bird, state


# Kinematic parameters the adjoint differentiates, as (row, column) of the bird rows.
KINEMATIC_PARAMETERS = (("stroke amplitude", 5, 1), ("pitch amplitude", 6, 0), ("pitch phase", 6, 1),
                        ("deviation amplitude", 6, 2))


def kinematic_parameters(rows) -> tuple:
    """theta = (stroke amplitude, pitch amplitude, pitch phase, deviation amplitude) of bird rows."""
    return tuple(float(rows[r][c]) for _, r, c in KINEMATIC_PARAMETERS)


def with_kinematic_parameters(rows, theta):
    """Copy of the bird rows with theta written into the kinematic slots."""
    out = [tuple(r) for r in rows]
    for (name, r, c), v in zip(KINEMATIC_PARAMETERS, theta):
        row = list(out[r])
        row[c] = float(f32(v))
        out[r] = tuple(row)
    return out


def adjoint_plates(nx=96, ny=64, nz=64, span=20.0, chord=6.0, thickness=2.0, period=600.0, stroke_deg=60.0,
                   pitch_deg=45.0, deviation_deg=5.0, viscosity=0.02, storage=L.STORAGE_F32,
                   link_rule=L.LINK_LINEAR, n_chord=8, n_span=24):
    """Flapping plate pair for the adjoint: TRT, prescribed stroke / pitch /
    deviation, far-field faces."""
    return flapping_plates(nx=nx, ny=ny, nz=nz, span=span, chord=chord, thickness=thickness, n_chord=n_chord,
                           n_span=n_span, period=period, stroke_deg=stroke_deg, pitch_deg=pitch_deg,
                           viscosity=viscosity, storage=storage, link_rule=link_rule, sponge_width=6.0,
                           deviation_deg=deviation_deg)
