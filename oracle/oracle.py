"""ctypes wrapper of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
may import this module, as the checker.  The product (the CUDA library and
its Python host mirror) never imports it.

The oracle restates the BirdFlowMetal hot path on the CPU (see
``bfx_oracle.h`` for the reference file:line map).  ``OracleSim`` drives it
the way ``BirdFlowSimulation.encodeBatch`` (Sources/BirdFlowMetal/
BirdFlowSimulation.swift:1359-1449) drives the Metal kernels: A/B population
buffers, prepare -> classify -> links -> fused step -> reduce -> integrate ->
safety -> swap.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

BC_FARFIELD, BC_PERIODIC, BC_VELOCITY, BC_OUTFLOW = 0, 1, 2, 3
COLLISION_TRT, COLLISION_TRT_LIMITER, COLLISION_REGULARIZED, COLLISION_RR3 = 0, 1, 2, 3


def build() -> str:
    """Compiles liboracle.so with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Params(ct.Structure):
    _fields_ = [
        ("nx", ct.c_int32), ("ny", ct.c_int32), ("nz", ct.c_int32), ("_pad0", ct.c_int32),
        ("origin", ct.c_float * 3), ("dx", ct.c_float),
        ("time", ct.c_float), ("dt", ct.c_float), ("v2l", ct.c_float), ("f2p", ct.c_float),
        ("omega_p", ct.c_float), ("omega_m", ct.c_float),
        ("sponge_strength", ct.c_float), ("sponge_width", ct.c_float),
        ("far", ct.c_float * 4), ("gravity", ct.c_float * 3),
        ("accumulate_loads", ct.c_int32), ("interpolated", ct.c_int32), ("collision", ct.c_int32),
        ("load_component", ct.c_int32), ("force_mode", ct.c_int32), ("selected_part", ct.c_int32),
        ("free_flight", ct.c_int32), ("capture_fields", ct.c_int32), ("has_prev_geom", ct.c_int32),
        ("face_bc", ct.c_int32 * 6), ("face_velocity", (ct.c_float * 3) * 6),
        ("substeps", ct.c_int32), ("local_density", ct.c_int32), ("_pad1", ct.c_int32), ("_pad2", ct.c_int32),
    ]


class Loads(ct.Structure):
    _fields_ = [
        ("f64_force_lattice", ct.c_double * 3), ("f64_force", ct.c_double * 3),
        ("f64_torque", ct.c_double * 3), ("activation", ct.c_double), ("max_restriction", ct.c_double),
        ("f32_force", ct.c_float * 4), ("f32_torque", ct.c_float * 4),
        ("link_count", ct.c_int64), ("covered_count", ct.c_int64), ("uncovered_count", ct.c_int64),
    ]


class F4(ct.Structure):
    _fields_ = [("v", ct.c_float * 4)]


class Bird(ct.Structure):
    _fields_ = [(name, F4) for name in (
        "body_radii_mass", "inertia", "wing_geometry0", "wing_geometry1", "tail_geometry",
        "wing_kinematics0", "wing_kinematics1", "safety_geometry", "safety_limits",
        "left_wing_mass_com", "left_wing_inertia", "right_wing_mass_com", "right_wing_inertia")]


class Prepared(ct.Structure):
    _fields_ = [(name, F4) for name in (
        "body_position", "orientation", "linear_velocity", "omega_body_world",
        "left_root", "left_chord", "left_span", "left_normal", "left_angular_velocity",
        "right_root", "right_chord", "right_span", "right_normal", "right_angular_velocity")]


class Wing(ct.Structure):
    _fields_ = [(name, F4) for name in ("root_and_chord", "geometry", "kinematics0", "kinematics1")]


class WingPrepared(ct.Structure):
    _fields_ = [(name, F4) for name in ("root", "chord", "span", "normal", "angular_velocity", "state")]


class BodyF32(ct.Structure):
    _fields_ = [("position", ct.c_float * 3), ("orientation", ct.c_float * 4),
                ("velocity", ct.c_float * 3), ("omega_body", ct.c_float * 3)]


class BodyF64(ct.Structure):
    _fields_ = [("position", ct.c_double * 3), ("orientation", ct.c_double * 4),
                ("velocity", ct.c_double * 3), ("omega_body", ct.c_double * 3)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ct.CDLL(_LIB_PATH)
        P = ct.POINTER
        fp, u8p, dp = P(ct.c_float), P(ct.c_uint8), P(ct.c_double)
        L.or_equilibrium.restype = ct.c_float
        L.or_equilibrium.argtypes = [ct.c_int, ct.c_float, fp]
        L.or_collide_regularized.argtypes = [ct.c_int, fp, ct.c_float, ct.c_int, fp, fp, fp]
        L.or_trt_collision.argtypes = [fp, ct.c_float, fp, ct.c_float, ct.c_float, fp]
        L.or_init_equilibrium.argtypes = [P(Params), fp, u8p, fp, fp, fp]
        L.or_init_shear_wave.argtypes = [P(Params), ct.c_float, ct.c_int, fp, fp, fp]
        L.or_macroscopic.argtypes = [P(Params), fp, fp, fp]
        L.or_step.argtypes = [P(Params), fp, fp, u8p, u8p, fp, fp, fp, fp, fp, dp, P(Loads), fp]
        L.or_fluid_mass_momentum.argtypes = [P(Params), fp, u8p, dp]
        L.or_prepare_bird.argtypes = [P(Bird), P(BodyF32), ct.c_float, ct.c_float, P(Prepared)]
        L.or_build_bird.argtypes = [P(Params), P(Bird), P(Prepared), u8p, u8p, fp]
        L.or_build_ellipsoid.argtypes = [P(Params), P(Bird), P(Prepared), u8p, u8p, fp]
        L.or_prepare_wing.argtypes = [P(Wing), ct.c_float, P(WingPrepared)]
        L.or_build_wing.argtypes = [P(Params), P(Wing), P(WingPrepared), u8p, u8p, fp]
        L.or_wing_link_fraction.restype = ct.c_float
        L.or_wing_link_fraction.argtypes = [P(Params), P(Wing), P(WingPrepared)] + [ct.c_int] * 4
        L.or_wing_violation.restype = ct.c_float
        L.or_wing_violation.argtypes = [P(Params), P(Wing), P(WingPrepared), fp]
        L.or_wing_link_fractions.argtypes = [P(Params), P(Wing), P(WingPrepared), P(ct.c_uint32), u8p, ct.c_int64, fp]
        L.or_ledger_sources.argtypes = [P(Params), fp, fp, u8p, u8p, fp, dp]
        L.or_powf.restype = ct.c_float
        L.or_powf.argtypes = [ct.c_float, ct.c_float]
        L.or_ellipsoid_link_fraction.restype = ct.c_float
        L.or_ellipsoid_link_fraction.argtypes = [P(Params), P(Bird), P(Prepared)] + [ct.c_int] * 6
        L.or_write_links.restype = ct.c_int64
        L.or_write_links.argtypes = [P(Params), ct.c_int, P(Bird), P(Prepared), fp, P(ct.c_uint32), ct.c_uint32,
                                     ct.c_float, P(ct.c_uint64), fp, u8p, u8p, fp, fp]
        L.or_enumerate_links.restype = ct.c_int64
        L.or_enumerate_links.argtypes = [P(Params), u8p, u8p, P(ct.c_uint32), u8p, ct.c_int64]
        L.or_mesh_prepare_articulated.argtypes = [P(Prepared), fp, u8p, ct.c_uint32, ct.c_float, fp, fp]
        L.or_mesh_prepare_keyframes.argtypes = [P(Prepared), fp, ct.c_uint32, fp, ct.c_uint32, ct.c_float, ct.c_float,
                                                fp, fp]
        L.or_prepare_segments.argtypes = [P(Bird), P(Prepared), fp, ct.c_int, ct.c_float, fp]
        L.or_mesh_prepare_segments.argtypes = [P(Prepared), fp, fp, u8p, ct.c_uint32, ct.c_float, fp, fp]
        L.or_mesh_rasterize.argtypes = [P(Params), fp, P(ct.c_uint32), ct.c_uint32, ct.c_float, P(ct.c_uint64)]
        L.or_mesh_resolve.argtypes = [P(Params), fp, fp, P(ct.c_uint32), u8p, ct.c_uint32, ct.c_float,
                                      P(ct.c_uint64), u8p, fp]
        L.or_mesh_ray_root.restype = ct.c_float
        L.or_mesh_ray_root.argtypes = [P(Params), fp, P(ct.c_uint32), ct.c_uint32, ct.c_float, P(ct.c_uint64)] + [ct.c_int] * 6
        L.or_integrate_body_f32.argtypes = [P(BodyF32), P(Bird), fp, fp, fp, ct.c_float, ct.c_int]
        L.or_integrate_body_f64.argtypes = [P(BodyF64), P(Bird), dp, dp, dp, ct.c_double, ct.c_int]
        L.or_rigid_body_swift_f32.argtypes = [P(BodyF32), ct.c_float, fp, fp, fp, fp, ct.c_float, ct.c_int]
        L.or_wing_reaction.argtypes = [P(Prepared), P(Bird), ct.c_float, ct.c_int, fp, fp]
        L.or_safety.argtypes = [P(BodyF32), P(Bird), P(Params), ct.c_uint32, ct.c_uint32, fp, P(ct.c_uint32)]
        L.or_link_fraction.restype = ct.c_double
        L.or_link_fraction.argtypes = [ct.c_double, ct.c_double]
        L.or_interpolated_population.restype = ct.c_double
        L.or_interpolated_population.argtypes = [ct.c_double] * 5
        L.or_uncovered_impulse.argtypes = [dp, dp, dp, dp, ct.c_int, dp]
        _lib = L
    return _lib


def _p(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ct.POINTER(ctype))


def fptr(a):
    return _p(a, ct.c_float)


def u8ptr(a):
    return _p(a, ct.c_uint8)


def dptr(a):
    return _p(a, ct.c_double)


def make_params(nx, ny, nz, *, dx=1.0, origin=(0.0, 0.0, 0.0), dt=1.0, v2l=1.0, f2p=1.0,
                omega_p=1.0, omega_m=1.0, sponge_strength=0.0, sponge_width=4.0,
                far=(0.0, 0.0, 0.0, 1.0), gravity=(0.0, 0.0, 0.0), accumulate_loads=True,
                interpolated=False, collision=COLLISION_TRT, load_component=0, force_mode=6,
                selected_part=0, free_flight=False, capture_fields=False, has_prev_geom=True,
                face_bc=(BC_FARFIELD,) * 6, face_velocity=None, substeps=1, local_density=False,
                time=0.0) -> Params:
    p = Params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.origin[:] = list(origin)
    p.dx = dx
    p.time, p.dt, p.v2l, p.f2p = time, dt, v2l, f2p
    p.omega_p, p.omega_m = omega_p, omega_m
    p.sponge_strength, p.sponge_width = sponge_strength, sponge_width
    p.far[:] = list(far)
    p.gravity[:] = list(gravity)
    p.accumulate_loads = int(accumulate_loads)
    p.interpolated = int(interpolated)
    p.collision = collision
    p.load_component, p.force_mode, p.selected_part = load_component, force_mode, selected_part
    p.free_flight, p.capture_fields, p.has_prev_geom = int(free_flight), int(capture_fields), int(has_prev_geom)
    p.face_bc[:] = list(face_bc)
    if face_velocity is not None:
        for i in range(6):
            p.face_velocity[i][:] = list(face_velocity[i])
    p.substeps, p.local_density = substeps, int(local_density)
    return p


def bird_from_dict(d: dict) -> Bird:
    b = Bird()
    for name, _ in Bird._fields_:
        v = d.get(name, (0.0, 0.0, 0.0, 0.0))
        getattr(b, name).v[:] = list(v)
    return b


def prepared_to_array(prep: Prepared) -> np.ndarray:
    return np.array([list(getattr(prep, n).v) for n, _ in Prepared._fields_], dtype=np.float32)


def equilibrium(q: int, rho: float, u) -> float:
    u = np.asarray(u, dtype=np.float32)
    return lib().or_equilibrium(q, rho, fptr(u))


def collide_regularized(f, omega_p: float, rr3: bool, order: int):
    """One regularized / RR3 collision of 19 populations: order 0 = the
    reference's literal per-direction form, 1 = the pair order the stepping
    uses.  Returns (post, activation, restriction)."""
    f = np.ascontiguousarray(f, dtype=np.float32)
    post = np.zeros(19, np.float32)
    act = np.zeros(1, np.float32)
    res = np.zeros(1, np.float32)
    lib().or_collide_regularized(order, fptr(f), omega_p, 1 if rr3 else 0, fptr(post), fptr(act), fptr(res))
    return post, float(act[0]), float(res[0])


def lattice():
    c = np.zeros((19, 3), np.int32)
    opp = np.zeros(19, np.int32)
    w = np.zeros(19, np.float32)
    lib().or_lattice(c.ctypes.data_as(ct.POINTER(ct.c_int32)), opp.ctypes.data_as(ct.POINTER(ct.c_int32)), fptr(w))
    return c, opp, w


class OracleSim:
    """CPU restatement of one simulation: A/B populations, masks, wall field.

    geometry: None (all fluid), "bird" (analytic bird, halfway links),
    "ellipsoid" (body ellipsoid, interpolated bisection links), "mesh"
    (articulated triangle mesh; link_rule "linear" or "ray") or "wing" (the
    prescribed flapping wing of ``wing``, held at its root).
    """

    def __init__(self, params: Params, *, geometry=None, bird: Bird | None = None,
                 body=None, body_f64=True, mesh=None, link_rule="linear", shear=None, wing: Wing | None = None):
        self.p = params
        self.n = params.nx * params.ny * params.nz
        n = self.n
        self.geometry = geometry
        self.wing = wing
        self.wing_prep = WingPrepared()
        self._absolute = 0
        if geometry == "wing":
            body = (tuple(wing.root_and_chord.v[:3]), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
        self.bird = bird
        self.mesh = mesh
        self.link_rule = link_rule
        self.body_f64 = body_f64
        self.pa = np.zeros(19 * n, np.float32)
        self.pb = np.zeros(19 * n, np.float32)
        self.mcur = np.zeros(n, np.uint8)
        self.mnext = np.zeros(n, np.uint8)
        self.wall = np.zeros(4 * n, np.float32)
        self.covered = np.zeros(4 * n, np.float32)
        self.density = np.ones(n, np.float32)
        self.velocity = np.zeros(4 * n, np.float32)
        self.keys = None
        self.prep = Prepared()
        self.body32 = BodyF32()
        self.body64 = BodyF64()
        if body is not None:
            pos, orient, vel, omega = body
            self.body64.position[:] = list(pos)
            self.body64.orientation[:] = list(orient)
            self.body64.velocity[:] = list(vel)
            self.body64.omega_body[:] = list(omega)
        else:
            self.body64.orientation[:] = [0.0, 0.0, 0.0, 1.0]
        self._sync_body32()
        self.step_index = 0
        self.loads = Loads()
        self.load_history = []
        self.safety_metrics = np.array([0.0, np.inf, 0.0, 0.0], np.float32)
        self.safety_event = np.zeros(4, np.uint32)
        self.wing_prev = np.zeros(16, np.float32)
        self.wing_reaction = np.zeros(16, np.float32)
        L = lib()
        if geometry is None:
            if shear is not None:
                amplitude, axis = shear
                L.or_init_shear_wave(ct.byref(self.p), amplitude, axis, fptr(self.pa), fptr(self.density),
                                     fptr(self.velocity))
            else:
                L.or_init_equilibrium(ct.byref(self.p), fptr(self.pa), u8ptr(self.mcur), fptr(self.wall),
                                      fptr(self.density), fptr(self.velocity))
        else:
            hp = self.p.has_prev_geom
            self.p.has_prev_geom = 0
            self._geometry(0.0, self.mcur, init=True)
            self.p.has_prev_geom = hp
            L.or_init_equilibrium(ct.byref(self.p), fptr(self.pa), u8ptr(self.mcur), fptr(self.wall),
                                  fptr(self.density), fptr(self.velocity))

    def _sync_body32(self):
        for k in range(3):
            self.body32.position[k] = self.body64.position[k]
            self.body32.velocity[k] = self.body64.velocity[k]
            self.body32.omega_body[k] = self.body64.omega_body[k]
        for k in range(4):
            self.body32.orientation[k] = self.body64.orientation[k]

    def _geometry(self, time: float, target: np.ndarray, init: bool = False):
        L = lib()
        if self.geometry == "wing":
            # the validator's time is the absolute step index (MetalFlappingWingValidation.swift:3631-3634)
            L.or_prepare_wing(ct.byref(self.wing), float(0 if init else self._absolute), ct.byref(self.wing_prep))
            L.or_build_wing(ct.byref(self.p), ct.byref(self.wing), ct.byref(self.wing_prep), u8ptr(self.mcur),
                            u8ptr(target), fptr(self.wall))
            if target is not self.mcur:
                L.or_write_links(ct.byref(self.p), 3, ct.cast(ct.byref(self.wing), ct.POINTER(Bird)),
                                 ct.cast(ct.byref(self.wing_prep), ct.POINTER(Prepared)), None, None, 0, 0.0, None,
                                 fptr(self.pa), u8ptr(self.mcur), u8ptr(target), fptr(self.wall), fptr(self.covered))
            return
        L.or_prepare_bird(ct.byref(self.bird), ct.byref(self.body32), time, self.p.dx, ct.byref(self.prep))
        if self.bird.left_wing_inertia.v[3] >= 0.5:
            L.or_wing_reaction(ct.byref(self.prep), ct.byref(self.bird), self.p.dt, int(init),
                               fptr(self.wing_prev), fptr(self.wing_reaction))
        if self.geometry == "bird":
            L.or_build_bird(ct.byref(self.p), ct.byref(self.bird), ct.byref(self.prep), u8ptr(self.mcur),
                            u8ptr(target), fptr(self.wall))
        elif self.geometry == "ellipsoid":
            L.or_build_ellipsoid(ct.byref(self.p), ct.byref(self.bird), ct.byref(self.prep), u8ptr(self.mcur),
                                 u8ptr(target), fptr(self.wall))
            if target is not self.mcur:
                L.or_write_links(ct.byref(self.p), 0, ct.byref(self.bird), ct.byref(self.prep), None, None, 0, 0.0,
                                 None, fptr(self.pa), u8ptr(self.mcur), u8ptr(target), fptr(self.wall),
                                 fptr(self.covered))
        elif self.geometry == "mesh":
            m = self.mesh
            nv = m["local"].shape[0]
            self.mesh_pos = np.zeros(4 * nv, np.float32)
            self.mesh_vel = np.zeros(4 * nv, np.float32)
            joints = m.get("joints") or []
            if m.get("kf_times") is not None:
                L.or_mesh_prepare_keyframes(ct.byref(self.prep), fptr(m["kf_times"]), len(m["kf_times"]),
                                            fptr(m["kf_points"]), nv, time, self.p.v2l, fptr(self.mesh_pos),
                                            fptr(self.mesh_vel))
            elif joints:
                # or_joint: origin[3], axis[3], bias, amplitude, phase, reserved
                jarr = np.array([list(j["origin"]) + list(j["axis"]) + [j["bias"], j["amplitude"], j["phase"], 0.0]
                                 for j in joints], dtype=np.float32).ravel()
                segs = np.zeros(4 * 24, np.float32)
                L.or_prepare_segments(ct.byref(self.bird), ct.byref(self.prep), fptr(jarr), len(joints), time,
                                      fptr(segs))
                L.or_mesh_prepare_segments(ct.byref(self.prep), fptr(segs), fptr(m["local"]), u8ptr(m["segment"]),
                                           nv, self.p.v2l, fptr(self.mesh_pos), fptr(self.mesh_vel))
            else:
                L.or_mesh_prepare_articulated(ct.byref(self.prep), fptr(m["local"]), u8ptr(m["segment"]), nv,
                                              self.p.v2l, fptr(self.mesh_pos), fptr(self.mesh_vel))
            self.keys = np.full(self.n, np.iinfo(np.uint64).max, np.uint64)
            ntri = m["tris"].shape[0]
            tris = m["tris"].astype(np.uint32).ravel()
            L.or_mesh_rasterize(ct.byref(self.p), fptr(self.mesh_pos), tris.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                                ntri, m["half_thickness"], self.keys.ctypes.data_as(ct.POINTER(ct.c_uint64)))
            target[:] = 0
            self.wall[:] = 0.0
            self.wall[3::4] = 16.0
            L.or_mesh_resolve(ct.byref(self.p), fptr(self.mesh_pos), fptr(self.mesh_vel),
                              tris.ctypes.data_as(ct.POINTER(ct.c_uint32)), u8ptr(m["tri_part"]), ntri,
                              m["half_thickness"], self.keys.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                              u8ptr(target), fptr(self.wall))
            if target is not self.mcur and self.p.interpolated:
                kind = 1 if self.link_rule == "linear" else 2
                L.or_write_links(ct.byref(self.p), kind, None, None, fptr(self.mesh_pos),
                                 tris.ctypes.data_as(ct.POINTER(ct.c_uint32)), ntri, m["half_thickness"],
                                 self.keys.ctypes.data_as(ct.POINTER(ct.c_uint64)), fptr(self.pa),
                                 u8ptr(self.mcur), u8ptr(target), fptr(self.wall), fptr(self.covered))

    def step(self, capture_fields=False, per_cell_loads=False, ledger=False):
        """One step; with ``ledger`` the step's coupled-momentum ledger sums
        (or_ledger_sources) are left in ``self.ledger``."""
        L = lib()
        self.p.capture_fields = int(capture_fields)
        absolute = self.step_index + 1
        self._absolute = absolute
        time = np.float32(float(absolute) * float(self.p.dt))
        self.p.time = float(time)
        if self.geometry is not None:
            self._geometry(float(time), self.mnext)
        else:
            self.mnext[:] = self.mcur
        body_f = np.array(list(self.body32.position), np.float32)
        body_d = np.array(list(self.body64.position), np.float64)
        pcl = np.zeros(8 * self.n, np.float32) if per_cell_loads else None
        L.or_step(ct.byref(self.p), fptr(self.pa), fptr(self.pb), u8ptr(self.mcur), u8ptr(self.mnext),
                  fptr(self.wall), fptr(self.covered), fptr(self.density), fptr(self.velocity), fptr(body_f),
                  dptr(body_d), ct.byref(self.loads), fptr(pcl))
        if ledger:
            self.ledger = np.zeros(24, np.float64)
            L.or_ledger_sources(ct.byref(self.p), fptr(self.pa), fptr(self.pb), u8ptr(self.mcur), u8ptr(self.mnext),
                                fptr(self.wall), dptr(self.ledger))
        self.load_history.append((np.array(self.loads.f64_force), np.array(self.loads.f64_torque)))
        if self.p.free_flight:
            force = np.array(self.loads.f64_force, np.float64)
            torque = np.array(self.loads.f64_torque, np.float64)
            force = force + self.wing_reaction[0:3].astype(np.float64) + self.wing_reaction[8:11].astype(np.float64)
            torque = torque + self.wing_reaction[4:7].astype(np.float64) + self.wing_reaction[12:15].astype(np.float64)
            grav = np.array(list(self.p.gravity), np.float64)
            L.or_integrate_body_f64(ct.byref(self.body64), ct.byref(self.bird), dptr(force), dptr(torque), dptr(grav),
                                    float(self.p.dt), self.p.substeps)
            self._sync_body32()
            L.or_safety(ct.byref(self.body32), ct.byref(self.bird), ct.byref(self.p), absolute & 0xFFFFFFFF,
                        absolute >> 32, fptr(self.safety_metrics),
                        self.safety_event.ctypes.data_as(ct.POINTER(ct.c_uint32)))
        self.pa, self.pb = self.pb, self.pa
        self.mcur, self.mnext = self.mnext, self.mcur
        self.step_index += 1
        return pcl

    def advance(self, steps: int, **kw):
        for _ in range(steps):
            self.step(**kw)

    def populations(self) -> np.ndarray:
        return self.pa.reshape(19, self.p.nz, self.p.ny, self.p.nx)

    def macroscopic(self):
        rho = np.zeros(self.n, np.float32)
        vel = np.zeros(4 * self.n, np.float32)
        lib().or_macroscopic(ct.byref(self.p), fptr(self.pa), fptr(rho), fptr(vel))
        return rho, vel.reshape(-1, 4)[:, :3]

    def fluid_mass_momentum(self):
        out = np.zeros(4, np.float64)
        lib().or_fluid_mass_momentum(ct.byref(self.p), fptr(self.pa), u8ptr(self.mcur), dptr(out))
        return out
