"""Workload builders: the lattice configurations the library is measured and
tested on, each as (bfx config, bird rows, body state, mesh).

All sizes are in lattice units (dx = dt = 1) unless a case says otherwise.
  shear_wave            periodic TRT shear-wave decay (64^3, nu 0.01, magic 1/4)
  ellipsoid_channel     RR3 channel past a stationary ellipsoid, velocity inlet,
                        zero-gradient outlet, periodic y/z, interpolated links
  flapping_plates       two rectangular flat-plate wings as a triangle mesh,
                        stroke 60 deg sin, pitch 45 deg cos, links rebuilt each step
  compact_bird          the reference's compact analytic bird on 48^3
  flapping_wing         the prescribed Li-Nabawy beta-planform wing of
                        MetalFlappingWingValidation (analytic link fractions)
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


def keyframed_plates(nx=96, ny=64, nz=64, span=16.0, chord=6.0, thickness=2.0, n_chord=6, n_span=16, frames=24,
                     frame_interval=4.0, stroke_deg=40.0, period=1000.0, jitter=0.02, seed=7, viscosity=0.02,
                     storage=L.STORAGE_F32, link_rule=L.LINK_RAY_ROOT, sponge_width=6.0):
    """A keyframe replay standing in for a measured surface sequence
    (MeasuredBirdSurfaceSequence): the two plates of flapping_plates as one
    body-fixed mesh whose vertices are given at `frames` keyframes every
    `frame_interval` seconds (one second per step here): a stroke rotation about
    the body x axis, mirrored on the right plate, plus a seeded per-vertex
    perturbation of `jitter` cells normal to the plates.  The replay
    interpolates linearly between keyframes."""
    cfg, rows, body, mesh = flapping_plates(nx=nx, ny=ny, nz=nz, span=span, chord=chord, thickness=thickness,
                                            n_chord=n_chord, n_span=n_span, period=period, stroke_deg=0.0,
                                            pitch_deg=0.0, viscosity=viscosity, storage=storage, link_rule=link_rule,
                                            sponge_width=sponge_width)
    nv = mesh["local"].shape[0] // 2
    one = mesh["local"][:nv].astype(np.float64)  # (chord, span, 0) of one plate
    root = 2.0
    rng = np.random.default_rng(seed)
    times = np.arange(frames, dtype=np.float64) * frame_interval
    pts = np.zeros((frames, 2 * nv, 3), np.float64)
    for f, t in enumerate(times):
        phi = math.radians(stroke_deg) * math.sin(2.0 * math.pi * t / period)
        for side, sign in ((0, 1.0), (1, -1.0)):
            y = sign * (root + one[:, 1])
            z = rng.uniform(-jitter, jitter, nv)
            c, s = math.cos(sign * phi), math.sin(sign * phi)
            blk = pts[f, side * nv:(side + 1) * nv]
            blk[:, 0] = one[:, 0]
            blk[:, 1] = y * c - z * s
            blk[:, 2] = y * s + z * c
    mesh = dict(mesh)
    mesh["segment"] = np.zeros(2 * nv, np.uint8)
    mesh["local"] = pts[0].astype(np.float32)
    mesh["kf_times"] = times.astype(np.float32)
    mesh["kf_points"] = pts.astype(np.float32)
    return cfg, rows, body, mesh


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


def _quad_strip(c0, c1, span, n_chord, n_span, chord_offset):
    """Triangulated trapezoid in a segment frame: chord c0 at span 0 tapering
    to c1 at `span`, leading edge at chord_offset * chord."""
    verts, tris = [], []
    for j in range(n_span + 1):
        s = span * j / n_span
        c = c0 + (c1 - c0) * j / n_span
        for i in range(n_chord + 1):
            verts.append((chord_offset * c + c * i / n_chord, s, 0.0))
    w = n_chord + 1
    for j in range(n_span):
        for i in range(n_chord):
            a = j * w + i
            tris.append((a, a + 1, a + w))
            tris.append((a + w + 1, a + w, a + 1))
    return np.asarray(verts, np.float32), np.asarray(tris, np.uint32)


def jointed_wing_mesh(spans=(24.0, 24.0, 24.0), chords=(12.0, 10.0, 8.0, 6.0), n_chord=6, n_span=8,
                      elbow=(0.0, 20.0, 0.5), wrist=(0.0, 20.0, 1.0), axis=(0.0, 0.0, 1.0)):
    """Two 3-segment flat wings (inner, middle, outer) hinged at the elbow and
    the wrist, as jointed mesh segments 1-6.  spans: segment spans; chords:
    chord at the root, elbow, wrist and tip; elbow / wrist: (bias deg,
    amplitude deg, phase rad) of the hinge angle about `axis` (segment frame;
    the default folds the wing in its own plane)."""
    verts, tris, segs, parts = [], [], [], []
    base = 0
    for side in (0, 1):
        for k in range(3):
            v, t = _quad_strip(chords[k], chords[k + 1], spans[k], n_chord, n_span, -0.25)
            verts.append(v)
            tris.append(t + base)
            seg = (1 + side) if k == 0 else (3 + 2 * (k - 1) + side)
            segs.append(np.full(v.shape[0], seg, np.uint8))
            parts.append(np.full(t.shape[0], 2 + side, np.uint8))
            base += v.shape[0]
    joints = []
    for k, (bias_deg, amp_deg, phase) in enumerate((elbow, wrist)):
        joints.append({"origin": (0.0, spans[k], 0.0), "axis": axis, "bias": math.radians(bias_deg),
                       "amplitude": math.radians(amp_deg), "phase": phase})
    return {"local": np.concatenate(verts), "segment": np.concatenate(segs), "tris": np.concatenate(tris),
            "tri_part": np.concatenate(parts), "joints": joints}


def jointed_plates(nx=96, ny=96, nz=64, spans=(10.0, 9.0, 8.0), chords=(8.0, 7.0, 6.0, 5.0), thickness=2.0,
                   period=800.0, stroke_deg=50.0, pitch_deg=30.0, viscosity=0.02, storage=L.STORAGE_F32,
                   collision=L.COLLISION_TRT, link_rule=L.LINK_LINEAR, n_chord=4, n_span=6):
    """Flapping 3-segment plate wings (elbow and wrist folding in the wing
    plane) about a fixed body point: the jointed-mesh parity case."""
    op, om = _trt_rates(viscosity, 3.0 / 16.0)
    rows = zero_bird_rows()
    rows[0] = (4.0, 4.0, 4.0, 1.0)
    rows[1] = (1.0, 1.0, 1.0, 0.0)
    rows[2] = (sum(spans), chords[0], chords[-1], thickness)
    rows[5] = (1.0 / period, float(f32(math.radians(stroke_deg))), 0.0, 0.0)
    rows[6] = (float(f32(math.radians(pitch_deg))), float(f32(math.pi / 2.0)), 0.0, 0.0)
    rows[8] = (0.0, 0.15, 0.0, 0.0)
    mesh = jointed_wing_mesh(spans, chords, n_chord, n_span, elbow=(0.0, 20.0, 0.5), wrist=(0.0, 25.0, 1.0))
    cfg = default_config(nx, ny, nz, omega_plus=op, omega_minus=om, face_bc=[L.BC_FARFIELD] * 6,
                         geometry=L.GEOMETRY_MESH, wall_rule=L.WALL_INTERPOLATED, collision=collision,
                         storage=storage, link_rule=link_rule, mesh_half_thickness=0.5 * thickness,
                         sponge_width=6.0, sponge_strength=0.05)
    body = ((nx / 2.0, ny / 2.0, nz / 2.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return cfg, rows, body, mesh


def _ellipsoid_surface(radii, n_theta, n_phi):
    """Latitude-longitude triangulation of an ellipsoid surface (body frame)."""
    verts = [(0.0, 0.0, radii[2])]
    for i in range(1, n_theta):
        th = math.pi * i / n_theta
        for j in range(n_phi):
            ph = 2.0 * math.pi * j / n_phi
            verts.append((radii[0] * math.sin(th) * math.cos(ph), radii[1] * math.sin(th) * math.sin(ph),
                          radii[2] * math.cos(th)))
    verts.append((0.0, 0.0, -radii[2]))
    tris = []
    for j in range(n_phi):
        tris.append((0, 1 + j, 1 + (j + 1) % n_phi))
    for i in range(n_theta - 2):
        r0, r1 = 1 + i * n_phi, 1 + (i + 1) * n_phi
        for j in range(n_phi):
            a, b = r0 + j, r0 + (j + 1) % n_phi
            c, d = r1 + j, r1 + (j + 1) % n_phi
            tris.append((a, c, b))
            tris.append((b, c, d))
    south = len(verts) - 1
    r0 = 1 + (n_theta - 2) * n_phi
    for j in range(n_phi):
        tris.append((r0 + j, south, r0 + (j + 1) % n_phi))
    return np.asarray(verts, np.float32), np.asarray(tris, np.uint32)


def articulated_bird(nx=768, ny=384, nz=384, storage=L.STORAGE_F16_DEVIATION, collision=L.COLLISION_RR3,
                     inflow=0.04, viscosity=0.002, sponge_width=32.0, mass_ratio=50.0, seed=5,
                     body_radii=(60.0, 18.0, 18.0), wing_spans=(50.0, 48.0, 42.0), chords=(36.0, 28.0, 20.0, 12.0),
                     resolution=1.0, free_flight=True, period=16000.0, mach_limit=0.25):
    """Synthetic articulated bird: ellipsoid body (semi-axes 60, 18, 18 cells),
    two 3-segment wings (span 140, chord 36 -> 12) hinged at shoulder / elbow /
    wrist with seeded sinusoidal joint angles, a tapered tail plate, about 150k
    triangles; inflow u_x = 0.04, nu = 0.002, RR3, sponge 32, free 6-DOF body
    with mass ratio 50 (mass = 50 x the displaced fluid mass of the body).
    The wing-beat period (16000 steps) keeps the wing tip near lattice Mach
    0.15 over the inflow (tip speed 2 pi A span / T); the safety ledger's Mach
    limit is raised to 0.25 to leave room for the joint motion."""
    rng = np.random.default_rng(seed)
    op, om = _trt_rates(viscosity, 3.0 / 16.0)
    stroke = math.radians(float(rng.uniform(50, 65)))
    n_th, n_ph = int(round(96 * resolution)), int(round(192 * resolution))
    bv, bt = _ellipsoid_surface(body_radii, n_th, n_ph)
    # tail: tapered plate behind the body (body frame), 2 cells thick, scaled
    # with the body (length 2/3 of the semi-axis, width 1/2 -> 1/5 of it)
    a0 = body_radii[0]
    tail_len = 2.0 * a0 / 3.0
    tv, tt = _quad_strip(0.5 * a0, 0.2 * a0, tail_len, max(2, int(24 * resolution)), max(2, int(32 * resolution)),
                         -0.5)
    tv = np.stack([-(tv[:, 1] + a0 - 0.1 * a0), tv[:, 0], np.zeros(len(tv))], axis=1).astype(np.float32)
    ang = lambda lo, hi: float(rng.uniform(lo, hi))
    wing = jointed_wing_mesh(wing_spans, chords, int(64 * resolution), int(140 * resolution),
                             elbow=(ang(-5, 5), ang(15, 30), ang(0.3, 0.9)),
                             wrist=(ang(-5, 5), ang(20, 35), ang(0.6, 1.4)))
    verts = np.concatenate([bv, tv, wing["local"]])
    nb, nt = len(bv), len(tv)
    tris = np.concatenate([bt, tt + nb, wing["tris"] + nb + nt])
    segs = np.concatenate([np.zeros(nb + nt, np.uint8), wing["segment"]])
    parts = np.concatenate([np.full(len(bt), 1, np.uint8), np.full(len(tt), 4, np.uint8), wing["tri_part"]])
    mesh = {"local": verts, "segment": segs, "tris": tris, "tri_part": parts, "joints": wing["joints"]}
    volume = 4.0 / 3.0 * math.pi * body_radii[0] * body_radii[1] * body_radii[2]
    mass = mass_ratio * volume
    a, b, c = body_radii
    inertia = (mass * (b * b + c * c) / 5.0, mass * (a * a + c * c) / 5.0, mass * (a * a + b * b) / 5.0)
    rows = zero_bird_rows()
    rows[0] = (float(a), float(b), float(c), float(mass))
    rows[1] = inertia + (0.0,)
    span = float(sum(wing_spans))
    rows[2] = (span, chords[0], chords[-1], 2.0)
    rows[3] = (0.0, 0.0, float(0.6 * b), 0.0)
    rows[4] = (float(tail_len), float(0.25 * a0), 2.0, 0.0)
    rows[5] = (1.0 / period, float(f32(stroke)), 0.0, 0.0)
    rows[6] = (float(f32(math.radians(ang(20, 35)))), float(f32(math.pi / 2.0)), 0.0, 0.0)
    root_y = 0.6 * b
    half = (a + tail_len, span + root_y + 1.0, span * math.sin(stroke) + b)
    rows[7] = half + (float(math.sqrt(sum(h * h for h in half))),)
    rows[8] = (float(2.0 * math.pi / period * stroke * span), float(mach_limit), 0.0, 0.0)
    cfg = default_config(nx, ny, nz, omega_plus=op, omega_minus=om,
                         face_bc=[L.BC_VELOCITY, L.BC_FARFIELD, L.BC_FARFIELD, L.BC_FARFIELD, L.BC_FARFIELD,
                                  L.BC_FARFIELD],
                         face_velocity=[(inflow, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5,
                         far_field=[inflow, 0.0, 0.0, 1.0], geometry=L.GEOMETRY_MESH,
                         wall_rule=L.WALL_INTERPOLATED, collision=collision, storage=storage,
                         link_rule=L.LINK_LINEAR, mesh_half_thickness=1.0, sponge_width=sponge_width,
                         sponge_strength=0.05, free_flight=1 if free_flight else 0)
    body = ((nx * 0.4, ny / 2.0, nz / 2.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return cfg, rows, body, mesh


# Li and Nabawy's Re = 100 beta-planform baseline as MetalFlappingWingValidator
# states it (Sources/BirdFlowMetal/MetalFlappingWingValidation.swift:535-566).
LI_NABAWY = dict(reynolds=100.0, aspect_ratio=3.0, radius_of_gyration=0.5593218135819926,
                 beta_shape=1.4891506583557845, beta_normalization=2.497931737168364,
                 stroke_half_amplitude=80.0 * math.pi / 180.0, acceleration_duration=0.25, pitch_duration=0.25,
                 pitch_low=45.0 * math.pi / 180.0, pitch_high=135.0 * math.pi / 180.0, lattice_speed=0.035,
                 horizontal_chords=10, vertical_chords=8)


def flapping_wing(chord=8, storage=L.STORAGE_F32, collision=L.COLLISION_TRT, cycle_steps=None, nx=None, ny=None,
                  nz=None, viscosity=None):
    """The validator's prescribed-wing simulation (MetalPrescribedWingSimulation,
    MetalFlappingWingValidation.swift:3312-3600 with the batchDifference grid of
    :3103-3125): a (10 c, 10 c, 8 c) lattice in lattice units, the root at
    (0.5, 0.5, 0.65) of it, one cycle of round(4 A r_g AR c / U) steps, the
    wing's radius AR c and thickness 0.05 c, Re 100 on the radius-of-gyration
    speed U, a far-field sponge of max(4, c / 2) cells at strength 0.04,
    interpolated links and the conservative moving-domain estimator (6).
    ``viscosity`` overrides the Re = 100 value (tests run faster cycles at a
    higher viscosity).  Returns (config, wing record)."""
    p = LI_NABAWY
    nx = nx or p["horizontal_chords"] * chord
    ny = ny or p["horizontal_chords"] * chord
    nz = nz or p["vertical_chords"] * chord
    if cycle_steps is None:
        travel = 4.0 * p["stroke_half_amplitude"] * p["radius_of_gyration"] * p["aspect_ratio"]
        cycle_steps = int(round(travel * chord / p["lattice_speed"]))
    if viscosity is None:
        viscosity = p["lattice_speed"] * chord / p["reynolds"]
    op, om = _trt_rates(viscosity, 3.0 / 16.0)
    cfg = default_config(nx, ny, nz, omega_plus=op, omega_minus=om, geometry=L.GEOMETRY_FLAPPING_WING,
                         wall_rule=L.WALL_INTERPOLATED, collision=collision, storage=storage,
                         sponge_strength=0.04, sponge_width=float(max(4, chord // 2)))
    max_rate = 2.0 * p["stroke_half_amplitude"] / (p["acceleration_duration"] +
                                                   2.0 * p["acceleration_duration"] / math.pi)
    w = L.FlappingWing()
    w.root_and_chord.v[:] = [float(f32(0.5 * nx)), float(f32(0.5 * ny)), float(f32(0.65) * f32(nz)), float(chord)]
    w.geometry.v[:] = [p["aspect_ratio"] * chord, 0.05 * chord, p["beta_shape"] - 1.0, p["beta_normalization"]]
    w.kinematics0.v[:] = [float(cycle_steps), p["stroke_half_amplitude"], p["acceleration_duration"],
                          p["pitch_duration"]]
    w.kinematics1.v[:] = [p["pitch_low"], p["pitch_high"], max_rate, p["lattice_speed"]]
    return cfg, w


def measured_surface_replay(surface, first=60, frames=4, cell_size=0.004, steps_per_frame=5, viscosity=0.02,
                            half_thickness_cells=0.75, margin_cells=12, storage=L.STORAGE_F32,
                            link_rule=L.LINK_LINEAR):
    """A keyframe replay of a measured bird surface sequence (bfx.measured),
    frames first ... first + frames - 1, on a lattice that covers the window's
    positions plus `margin_cells`: the body (all vertices, held at the
    sequence's body origin) with the frames' positions as body-frame offsets,
    half thickness 0.75 cells (MetalFlappingWingValidation's default measured
    half thickness), `steps_per_frame` steps per frame interval, parts 1-4 from
    the sequence's components, far-field faces."""
    mesh = surface.keyframe_mesh(first, frames)
    pts = surface.positions[first:first + frames].reshape(-1, 3).astype(np.float64)
    lo = pts.min(axis=0) - margin_cells * cell_size
    hi = pts.max(axis=0) + margin_cells * cell_size
    n = [int(math.ceil((h - l) / cell_size)) for l, h in zip(lo, hi)]
    interval = float(surface.times[first + 1] - surface.times[first])
    dt = interval / steps_per_frame
    op, om = _trt_rates(viscosity, 3.0 / 16.0)
    rho = 1.225
    cfg = default_config(n[0], n[1], n[2], origin=[float(v) for v in lo], cell_size=cell_size, time_step=dt,
                         velocity_to_lattice=dt / cell_size, force_to_physical=rho * cell_size ** 4 / dt ** 2,
                         omega_plus=op, omega_minus=om, face_bc=[L.BC_FARFIELD] * 6, geometry=L.GEOMETRY_MESH,
                         wall_rule=L.WALL_INTERPOLATED, storage=storage, link_rule=link_rule,
                         mesh_half_thickness=half_thickness_cells * cell_size, sponge_width=4.0,
                         sponge_strength=0.02)
    rows = zero_bird_rows()
    rows[0] = (0.05, 0.03, 0.03, 0.3)
    rows[1] = (1e-4, 1e-4, 1e-4, 0.0)
    rows[8] = (0.0, 0.15, 0.0, 0.0)
    body = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return cfg, rows, body, mesh
