"""CPU oracle pinned against the reference: golden vectors from
Reference/shear_wave_reference.py (tests/golden/make_golden.py) and the
known-answer tests of the reference's Swift test suite."""
from __future__ import annotations

import ctypes as ct
import json
import math
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def trt_rates(nu, magic):
    f = np.float32
    tp = f(0.5) + f(3) * f(nu)
    tm = f(0.5) + f(magic) / (tp - f(0.5))
    return float(f(1) / tp), float(f(1) / tm)


def shear_sim(n, nu, magic, amplitude=0.01, axis=1):
    op, om = trt_rates(nu, magic)
    p = O.make_params(n, n, n, omega_p=op, omega_m=om, face_bc=(O.BC_PERIODIC,) * 6, accumulate_loads=False)
    return O.OracleSim(p, shear=(amplitude, axis))


def mode_amplitude(sim, n, axis=1):
    _, vel = sim.macroscopic()
    ux = vel[:, 0].reshape(n, n, n)  # [z, y, x]
    prof = ux.mean(axis=(0, 2)) if axis == 1 else ux.mean(axis=(1, 2))
    c = np.arange(n)
    return float(2.0 * np.dot(prof, np.sin(2 * np.pi * c / n)) / n)


def test_oracle_matches_numpy_reference_populations():
    """Metal-vs-CPU gate of MetalShearWaveValidation.swift:56-63: max |df| < 5e-6."""
    g = np.load(os.path.join(GOLDEN, "shear_wave_ref_n12_s8.npz"))
    ref = g["populations"]  # [q, x, y, z], FP64
    sim = shear_sim(12, 0.03, 3.0 / 16.0)
    sim.advance(int(g["steps"]))
    pops = sim.populations().transpose(0, 3, 2, 1).astype(np.float64)
    assert np.max(np.abs(pops - ref)) < 5e-6


def test_oracle_decay_and_mass_match_reference_metrics():
    m = json.load(open(os.path.join(GOLDEN, "shear_wave_ref_metrics.json")))
    d = m["default_case"]
    n, steps = d["resolution"], d["steps"]
    sim = shear_sim(n, d["viscosity"], 3.0 / 16.0)
    mass0 = float(sim.pa.astype(np.float64).sum())
    a0 = mode_amplitude(sim, n)
    sim.advance(steps)
    a = mode_amplitude(sim, n)
    analytic = a0 * math.exp(-d["viscosity"] * (2 * math.pi / n) ** 2 * steps)
    err = abs(a - analytic) / analytic
    mass = float(sim.pa.astype(np.float64).sum())
    assert err < 0.03
    assert abs(err - d["relative_decay_error"]) < 2e-4
    assert abs(a - d["measured_amplitude"]) < 2e-6
    assert abs(mass - mass0) / mass0 < 5e-6


def test_oracle_convergence_order():
    """Reference/shear_wave_convergence.py: order >= 1.8 on 12/16/24/32."""
    m = json.load(open(os.path.join(GOLDEN, "shear_wave_ref_metrics.json")))
    errs, hs = [], []
    for row in m["ladder"]:
        n, steps = row["resolution"], row["steps"]
        sim = shear_sim(n, 0.03, 3.0 / 16.0)
        a0 = mode_amplitude(sim, n)
        sim.advance(steps)
        a = mode_amplitude(sim, n)
        analytic = a0 * math.exp(-0.03 * (2 * math.pi / n) ** 2 * steps)
        errs.append(abs(a - analytic) / analytic)
        hs.append(1.0 / n)
        assert abs(errs[-1] - row["relative_decay_error"]) < 2e-4
    order = float(np.polyfit(np.log(hs), np.log(errs), 1)[0])
    assert order >= 1.8
    assert abs(order - m["estimated_order"]) < 0.05


# ---- D3Q19Tests.swift:4-45 -------------------------------------------------
def test_equilibrium_recovers_density_and_velocity():
    rho, u = 1.037, (0.041, -0.017, 0.009)
    c, _, _ = O.lattice()
    f = np.array([O.equilibrium(q, rho, u) for q in range(19)], np.float64)
    assert abs(f.sum() - rho) < 1e-6
    assert np.linalg.norm((f[:, None] * c).sum(0) / f.sum() - np.array(u)) < 1e-6


def test_trt_leaves_equilibrium_unchanged():
    rho, u = 0.996, np.array([0.025, 0.006, -0.013], np.float32)
    eq = np.array([O.equilibrium(q, rho, u) for q in range(19)], np.float32)
    out = np.zeros(19, np.float32)
    O.lib().or_trt_collision(O.fptr(eq), rho, O.fptr(u), 1.7, 0.31, O.fptr(out))
    assert np.max(np.abs(out - eq)) < 1e-7


def test_directions_and_opposites_are_consistent():
    c, opp, w = O.lattice()
    for q in range(19):
        assert opp[opp[q]] == q
        assert np.array_equal(c[opp[q]], -c[q])
        assert w[opp[q]] == w[q]
    assert abs(float(w.astype(np.float64).sum()) - 1.0) < 1e-6


# ---- MetalExecutionTests.swift:2245-2316 (interpolated BB known answers) ------
def test_interpolated_bounce_back_known_answers():
    L = O.lib()
    corr, refl, far, prev = 0.07, 0.31, 0.19, 0.23
    assert abs(L.or_interpolated_population(0.5, refl, far, prev, corr) - (refl + corr)) < 1e-15
    assert abs(L.or_interpolated_population(0.25, refl, far, prev, corr) - (0.5 * refl + 0.5 * far + corr)) < 1e-15
    assert abs(L.or_interpolated_population(0.75, refl, far, prev, corr) - ((refl + corr) / 1.5 + prev / 3)) < 1e-15
    assert abs(L.or_link_fraction(0.25, -0.75) - 0.25) < 1e-15


def test_moving_domain_uncovered_impulse_known_answer():
    refill = np.array([1.0, 2.0, 3.0])
    dirs = np.array([[1.0, 0, 0], [0, 1.0, 0]]).ravel()
    old = np.array([0.2, 0.1])
    sup = np.array([0.3, 0.4])
    out = np.zeros(3)
    O.lib().or_uncovered_impulse(O.dptr(refill), O.dptr(dirs), O.dptr(old), O.dptr(sup), 2, O.dptr(out))
    assert np.array_equal(out, np.array([-1.5, -2.5, -3.0]))


# ---- rigid body: RigidBody.swift:88-126 vs integrateBirdBody restatement -----
def _bird_for_body():
    b = O.Bird()
    b.body_radii_mass.v[:] = [0.015, 0.011, 0.012, 0.025]
    b.inertia.v[:] = [0.000004, 0.000007, 0.000008, 0.0]
    return b


@pytest.mark.parametrize("substeps", [1, 4])
def test_rigid_body_integrators_agree(substeps):
    """The GPU-kernel restatement (FP32 and FP64) agrees with the Swift CPU
    integrator within the reference's 1e-6 gate (MetalExecutionTests.swift:594-688)."""
    bird = _bird_for_body()
    half = 0.5 * 0.31
    ax = np.array([0.2, 0.7, -0.1], np.float32)
    ax = ax / np.float32(np.sqrt(np.dot(ax, ax)))
    q0 = [float(ax[0] * np.sin(half)), float(ax[1] * np.sin(half)), float(ax[2] * np.sin(half)), float(np.cos(half))]
    force = np.array([0.03, -0.01, 0.02], np.float32)
    torque = np.array([0.00001, -0.00002, 0.000015], np.float32)
    grav = np.zeros(3, np.float32)
    dt = 0.0005
    a = O.BodyF32()
    a.position[:] = [0.1, 0.2, 0.3]
    a.orientation[:] = q0
    a.velocity[:] = [0.8, -0.1, 0.05]
    a.omega_body[:] = [0.3, -0.2, 0.1]
    b = O.BodyF32()
    ct.pointer(b)[0] = a
    c = O.BodyF64()
    c.position[:] = list(a.position)
    c.orientation[:] = list(a.orientation)
    c.velocity[:] = list(a.velocity)
    c.omega_body[:] = list(a.omega_body)
    L = O.lib()
    L.or_integrate_body_f32(ct.byref(a), ct.byref(bird), O.fptr(force), O.fptr(torque), O.fptr(grav), dt, substeps)
    inertia = np.array(bird.inertia.v[:3], np.float32)
    L.or_rigid_body_swift_f32(ct.byref(b), bird.body_radii_mass.v[3], O.fptr(inertia), O.fptr(force),
                              O.fptr(torque), O.fptr(grav), dt, substeps)
    fd, td, gd = force.astype(np.float64), torque.astype(np.float64), grav.astype(np.float64)
    L.or_integrate_body_f64(ct.byref(c), ct.byref(bird), O.dptr(fd), O.dptr(td), O.dptr(gd), dt, substeps)
    for name in ("position", "velocity", "omega_body", "orientation"):
        va, vb, vc = (np.array(list(getattr(x, name)), np.float64) for x in (a, b, c))
        assert np.max(np.abs(va - vb)) < 1e-6, name
        assert np.max(np.abs(vc - vb)) < 1e-6, name


def test_safety_ledger_records_first_mach_violation():
    """metalRuntimeSafetyLedgerRecordsExactFirstMachViolation (MetalExecutionTests.swift:690-736)."""
    bird = _bird_for_body()
    bird.safety_geometry.v[:] = [0.05, 0.05, 0.05, 0.07]
    bird.safety_limits.v[:] = [0.5, 0.15, 0.0, 0.0]
    p = O.make_params(48, 48, 48, dx=0.0025, v2l=0.075, sponge_width=4.0)
    body = O.BodyF32()
    body.position[:] = [0.06, 0.06, 0.06]
    body.orientation[:] = [0, 0, 0, 1]
    body.velocity[:] = [100.0, 0.0, 0.0]
    metrics = np.array([0.0, np.inf, 0.0, 0.0], np.float32)
    event = np.zeros(4, np.uint32)
    O.lib().or_safety(ct.byref(body), ct.byref(bird), ct.byref(p), 42, 0, O.fptr(metrics),
                      event.ctypes.data_as(ct.POINTER(ct.c_uint32)))
    assert event[0] == 42 and (event[2] & 1) and metrics[0] > 0.15


def test_oracle_twins_of_every_case_step():
    """Every workload builder produces an oracle twin that advances (CPU)."""
    import bfx.cases as cases
    from helpers import oracle_twin
    for cfg, rows, body, mesh in (
        cases.ellipsoid_channel(nx=32, ny=16, nz=16, radii=(5.0, 3.0, 3.0)),
        cases.flapping_plates(nx=48, ny=32, nz=32, span=8.0, chord=4.0, n_chord=4, n_span=8, period=100.0,
                              sponge_width=4.0),
    ):
        osim = oracle_twin(cfg, rows, body, mesh)
        osim.advance(2)
        assert np.all(np.isfinite(osim.pa))
        assert osim.mcur.any()


def test_jointed_wing_chain_stays_connected_at_the_joints():
    """Elbow and wrist frames (or_prepare_segments): the joint point of each
    segment coincides with the matching point of its parent at every phase, and
    the chain mirrors between the wings."""
    import bfx.cases as cases
    from helpers import oracle_twin
    spans, chords = (10.0, 9.0, 8.0), (8.0, 7.0, 6.0, 5.0)
    cfg, rows, body, mesh = cases.jointed_plates(nx=96, ny=96, nz=64, spans=spans, chords=chords, n_chord=4,
                                                 n_span=6)
    osim = oracle_twin(cfg, rows, body, mesh)
    local, seg = mesh["local"], mesh["segment"]
    for steps in (0, 37, 150):
        osim.advance(steps)
        pos = osim.mesh_pos.reshape(-1, 4)[:, :3]
        for side in (0, 1):
            chain = [1 + side, 3 + side, 5 + side]
            for k in range(2):
                parent, child = chain[k], chain[k + 1]
                tip = np.where((seg == parent) & np.isclose(local[:, 1], spans[k]) & np.isclose(local[:, 0], 0.0))[0]
                root = np.where((seg == child) & np.isclose(local[:, 1], 0.0) & np.isclose(local[:, 0], 0.0))[0]
                assert len(tip) == 1 and len(root) == 1
                assert np.max(np.abs(pos[tip[0]] - pos[root[0]])) < 1e-4
        # mirror symmetry of the two wings about the body's x-z plane (y -> 2 y_c - y)
        yc = body[0][1]
        left = pos[seg == 5]
        right = pos[seg == 6]
        mirrored = right.copy()
        mirrored[:, 1] = 2.0 * yc - mirrored[:, 1]
        assert np.max(np.abs(left - mirrored)) < 1e-3


@pytest.mark.parametrize("rr3", [False, True])
def test_regularized_pair_order_agrees_with_literal_order(rr3):
    """The stepping evaluates the regularized / RR3 operator on opposite
    direction pairs (moments from pair sums, the equilibrium's even and odd
    parts, the stress from pair non-equilibria).  The reference's literal
    per-direction order gives the same operator to FP32 rounding: within
    1e-6 relative per population (each value against its own magnitude) for
    populations within 20 % of equilibrium, and with the same admission
    decisions for ones far enough out (95 %) to engage the positivity
    admission.  There the admitted outputs include populations cut to
    ~1e-7 w_q, whose few-ulp differences (a cancellation of terms of size
    w_q) are judged against max(|f_q|, w_q) instead."""
    _, _, w = O.lattice()
    w = w.astype(np.float64)
    rng = np.random.default_rng(5)
    engaged = 0
    for amp in (0.01, 0.2, 0.95):
        for _ in range(400):
            f = (w * (1.0 + amp * rng.uniform(-1.0, 1.0, 19))).astype(np.float32)
            lit, act_l, res_l = O.collide_regularized(f, 1.9, rr3, 0)
            par, act_p, res_p = O.collide_regularized(f, 1.9, rr3, 1)
            lit64 = lit.astype(np.float64)
            scale = np.abs(lit64) if amp <= 0.2 else np.maximum(np.abs(lit64), w)
            assert np.max(np.abs(lit64 - par) / scale) <= 1e-6
            assert act_l == act_p
            assert abs(res_l - res_p) <= 1e-5
            engaged += act_l
    assert engaged > 50



def test_portable_power_matches_double_pow():
    """bfx_powf (the beta-planform chord law's power, portable log / exp in
    double): the correctly rounded float of the double power on the wing's
    range of bases, pow(0, e) = 0 and pow(1, e) = 1."""
    L = O.lib()
    rng = np.random.default_rng(5)
    e = np.float32(1.4891506583557845 - 1.0)
    b = np.concatenate([rng.uniform(0.0, 0.25, 4000), np.geomspace(1e-30, 0.25, 1000)]).astype(np.float32)
    got = np.array([L.or_powf(float(x), float(e)) for x in b], np.float32)
    ref = (b.astype(np.float64) ** np.float64(e)).astype(np.float32)
    assert np.max(np.abs(got.view(np.int32) - ref.view(np.int32))) <= 1
    assert L.or_powf(0.0, float(e)) == 0.0 and L.or_powf(1.0, float(e)) == 1.0


def _wing_kinematics_double(phase, amplitude, duration, max_rate, pitch_duration, low, high):
    """MetalFlappingWingValidator.kinematicState (MetalFlappingWingValidation.swift:567-640),
    the reference's double-precision form of the prescribed stroke and pitch."""
    half = 0.5 * duration
    if phase < half:
        a = math.pi * (phase + half) / duration
        stroke, rate = amplitude + max_rate * duration / math.pi * (math.sin(a) - 1), max_rate * math.cos(a)
    elif phase < 0.5 - half:
        stroke, rate = amplitude - max_rate * duration / math.pi - max_rate * (phase - half), -max_rate
    elif phase < 0.5 + half:
        a = math.pi * (phase - (0.5 - half)) / duration
        stroke = -amplitude + max_rate * duration / math.pi - max_rate * duration / math.pi * math.sin(a)
        rate = -max_rate * math.cos(a)
    elif phase < 1 - half:
        stroke, rate = -amplitude + max_rate * duration / math.pi + max_rate * (phase - (0.5 + half)), max_rate
    else:
        a = math.pi * (phase - (1 - half)) / duration
        stroke, rate = amplitude - max_rate * duration / math.pi + max_rate * duration / math.pi * math.sin(a), \
            max_rate * math.cos(a)
    ph = 0.5 * pitch_duration
    if phase < ph or phase >= 1 - ph:
        w = phase + 1 if phase < ph else phase
        x, start, change = (w - (1 - ph)) / pitch_duration, high, -(high - low)
    elif 0.5 - ph <= phase < 0.5 + ph:
        x, start, change = (phase - (0.5 - ph)) / pitch_duration, low, high - low
    else:
        return stroke, rate, (low if phase < 0.5 else high), 0.0
    pitch = start + change * (x - math.sin(2 * math.pi * x) / (2 * math.pi))
    prate = change / pitch_duration * (1 - math.cos(2 * math.pi * x))
    return stroke, rate, pitch, prate


def test_prescribed_wing_kinematics_follow_the_reference_double_form():
    """The oracle's FP32 stroke / pitch kinematics (preparePrescribedFlappingWing,
    BF.metal:945-1078) agree with the reference's double-precision kinematic
    state at phases in every branch, within FP32 rounding; the span is the
    stroke rotation of x about z and the frame is orthonormal."""
    import bfx.cases as cases
    from helpers import oracle_wing
    cfg, wing = cases.flapping_wing(chord=8)
    w = oracle_wing(wing)
    L = O.lib()
    cyc = w.kinematics0.v[0]
    args = (w.kinematics0.v[1], w.kinematics0.v[2], w.kinematics1.v[2], w.kinematics0.v[3], w.kinematics1.v[0],
            w.kinematics1.v[1])
    for phase in (0.02, 0.1, 0.2, 0.3, 0.4, 0.45, 0.5, 0.55, 0.6, 0.7, 0.8, 0.9, 0.97):
        t = float(np.float32(phase * cyc))
        prep = O.WingPrepared()
        L.or_prepare_wing(ct.byref(w), t, ct.byref(prep))
        ph = float(np.fmod(np.float32(t) / np.float32(cyc), np.float32(1.0)))
        stroke, rate, pitch, prate = _wing_kinematics_double(ph, *args)
        st = list(prep.state.v)
        assert abs(st[0] - stroke) < 2e-6 and abs(st[1] - pitch) < 2e-6, phase
        assert abs(st[2] - rate / cyc) < 1e-7 and abs(st[3] - prate / cyc) < 1e-7, phase
        span = np.array(prep.span.v[:3])
        assert np.allclose(span, [math.cos(stroke), math.sin(stroke), 0.0], atol=2e-6)
        frame = np.array([prep.chord.v[:3], prep.span.v[:3], prep.normal.v[:3]], np.float64)
        assert np.allclose(frame @ frame.T, np.eye(3), atol=1e-6)
