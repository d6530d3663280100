"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Tolerances (from the reference's own gates and the task contract):
  FP32 populations   <= 1e-6 relative per value (the FP32 path is built to be
                     bit-identical; the tests also report exact equality)
  body loads         <= 1e-5 relative (FP64 sums of identical contributions)
  masks, cut links   bit-exact (set of (fluid cell, direction) pairs)
"""
from __future__ import annotations

import ctypes as ct
import math

import numpy as np
import pytest

import bfx._lib as L
import bfx.cases as cases
import oracle as O
from bfx.simulation import Lattice, bird_struct
from helpers import body_struct_from_tuple, oracle_twin, rel_diff

pytestmark = pytest.mark.gpu

POP_RTOL = 1e-6
LOAD_RTOL = 1e-5


def make_pair(cfg, rows=None, body=None, mesh=None):
    lat = Lattice(cfg, bird_struct(rows) if rows is not None else None,
                  body_struct_from_tuple(body) if body is not None else None, mesh)
    osim = oracle_twin(cfg, rows, body, mesh)
    return lat, osim


def compare_pops(lat, osim, what="", rtol=POP_RTOL):
    g = lat.populations().ravel()
    o = osim.pa
    d = np.abs(g.astype(np.float64) - o.astype(np.float64))
    rel = float(np.max(d / np.maximum(np.abs(o.astype(np.float64)), 1e-12)))
    assert np.all(np.isfinite(g)), what
    assert rel <= rtol, f"{what}: max relative population difference {rel:.3e}"
    return rel, bool(np.array_equal(g, o))


def compare_loads(lat, osim, what="", lever_arm=None):
    """Loads within LOAD_RTOL of the oracle.  With ``lever_arm`` (metres) the
    torque is judged against |F| x lever_arm: on a symmetric body the torque is
    a cancellation residue far below that scale, and a run that is not
    bit-identical (FMA contraction) moves the residue by round-off x radius."""
    ld = lat.loads()
    gf = np.array(ld.force)
    gt = np.array(ld.torque)
    of = np.array(osim.loads.f64_force)
    ot = np.array(osim.loads.f64_torque)
    fscale = max(np.max(np.abs(of)), 1e-30)
    tscale = max(np.max(np.abs(ot)), 1e-30)
    if lever_arm is not None:
        tscale = max(tscale, fscale * lever_arm)
    assert np.max(np.abs(gf - of)) <= LOAD_RTOL * fscale + 1e-300, f"{what}: force {gf} vs {of}"
    assert np.max(np.abs(gt - ot)) <= LOAD_RTOL * tscale + 1e-300, f"{what}: torque {gt} vs {ot}"
    return gf, of


def oracle_links(osim):
    n = osim.n
    cap = 18 * n
    cell = np.zeros(cap, np.uint32)
    d = np.zeros(cap, np.uint8)
    cnt = O.lib().or_enumerate_links(ct.byref(osim.p), O.u8ptr(osim.mnext), O.u8ptr(osim.mcur),
                                     cell.ctypes.data_as(ct.POINTER(ct.c_uint32)), O.u8ptr(d), cap)
    return cell[:cnt], d[:cnt]


def link_set(cell, d):
    key = cell.astype(np.uint64) * 32 + d.astype(np.uint64)
    return np.sort(key)


# --------------------------------------------------------------------------
# Periodic shear wave (config 1 family): full-lattice pull + TRT
# --------------------------------------------------------------------------
def test_shear_wave_per_step_matches_oracle():
    cfg, _, _, _ = cases.shear_wave(n=24, viscosity=0.03, magic=3.0 / 16.0, axis="y")
    lat, osim = make_pair(cfg)
    compare_pops(lat, osim, "initial")
    exact = True
    for step in range(8):
        lat.advance(1)
        osim.step()
        rel, eq = compare_pops(lat, osim, f"step {step + 1}")
        exact &= eq
    # odd and even AA parities both covered; the FP32 build reproduces the oracle bit for bit
    assert exact


def test_shear_wave_64_analytic_decay_and_oracle():
    """64^3, nu = 0.01, magic 1/4, u_x = 0.01 sin(2 pi z / 64), 2000 steps."""
    cfg, _, _, _ = cases.shear_wave(n=64, viscosity=0.01, magic=0.25, amplitude=0.01, axis="z")
    lat, osim = make_pair(cfg)
    lat.advance(2000, batch_size=256, capture_fields=True)
    rho, vel = lat.fields()
    z = np.arange(64)
    prof = vel[:, 0].reshape(64, 64, 64).mean(axis=(1, 2))
    amp = 2.0 * np.dot(prof, np.sin(2 * np.pi * z / 64)) / 64
    analytic = 0.01 * math.exp(-0.01 * (2 * math.pi / 64) ** 2 * 2000)
    assert abs(amp - analytic) / analytic < 0.03
    osim.advance(2000)
    compare_pops(lat, osim, "2000 steps")
    # FP64 reduction of the same FP32 field; the FP32 step itself drifts by
    # ~3e-8 of the mass per step (the reference gates 5e-6 over 120 steps)
    mm = lat.mass_momentum()
    om = osim.fluid_mass_momentum()
    assert abs(mm[0] - om[0]) <= 1e-12 * om[0]
    assert np.max(np.abs(mm[1:] - om[1:])) <= 1e-12 * om[0]
    assert abs(mm[0] - 64 ** 3) / 64 ** 3 < 2000 * 5e-6 / 120


@pytest.mark.parametrize("collision", [L.COLLISION_TRT_LIMITER, L.COLLISION_REGULARIZED, L.COLLISION_RR3])
def test_collision_operators_match_oracle(collision):
    cfg, _, _, _ = cases.shear_wave(n=20, viscosity=0.02, magic=3.0 / 16.0, amplitude=0.05, axis="y",
                                    collision=collision)
    lat, osim = make_pair(cfg)
    for step in range(6):
        lat.advance(1)
        osim.step()
        compare_pops(lat, osim, f"collision {collision} step {step + 1}")


@pytest.mark.parametrize("form", ["f32", "fast_math", "f16"])
@pytest.mark.parametrize("collision", [L.COLLISION_REGULARIZED, L.COLLISION_RR3])
def test_regularized_admission_matches_oracle(collision, form):
    """Populations far from equilibrium (w_q (1 + 0.95 U(-1, 1))) at a low
    viscosity drive the positivity admission of the regularized operators in
    many cells.  The FP32 step matches the oracle bit for bit, populations and
    limiter statistics; fast_math (the contracted kernel's restated collision)
    stays within 1e-5 w_q and the FP16-deviation format (the staged kernel)
    within 2e-3 w_q, the format's quantisation of deviations up to 0.95 w_q."""
    storage = L.STORAGE_F16_DEVIATION if form == "f16" else L.STORAGE_F32
    n = 24
    cfg, _, _, _ = cases.shear_wave(n=n, viscosity=0.002, magic=3.0 / 16.0, amplitude=0.0, axis="y",
                                    storage=storage, collision=collision)
    if form == "fast_math":
        cfg.fast_math = 1
    lat, osim = make_pair(cfg)
    _, _, w = O.lattice()
    w = w.astype(np.float64)[:, None]
    rng = np.random.default_rng(11)
    pops = (w * (1.0 + 0.95 * rng.uniform(-1.0, 1.0, (19, n ** 3)))).astype(np.float32)
    lat.set_populations(pops)
    start = lat.populations().ravel()
    osim.pa[:] = start
    lat.advance(1)
    osim.step()
    g = lat.populations().reshape(19, -1).astype(np.float64)
    o = osim.pa.reshape(19, -1).astype(np.float64)
    act_g, act_o = lat.loads().limiter_activations, osim.loads.activation
    assert act_o > 0.02 * n ** 3, f"admission engaged in {act_o} cells only"
    err = float(np.max(np.abs(g - o) / w))
    if form == "f32":
        assert np.array_equal(g, o), f"max |diff| / w = {err:.3e}"
        assert act_g == act_o
        assert lat.loads().max_restriction == pytest.approx(osim.loads.max_restriction, rel=0, abs=0)
    elif form == "fast_math":
        assert err <= 1e-5, f"max |diff| / w = {err:.3e}"
        assert abs(act_g - act_o) <= 0.01 * act_o
    else:
        assert err <= 2e-3, f"max |diff| / w = {err:.3e}"
        assert abs(act_g - act_o) <= 0.05 * act_o
    lat.close()


# --------------------------------------------------------------------------
# Ellipsoid in a channel (config 2 family): RR3, interpolated links,
# velocity inlet, zero-gradient outflow, periodic y/z, static geometry
# --------------------------------------------------------------------------
@pytest.mark.parametrize("collision", [L.COLLISION_RR3, L.COLLISION_TRT])
def test_ellipsoid_channel_matches_oracle(collision):
    cfg, rows, body, _ = cases.ellipsoid_channel(nx=64, ny=32, nz=32, radii=(9.0, 5.0, 4.5), inflow=0.05,
                                                 viscosity=0.02, collision=collision)
    lat, osim = make_pair(cfg, rows, body)
    assert np.array_equal(lat.mask(), osim.mcur)
    for step in range(12):
        lat.advance(1)
        osim.step()
        compare_pops(lat, osim, f"ellipsoid step {step + 1}")
        compare_loads(lat, osim, f"ellipsoid step {step + 1}")
    cell, d, q = lat.links()
    oc, od = oracle_links(osim)
    assert len(cell) > 100
    assert np.array_equal(link_set(cell, d), link_set(oc, od))
    assert abs(lat.loads().force[0]) > 0.0
    # link fractions against the oracle's bisection
    nx, ny = cfg.nx, cfg.ny
    for i in range(0, len(cell), max(1, len(cell) // 200)):
        g = int(cell[i])
        x, y, z = g % nx, (g // nx) % ny, g // (nx * ny)
        qq = int(d[i])
        c, _, _ = O.lattice()
        sx, sy, sz = x - c[qq][0], y - c[qq][1], z - c[qq][2]
        oq = O.lib().or_ellipsoid_link_fraction(ct.byref(osim.p), ct.byref(osim.bird), ct.byref(osim.prep),
                                                x, y, z, sx, sy, sz)
        assert q[i] == np.float32(oq)


# --------------------------------------------------------------------------
# Analytic bird (reference production path): moving halfway links
# --------------------------------------------------------------------------
def _compact_bird_lattice(free_flight=False):
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=free_flight)
    sim = BirdFlowSimulation(config, bird, state)
    cfg = sim.lattice.config
    rows = bird.packed()
    body = (state.position_meters, state.orientation_body_to_world, state.linear_velocity_meters_per_second,
            state.angular_velocity_body_radians_per_second)
    osim = oracle_twin(cfg, rows, body)
    return sim, osim


def test_compact_bird_moving_boundary_matches_oracle():
    sim, osim = _compact_bird_lattice(False)
    lat = sim.lattice
    assert np.array_equal(lat.mask(), osim.mcur)
    for step in range(10):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        compare_pops(lat, osim, f"bird step {step + 1}")
        compare_loads(lat, osim, f"bird step {step + 1}")
        cell, d, _ = lat.links()
        oc, od = oracle_links(osim)
        assert np.array_equal(link_set(cell, d), link_set(oc, od)), f"links step {step + 1}"


def test_compact_bird_free_flight_matches_oracle():
    sim, osim = _compact_bird_lattice(True)
    lat = sim.lattice
    for step in range(10):
        lat.advance(1)
        osim.step()
        compare_pops(lat, osim, f"free flight step {step + 1}")
        compare_loads(lat, osim, f"free flight step {step + 1}")
        b = lat.body()
        assert rel_diff(list(b.position), list(osim.body64.position)) < 1e-12
        assert np.allclose(list(b.velocity), list(osim.body64.velocity), rtol=1e-9, atol=1e-12)
        assert np.allclose(list(b.orientation), list(osim.body64.orientation), rtol=1e-9, atol=1e-12)


# --------------------------------------------------------------------------
# Articulated triangle mesh (config 3 family): rasterise, resolve, cut links
# --------------------------------------------------------------------------
@pytest.mark.parametrize("link_rule", [L.LINK_LINEAR, L.LINK_RAY_ROOT])
def test_flapping_plate_mesh_matches_oracle(link_rule):
    cfg, rows, body, mesh = cases.flapping_plates(nx=96, ny=64, nz=64, span=16.0, chord=6.0, thickness=2.0,
                                                  n_chord=6, n_span=16, period=1000.0, viscosity=0.02,
                                                  link_rule=link_rule, sponge_width=6.0)
    lat, osim = make_pair(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    for step in range(8):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        compare_pops(lat, osim, f"mesh step {step + 1}")
        compare_loads(lat, osim, f"mesh step {step + 1}")
        cell, d, q = lat.links()
        oc, od = oracle_links(osim)
        assert np.array_equal(link_set(cell, d), link_set(oc, od)), f"links step {step + 1}"
        ld = lat.loads()
        assert ld.covered_count == osim.loads.covered_count and ld.uncovered_count == osim.loads.uncovered_count
    assert osim.loads.covered_count + osim.loads.uncovered_count > 0
    if link_rule == L.LINK_RAY_ROOT:
        # sampled ray-root fractions of the last step equal the oracle's search bit for bit
        tris = mesh["tris"].astype(np.uint32).ravel()
        c, _, _ = O.lattice()
        nx, ny = cfg.nx, cfg.ny
        sampled = range(0, len(cell), max(1, len(cell) // 300))
        for i in sampled:
            g = int(cell[i])
            x, y, z = g % nx, (g // nx) % ny, g // (nx * ny)
            qq = int(d[i])
            sx, sy, sz = x - c[qq][0], y - c[qq][1], z - c[qq][2]
            oq = O.lib().or_mesh_ray_root(ct.byref(osim.p), O.fptr(osim.mesh_pos),
                                          tris.ctypes.data_as(ct.POINTER(ct.c_uint32)), mesh["tris"].shape[0],
                                          cfg.mesh_half_thickness, osim.keys.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                          x, y, z, sx, sy, sz)
            assert q[i] == np.float32(oq), (i, float(q[i]), oq)
        assert len(sampled) > 50


@pytest.mark.parametrize("link_rule", [L.LINK_LINEAR, L.LINK_RAY_ROOT])
def test_jointed_wing_mesh_matches_oracle(link_rule):
    """3-segment wings hinged at elbow and wrist (mesh segments 1-6): masks,
    cut links and covered / uncovered counts bit-exact, populations and loads
    within tolerance, every step."""
    cfg, rows, body, mesh = cases.jointed_plates(link_rule=link_rule)
    assert set(mesh["segment"].tolist()) == {1, 2, 3, 4, 5, 6}
    lat, osim = make_pair(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    for step in range(8):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        compare_pops(lat, osim, f"jointed step {step + 1}")
        compare_loads(lat, osim, f"jointed step {step + 1}")
        cell, d, q = lat.links()
        oc, od = oracle_links(osim)
        assert np.array_equal(link_set(cell, d), link_set(oc, od)), f"links step {step + 1}"
    assert osim.loads.covered_count + osim.loads.uncovered_count > 0


def test_keyframed_mesh_replay_matches_oracle():
    """Keyframe replay (prepareIndexedBirdSurface, BF.metal:1585-1622) of a
    body-fixed mesh with keyframes every 4 steps: 13 steps cross three exact
    interior keyframe times; masks and cut-link sets stay bit-exact and
    populations and loads within the FP32 tolerances."""
    cfg, rows, body, mesh = cases.keyframed_plates()
    lat, osim = make_pair(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    for step in range(13):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        compare_pops(lat, osim, f"keyframed step {step + 1}")
        compare_loads(lat, osim, f"keyframed step {step + 1}")
        cell, d, _ = lat.links()
        oc, od = oracle_links(osim)
        assert np.array_equal(link_set(cell, d), link_set(oc, od)), f"links step {step + 1}"
    assert osim.loads.covered_count + osim.loads.uncovered_count > 0
    assert abs(lat.loads().force[2]) > 0.0


def test_articulated_bird_free_flight_matches_oracle():
    """Config-5 family at reduced size: ellipsoid body, tail plate and two
    jointed wings as one mesh, free 6-DOF body, RR3, velocity inlet."""
    cfg, rows, body, mesh = cases.articulated_bird(nx=160, ny=128, nz=96, storage=L.STORAGE_F32,
                                                   body_radii=(16.0, 5.0, 5.0), wing_spans=(12.0, 11.0, 10.0),
                                                   chords=(10.0, 8.0, 6.0, 4.0), resolution=0.25,
                                                   sponge_width=8.0, viscosity=0.01)
    assert set(mesh["segment"].tolist()) == {0, 1, 2, 3, 4, 5, 6}
    lat, osim = make_pair(cfg, rows, body, mesh)
    for step in range(3):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        compare_pops(lat, osim, f"bird step {step + 1}")
        compare_loads(lat, osim, f"bird step {step + 1}")
    lat.advance(20)
    assert np.all(np.isfinite(lat.populations()))
    assert lat.safety().event[2] == 0


def test_fast_math_fp32_stays_within_tolerance_of_oracle():
    """fast_math (the reference's SimulationConfiguration.fastMath) contracts
    a*b+c into FMA, uses one reciprocal for the velocity and evaluates RR3 in
    the pair-restated order of the contracted kernels: no longer bit-identical
    to the oracle's FP32 order, but within 3e-6 relative after 12 steps, and
    no farther from an FP64 run of the same steps than the bit-identical FP32
    path is (the difference is a different rounding sequence, not a loss of
    accuracy)."""
    def channel(storage=L.STORAGE_F32):
        return cases.ellipsoid_channel(nx=64, ny=32, nz=32, radii=(9.0, 5.0, 4.5), inflow=0.05, viscosity=0.02,
                                       collision=L.COLLISION_RR3, storage=storage)
    cfg, rows, body, _ = channel()
    cfg.fast_math = 1
    lat, osim = make_pair(cfg, rows, body)
    for step in range(12):
        lat.advance(1)
        osim.step()
    compare_pops(lat, osim, "fast_math after 12 steps", rtol=3e-6)
    compare_loads(lat, osim, "fast_math after 12 steps", lever_arm=9.0 * cfg.cell_size)
    fast = lat.populations().astype(np.float64)
    lat.close()
    runs = {}
    for st in (L.STORAGE_F32, L.STORAGE_F64):
        c, r, b, _ = channel(st)
        ref = Lattice(c, bird_struct(r), body_struct_from_tuple(b))
        ref.advance(12)
        runs[st] = ref.populations().astype(np.float64)
        ref.close()
    f64 = runs[L.STORAGE_F64]
    err_exact = float(np.max(np.abs(runs[L.STORAGE_F32] - f64) / np.abs(f64)))
    err_fast = float(np.max(np.abs(fast - f64) / np.abs(f64)))
    assert err_fast <= 1.5 * err_exact + 1e-7, f"fast {err_fast:.3e} vs exact {err_exact:.3e} against FP64"


# --------------------------------------------------------------------------
# Prescribed flapping wing (MetalFlappingWingValidation's analytic wing):
# beta-planform classification and 10-step bisection link fractions
# --------------------------------------------------------------------------
def _oracle_wing_fractions(osim, cell, d):
    out = np.zeros(len(cell), np.float32)
    cell = np.ascontiguousarray(cell, np.uint32)
    d = np.ascontiguousarray(d, np.uint8)
    O.lib().or_wing_link_fractions(ct.byref(osim.p), ct.byref(osim.wing), ct.byref(osim.wing_prep),
                                   cell.ctypes.data_as(ct.POINTER(ct.c_uint32)), O.u8ptr(d), len(cell), O.fptr(out))
    return out


def test_prescribed_flapping_wing_matches_oracle_over_a_cycle():
    """The Li-Nabawy wing (preparePrescribedFlappingWing +
    buildPrescribedFlappingWing, BF.metal:940-1297) over one full cycle of
    480 steps, so every branch of the stroke and pitch kinematics runs: masks,
    cut-link sets and every link fraction bit-exact against the oracle each
    step, loads within 1e-5, populations within 1e-6 every 40 steps."""
    from helpers import oracle_wing  # noqa: F401
    cfg, wing = cases.flapping_wing(chord=6, cycle_steps=480, viscosity=0.02)
    lat = Lattice(cfg, wing=wing)
    osim = oracle_twin(cfg, wing=wing)
    assert np.array_equal(lat.mask(), osim.mcur)
    covered = 0
    for step in range(480):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        cell, d, q = lat.links()
        oc, od = oracle_links(osim)
        assert np.array_equal(link_set(cell, d), link_set(oc, od)), f"links step {step + 1}"
        assert np.array_equal(q, _oracle_wing_fractions(osim, cell, d)), f"link fractions step {step + 1}"
        compare_loads(lat, osim, f"wing step {step + 1}")
        covered += osim.loads.covered_count + osim.loads.uncovered_count
        if (step + 1) % 40 == 0:
            compare_pops(lat, osim, f"wing step {step + 1}")
    assert covered > 0
    assert len(cell) > 100
    lat.close()
