"""Discrete adjoint (bfx_adjoint) on the flapping plate pair: gradient of the
window-mean lift and aerodynamic power with respect to the four wing-kinematic
parameters, checked against central finite differences of the forward step
(FP64 populations), the FP32 gradient against the FP64 one, checkpoint-interval
invariance, the final state, and the torch.autograd bridge."""
from __future__ import annotations

import numpy as np
import pytest

import bfx._lib as L
import bfx.cases as cases
from bfx.simulation import BirdFlowError, Lattice, bird_struct
from helpers import body_struct_from_tuple

pytestmark = pytest.mark.gpu

STEPS = 40


def build(theta=None, storage=L.STORAGE_F64, link_rule=L.LINK_LINEAR, coarse=False):
    kw = dict(n_chord=1, n_span=1) if coarse else {}
    cfg, rows, body, mesh = cases.adjoint_plates(storage=storage, link_rule=link_rule, **kw)
    if theta is not None:
        rows = cases.with_kinematic_parameters(rows, theta)
    return Lattice(cfg, bird_struct(rows), body_struct_from_tuple(body), mesh)


def theta0(link_rule=L.LINK_LINEAR):
    _, rows, _, _ = cases.adjoint_plates(link_rule=link_rule)
    return np.array(cases.kinematic_parameters(rows), dtype=np.float64)


def adjoint(theta, storage, link_rule, force_weight, power_weight, steps=STEPS, interval=0, coarse=False):
    lat = build(theta, storage, link_rule, coarse)
    try:
        return lat.adjoint(steps, force_weight, power_weight, checkpoint_interval=interval)
    finally:
        lat.close()


FD_STEPS = 12


def trajectory(theta, storage, link_rule, coarse, steps=FD_STEPS):
    """Per-step topology (links, covered, uncovered), lift F_z and power."""
    lat = build(theta, storage, link_rule, coarse)
    topo, lift, power = [], [], []
    for _ in range(steps):
        lat.advance(1)
        ld = lat.loads()
        topo.append((ld.link_count, ld.covered_count, ld.uncovered_count))
        lift.append(ld.force[2])
        power.append(ld.power)
    lat.close()
    return topo, np.array(lift), np.array(power)


def central_differences(storage, link_rule, coarse, h):
    """Central differences of the mean lift and mean power.  Both runs of a
    pair must see the same topology at every step: a cell that changes
    occupancy between them adds a jump the derivative does not have."""
    t0 = theta0(link_rule)
    lift, power = np.zeros(4), np.zeros(4)
    for k in range(4):
        tp, tm = t0.copy(), t0.copy()
        tp[k] += h
        tm[k] -= h
        topo_p, lift_p, pow_p = trajectory(tp, storage, link_rule, coarse)
        topo_m, lift_m, pow_m = trajectory(tm, storage, link_rule, coarse)
        assert topo_p == topo_m, f"parameter {k}: occupancy differs between theta +- {h}"
        lift[k] = (lift_p.mean() - lift_m.mean()) / (2 * h)
        power[k] = (pow_p.mean() - pow_m.mean()) / (2 * h)
    return lift, power


# FP64 populations, h = 1e-4 rad over 12 steps: no cell changes occupancy
# between the two runs of a pair (checked step by step), while the FP32 wing
# frames' round-off (about one ulp of the rotation angle, ~1e-7 rad, coherent
# over the whole wing) stays a ~0.1 % error of the difference.  The ray-root
# case uses one quad per wing: the root search looks at the two triangles that
# own the link's end cells, so a finer mesh makes its q jump where ownership
# changes, which no derivative describes.
@pytest.mark.parametrize("link_rule,coarse", [(L.LINK_LINEAR, False), (L.LINK_RAY_ROOT, True)])
def test_fp64_gradient_matches_central_differences(link_rule, coarse):
    fd_lift, fd_power = central_differences(L.STORAGE_F64, link_rule, coarse, 1e-4)
    for (fw, pw), fd in ((((0.0, 0.0, 1.0), 0.0), fd_lift), (((0.0, 0.0, 0.0), 1.0), fd_power)):
        g = np.array(list(adjoint(theta0(link_rule), L.STORAGE_F64, link_rule, fw, pw, steps=FD_STEPS,
                                  coarse=coarse).gradient))
        scale = np.max(np.abs(fd))
        assert scale > 0
        assert np.max(np.abs(g - fd)) <= 1e-2 * scale, f"adjoint {g} vs central differences {fd}"


def test_fp32_gradient_tracks_fp64():
    fw, pw = (0.0, 0.0, 1.0), 0.0
    g64 = np.array(list(adjoint(theta0(), L.STORAGE_F64, L.LINK_LINEAR, fw, pw).gradient))
    g32 = np.array(list(adjoint(theta0(), L.STORAGE_F32, L.LINK_LINEAR, fw, pw).gradient))
    assert np.max(np.abs(g32 - g64)) <= 1e-2 * np.max(np.abs(g64)), f"{g32} vs {g64}"


def test_checkpoint_interval_does_not_change_the_gradient():
    fw, pw = (0.0, 0.0, 1.0), 0.5
    a = adjoint(theta0(), L.STORAGE_F32, L.LINK_LINEAR, fw, pw, interval=0)
    b = adjoint(theta0(), L.STORAGE_F32, L.LINK_LINEAR, fw, pw, interval=3)
    c = adjoint(theta0(), L.STORAGE_F32, L.LINK_LINEAR, fw, pw, interval=STEPS)
    assert a.objective == b.objective == c.objective
    assert list(a.gradient) == list(b.gradient) == list(c.gradient)


def test_adjoint_leaves_the_forward_state_and_objective():
    """After bfx_adjoint the handle holds the state bfx_advance would reach, and
    J is the window mean of the per-step lift."""
    ref = build(storage=L.STORAGE_F32)
    forces = []
    for _ in range(STEPS):
        ref.advance(1)
        forces.append(ref.loads().force[2])
    lat = build(storage=L.STORAGE_F32)
    res = lat.adjoint(STEPS, (0.0, 0.0, 1.0), 0.0, window=(11, STEPS))
    assert np.array_equal(lat.populations(), ref.populations())
    assert lat.step_index()[0] == STEPS
    assert abs(res.objective - np.mean(forces[10:])) <= 1e-12 * max(1.0, abs(res.objective))
    lat.advance(3)   # the handle keeps stepping
    ref.advance(3)
    assert np.array_equal(lat.populations(), ref.populations())


def test_torch_autograd_bridge():
    torch = pytest.importorskip("torch")
    from bfx.autograd import kinematic_objective
    direct = adjoint(theta0(), L.STORAGE_F32, L.LINK_LINEAR, (0.0, 0.0, 1.0), 0.0)
    theta = torch.tensor(theta0(), dtype=torch.float64, requires_grad=True)
    J = kinematic_objective(theta, lambda t: build(t, L.STORAGE_F32), STEPS, force_weight=(0.0, 0.0, 1.0))
    (2.0 * J).backward()
    assert J.item() == direct.objective
    assert np.allclose(theta.grad.numpy(), 2.0 * np.array(list(direct.gradient)), rtol=0, atol=0)


def test_out_of_scope_configuration_is_rejected():
    cfg, rows, body, _ = cases.ellipsoid_channel(nx=48, ny=24, nz=24, radii=(7.0, 4.0, 4.0))
    lat = Lattice(cfg, bird_struct(rows), body_struct_from_tuple(body))
    with pytest.raises(BirdFlowError) as e:
        lat.adjoint(4, (1.0, 0.0, 0.0), 0.0)
    assert e.value.status == 10
    lat.advance(1)   # still usable


def frozen_objectives(theta, recording, mode, steps, storage=L.STORAGE_F64):
    """Window-mean lift and power of a run whose occupancy is recorded
    (mode 1) or replayed from the recording (mode 2) through the library's
    topology test hook."""
    lat = build(theta, storage)
    lat.replay_topology(mode, recording.data_ptr(), steps)
    lift, power = 0.0, 0.0
    for _ in range(steps):
        lat.advance(1)
        ld = lat.loads()
        lift += ld.force[2]
        power += ld.power
    lat.close()
    return lift / steps, power / steps


def test_full_period_gradient_matches_frozen_topology_differences():
    """A full stroke period (600 steps, every cell that the wings sweep
    covered and uncovered) in FP64: central differences of the window-mean
    lift and power with the occupancy of every step held at the unperturbed
    run's (recorded and replayed through the topology test hook), so that the
    differences see the smooth piece of J the adjoint differentiates, agree
    with the adjoint within 1 % of the largest component.  h = 1e-4 rad: a
    larger step moves fluid cells next to the wall across the link rule's
    clamps (q = 1e-4 once a fluid cell's signed distance turns negative), a
    smaller one reaches the FP32 resolution of the geometry.  Lift is checked
    on all four parameters, power on stroke and pitch amplitude: with the
    occupancy frozen, a link whose interpolation partner is solid still
    switches from the interpolated to the solid node's wall velocity when its
    q crosses 1/2, a jump that enters the power directly (through u_wall) and
    dominates its pitch-phase and deviation differences at every h."""
    torch = pytest.importorskip("torch")
    steps, h = 600, 1e-4
    t0 = theta0()
    cfg, _, _, _ = cases.adjoint_plates()
    n = int(cfg.nx) * int(cfg.ny) * int(cfg.nz)
    rec = torch.empty((steps, n), dtype=torch.uint8, device="cuda")
    base = frozen_objectives(t0, rec, 1, steps)
    for (fw, pw), j, checked in ((((0.0, 0.0, 1.0), 0.0), 0, [0, 1, 2, 3]), (((0.0, 0.0, 0.0), 1.0), 1, [0, 1])):
        res = adjoint(t0, L.STORAGE_F64, L.LINK_LINEAR, fw, pw, steps=steps)
        assert abs(res.objective - base[j]) <= 1e-9 * max(1.0, abs(base[j]))
        g = np.array(list(res.gradient))[checked]
        fd = np.zeros(len(checked))
        for i, k in enumerate(checked):
            tp, tm = t0.copy(), t0.copy()
            tp[k] += h
            tm[k] -= h
            fd[i] = (frozen_objectives(tp, rec, 2, steps)[j] - frozen_objectives(tm, rec, 2, steps)[j]) / (2 * h)
        print("adjoint", g, "frozen-topology differences", fd)
        assert np.max(np.abs(g - fd)) <= 1e-2 * np.max(np.abs(fd)), f"adjoint {g} vs frozen differences {fd}"
