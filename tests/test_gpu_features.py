"""GPU feature tests modelled on the reference's own test strategy
(Tests/BirdFlowMetalTests): batch-partition invariance (MetalExecutionTests.swift:473-592),
checkpoint round trip and continuation (ObservationAndCheckpointTests.swift:116-161),
runtime-safety failure (MetalExecutionTests.swift:690-736), field capture,
determinism, meshes beyond the reference's 4,096-triangle cap, and the
16-bit storage formats.
"""
from __future__ import annotations

import ctypes as ct
import math

import numpy as np
import pytest

import bfx._lib as L
import bfx.cases as cases
import oracle as O
from bfx.simulation import BirdFlowError, Lattice, bird_struct
from helpers import body_struct_from_tuple, oracle_twin

pytestmark = pytest.mark.gpu


def lattice(cfg, rows=None, body=None, mesh=None):
    return Lattice(cfg, bird_struct(rows) if rows is not None else None,
                   body_struct_from_tuple(body) if body is not None else None, mesh)


def small_mesh_case(**kw):
    # period 1000: tip speed ~0.1 cells/step (Mach ~0.17 at the tip), still
    # covering and uncovering cells every step
    args = dict(nx=96, ny=64, nz=64, span=16.0, chord=6.0, thickness=2.0, n_chord=6, n_span=16, period=1000.0,
                viscosity=0.02, sponge_width=6.0)
    args.update(kw)
    return cases.flapping_plates(**args)


@pytest.mark.parametrize("storage", [L.STORAGE_F32, L.STORAGE_F16_DEVIATION])
def test_batch_partition_invariance_is_bit_exact(storage):
    """16 steps as 16x1, 4x4 and 1x16 give identical populations and loads.
    With 16-bit storage, batches of more than one step build each next step's
    geometry on a side stream beside the fluid kernel (and replay pipelined
    graphs); one-step batches run every stage in order."""
    cfg, rows, body, mesh = small_mesh_case(storage=storage)
    results = []
    for batches in ((1,) * 16, (4,) * 4, (16,)):
        lat = lattice(cfg, rows, body, mesh)
        for b in batches:
            lat.advance(b, batch_size=b)
        results.append((lat.populations(), np.array(lat.loads().force)))
        lat.close()
    assert np.all(np.isfinite(results[0][0]))
    for pops, force in results[1:]:
        assert np.array_equal(pops, results[0][0])
        assert np.array_equal(force, results[0][1])


def test_pipelined_free_flight_bird_is_bit_exact():
    """The compact free-flying bird in FP16 deviation storage with RR3 (the
    staged kernel): 12 steps in one batch (geometry of each next step built
    beside the fluid kernel) equal 12 one-step batches bit for bit, body and
    loads included."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=True)
    out = []
    for batch in (12, 1):
        sim = BirdFlowSimulation(config, bird, state, storage=L.STORAGE_F16_DEVIATION, collision=L.COLLISION_RR3)
        sim.advance(12, batch_size=batch, field_capture="disabled")
        lat = sim.lattice
        out.append((lat.populations(), bytes(lat.body()), np.array(lat.loads().force), lat.mask()))
        sim.close()
    assert np.all(np.isfinite(out[0][0]))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][3], out[1][3])


def test_pipelined_batch_with_field_capture_is_bit_exact():
    """A 16-bit batch with required field capture: the pipelined steps hand the
    last one (which captures and builds no next geometry) the same state as
    one-step batches do; fields, populations and loads agree bit for bit."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird()
    out = []
    for batch in (6, 1):
        sim = BirdFlowSimulation(config, bird, state, storage=L.STORAGE_F16_DEVIATION, collision=L.COLLISION_RR3)
        res = sim.advance(6, batch_size=batch, field_capture="required")
        assert res.field_frame_published
        rho, vel = sim.lattice.fields()
        out.append((rho, vel, sim.lattice.populations(), np.array(sim.lattice.loads().force)))
        sim.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    assert np.all(np.isfinite(out[0][0])) and float(np.max(np.abs(out[0][1]))) > 0.0


def test_two_runs_are_bit_identical():
    cfg, rows, body, _ = cases.ellipsoid_channel(nx=64, ny=32, nz=32, radii=(9.0, 5.0, 4.5), viscosity=0.02)
    out = []
    for _ in range(2):
        lat = lattice(cfg, rows, body)
        lat.advance(25, batch_size=7)
        out.append((lat.populations(), np.array(lat.loads().force), np.array(lat.loads().torque)))
        lat.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_checkpoint_round_trip_and_continuation():
    cfg, rows, body, mesh = small_mesh_case()
    lat = lattice(cfg, rows, body, mesh)
    lat.advance(5)
    state = lat.save_state()
    pops_saved = lat.populations()
    lat.advance(7)
    cont = lat.populations()
    assert np.all(np.isfinite(cont))
    force = np.array(lat.loads().force)
    lat.restore_state(state)
    assert np.array_equal(lat.populations(), pops_saved)
    assert lat.step_index()[0] == 5
    lat.advance(7)
    assert np.array_equal(lat.populations(), cont)
    assert np.array_equal(np.array(lat.loads().force), force)
    # restoring into a fresh handle continues identically
    fresh = lattice(cfg, rows, body, mesh)
    fresh.restore_state(state)
    fresh.advance(7)
    assert np.array_equal(fresh.populations(), cont)


def test_checkpoint_archive_round_trip_and_continuation(tmp_path):
    """CheckpointArchive write / read (CheckpointArchive.swift:45-160; raw
    files where the reference uses LZFSE): the archive's populations and mask
    files equal the saved simulation's byte for byte, a fresh handle restored
    from it continues bit-identically (moving mesh: both mask buffers), and a
    flipped byte in any data file is refused by its SHA-256 digest."""
    import json
    import os
    import bfx.checkpoint as C
    cfg, rows, body, mesh = small_mesh_case()
    lat = lattice(cfg, rows, body, mesh)
    lat.advance(5)
    path = str(tmp_path / "ckpt")
    lat.save_archive(path)
    manifest = json.load(open(os.path.join(path, C.MANIFEST)))
    assert manifest["schema"] == 1 and manifest["step"] == 5
    assert open(os.path.join(path, C.POPULATIONS), "rb").read() == lat.populations().tobytes()
    assert open(os.path.join(path, C.SOLID_MASK), "rb").read() == lat.mask().tobytes()
    lat.advance(7)
    cont = lat.populations()
    fresh = lattice(cfg, rows, body, mesh)
    got = fresh.restore_archive(path)
    assert got["populationSHA256"] == manifest["populationSHA256"]
    assert fresh.step_index()[0] == 5
    fresh.advance(7)
    assert np.array_equal(fresh.populations(), cont)
    # init(checkpointURL:): a handle built from the archive alone (plus the mesh)
    rebuilt = Lattice.from_archive(path, mesh=mesh)
    assert rebuilt.step_index()[0] == 5
    rebuilt.advance(7)
    assert np.array_equal(rebuilt.populations(), cont)
    rebuilt.close()
    for name in (C.POPULATIONS, C.SOLID_MASK, C.RESTART_STATE):
        bad = str(tmp_path / f"bad-{name}")
        lat.save_archive(bad)
        f = os.path.join(bad, name)
        data = bytearray(open(f, "rb").read())
        data[len(data) // 3] ^= 0x01
        open(f, "wb").write(bytes(data))
        with pytest.raises(C.CheckpointError, match="checksum"):
            fresh.restore_archive(bad)
    fresh.advance(1)  # the handle stays usable


def test_corrupted_checkpoint_fails_cleanly():
    cfg, _, _, _ = cases.shear_wave(n=16, viscosity=0.03, magic=3.0 / 16.0, axis="y")
    lat = lattice(cfg)
    lat.advance(2)
    state = bytearray(lat.save_state())
    state[len(state) // 2] ^= 0xFF
    with pytest.raises(BirdFlowError) as e:
        lat.restore_state(bytes(state))
    assert e.value.status == 8
    lat.advance(1)  # the handle stays usable


def test_field_capture_matches_oracle():
    cfg, rows, body, _ = cases.ellipsoid_channel(nx=48, ny=24, nz=24, radii=(7.0, 4.0, 4.0), viscosity=0.02)
    lat = lattice(cfg, rows, body)
    osim = oracle_twin(cfg, rows, body)
    lat.advance(5, capture_fields=True)
    osim.advance(4)
    osim.step(capture_fields=True)
    rho, vel = lat.fields()
    assert np.array_equal(rho, osim.density)
    assert np.array_equal(vel, osim.velocity.reshape(-1, 4)[:, :3])


def test_mesh_beyond_4096_triangles_matches_oracle():
    """16,384 triangles: the reference's 12-bit key would cap this at 4,096."""
    cfg, rows, body, mesh = small_mesh_case(nx=80, ny=64, nz=64, span=20.0, chord=8.0, n_chord=32, n_span=128,
                                            link_rule=L.LINK_RAY_ROOT)
    assert mesh["tris"].shape[0] == 16384
    lat = lattice(cfg, rows, body, mesh)
    osim = oracle_twin(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    for step in range(3):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur)
        g = lat.populations().ravel()
        rel = np.max(np.abs(g.astype(np.float64) - osim.pa) / np.maximum(np.abs(osim.pa), 1e-12))
        assert rel <= 1e-6


def test_runtime_safety_violation_invalidates_the_handle():
    """A free-flying body launched far above Mach 0.15 trips the safety ledger
    on the first step (host-side check after the batch, as the reference's
    advance does); the handle is then terminally invalid."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=True)
    state.linear_velocity_meters_per_second = (60.0, 0.0, 0.0)
    sim = BirdFlowSimulation(config, bird, state)
    with pytest.raises(BirdFlowError) as e:
        sim.advance(3, batch_size=1)
    assert e.value.status == 5
    with pytest.raises(BirdFlowError) as e2:
        sim.advance(1)
    assert e2.value.status == 6


def test_invalid_advance_request():
    cfg, _, _, _ = cases.shear_wave(n=16, axis="y")
    lat = lattice(cfg)
    rc = lat.lib.bfx_advance(lat.handle, 1, 0, 0, None, 0, None)
    assert rc == 3


def test_bird_simulation_run_samples_and_snapshot():
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=True)
    sim = BirdFlowSimulation(config, bird, state)
    res = sim.advance(6, batch_size=4, record_run_samples=True)
    assert len(res.run_samples) == 6
    assert [s.step for s in res.run_samples] == [1, 2, 3, 4, 5, 6]
    snap = sim.snapshot()
    assert snap.step == 6
    assert res.runtime_safety["passed"]
    last = res.run_samples[-1]
    assert np.allclose(list(last.position), list(snap.body.position))
    rho, vel = sim.copy_macroscopic_fields()
    assert np.all(np.isfinite(rho)) and np.all(rho > 0.5)
    p = sim.copy_gauge_pressure_field_pascals()
    assert p.shape == rho.shape


# Shear-wave amplitude after 400 steps in each storage format against FP32
# (32^3, amplitude 0.02, nu 0.02).  The amplitude decays by ~8e-4 of itself per
# step; FP16 deviation storage resolves that with its 2^12 scale, and BF16
# (8 significant bits of f - w_q) does through the stochastic rounding of its
# fluid stores (round-to-nearest froze this flow, leaving the amplitude ~35 %
# high).  Measured on B200: FP16 1.3e-3, BF16 1.1e-4, FP64 1.1e-5.
@pytest.mark.parametrize("storage,tol", [(L.STORAGE_F16_DEVIATION, 3e-3), (L.STORAGE_BF16_DEVIATION, 2e-3),
                                         (L.STORAGE_F64, 1e-4)])
def test_storage_formats_track_f32(storage, tol):
    """Shear-wave amplitude after 400 steps in each storage format vs FP32."""
    amps = {}
    for st in (L.STORAGE_F32, storage):
        cfg, _, _, _ = cases.shear_wave(n=32, viscosity=0.02, magic=0.25, amplitude=0.02, axis="z", storage=st)
        lat = lattice(cfg)
        lat.advance(400, capture_fields=True)
        _, vel = lat.fields()
        prof = vel[:, 0].reshape(32, 32, 32).mean(axis=(1, 2))
        amps[st] = 2.0 * np.dot(prof, np.sin(2 * np.pi * np.arange(32) / 32)) / 32
        lat.close()
    assert abs(amps[storage] - amps[L.STORAGE_F32]) / abs(amps[L.STORAGE_F32]) < tol


# One 16-bit step against the FP64 storage run of the same kernels from the
# same populations, on the moving two-plate mesh (ray-root links, covered and
# uncovered cells every step).  The 16-bit step rounds each stored deviation
# once (FP16: 11 significant bits, round to nearest, relative error <= 2^-11;
# BF16: 8 bits, stochastic rounding, <= 2^-7 = 2 x 2^-8) and reads link and
# halo values that were rounded the same way; the collision carries an input
# error to its outputs with a gain below 2.  Per value:
#   |f16_i - f64_i| <= 4 q D_cell + 4e-7 w_i,   q = 2^-11 (FP16), 2^-8 (BF16),
# D_cell = max over the cell's directions of |f64_j - w_j|; 4e-7 w_i covers the
# FP32 read-out of both runs and of the shared start values (half an FP32 unit
# of w each) and the FP32 collision arithmetic.  Measured on B200 the largest
# ratio to the bound is about 0.5 in either format.
@pytest.mark.parametrize("collision", [L.COLLISION_TRT, L.COLLISION_RR3])
@pytest.mark.parametrize("storage", [L.STORAGE_F16_DEVIATION, L.STORAGE_BF16_DEVIATION])
def test_16bit_step_stays_within_its_quantum_of_fp64(storage, collision):
    _, _, w = O.lattice()
    w = w.astype(np.float64)[:, None]
    q = 2.0 ** -11 if storage == L.STORAGE_F16_DEVIATION else 2.0 ** -8
    kw = dict(nx=96, ny=64, nz=64, span=16.0, chord=6.0, thickness=2.0, n_chord=6, n_span=16, period=1000.0,
              viscosity=0.02, link_rule=L.LINK_RAY_ROOT, sponge_width=6.0, collision=collision)
    c16, rows, body, mesh = cases.flapping_plates(storage=storage, **kw)
    c64, _, _, _ = cases.flapping_plates(storage=L.STORAGE_F64, **kw)
    l16 = lattice(c16, rows, body, mesh)
    l64 = lattice(c64, rows, body, mesh)
    l16.advance(30)
    l64.advance(30)
    worst, events = 0.0, 0
    for _ in range(10):
        l64.set_populations(l16.populations())
        l16.advance(1)
        l64.advance(1)
        assert np.array_equal(l16.mask(), l64.mask())
        a = l16.populations().reshape(19, -1).astype(np.float64)
        b = l64.populations().reshape(19, -1).astype(np.float64)
        d_cell = np.abs(b - w).max(axis=0)[None, :]
        ratio = np.abs(a - b) / (4.0 * q * d_cell + 4e-7 * w)
        worst = max(worst, float(ratio.max()))
        ld = l16.loads()
        events += ld.covered_count + ld.uncovered_count
    print(f"storage {storage} collision {collision}: max ratio to the bound {worst:.3f}")
    assert worst <= 1.0
    assert events > 0
    l16.close()
    l64.close()


def test_coupled_momentum_ledger_closes_on_the_compact_bird():
    """advanceWithCoupledMomentumLedger (BirdFlowSimulation.swift:806-1085) on
    the compact free-flight bird: every step's balance is finite, the open
    far-field faces, sponge cells and persistent boundary links all
    contribute, and the boundary and total-system closures stay within the
    reference's 0.5 % relative-RMS gate."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=True)
    sim = BirdFlowSimulation(config, bird, state)
    report = sim.advance_with_coupled_momentum_ledger(24)
    assert report["steps"] == 24 and report["finite"]
    last = report["samples"][-1]
    assert last["far_field_links"] > 0 and last["sponge_cells"] > 0 and last["boundary_links"] > 0
    assert report["rms_aerodynamic_impulse"] > 0.0
    print({k: report[k] for k in ("relative_rms_boundary_closure_residual",
                                  "relative_rms_external_system_closure_residual", "rms_aerodynamic_impulse")})
    assert report["passed"], report["scientific_verdict"]
    assert sim.step_index == 24
    sim.close()


def test_coupled_momentum_ledger_requires_free_flight():
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=False)
    sim = BirdFlowSimulation(config, bird, state)
    with pytest.raises(BirdFlowError) as e:
        sim.lattice.advance_ledger(2)
    assert e.value.status == 10
    sim.close()


def test_observation_modes_do_not_change_numerical_state():
    """ObservationAndCheckpointTests.swift:9-60: six free-flight steps with
    capture disabled (one slot, then captureCurrentMacroscopicField) and with
    best-effort capture (three slots) end in the same snapshot, and the
    extracted fields equal the fields the fused kernel captured to 1e-6
    (density, and velocity in lattice units)."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=True)
    disabled = BirdFlowSimulation(config, bird, state, observation_buffer_count=1)
    observed = BirdFlowSimulation(config, bird, state, observation_buffer_count=3)
    r0 = disabled.advance(6, batch_size=3, field_capture="disabled")
    r1 = observed.advance(6, batch_size=3, field_capture="bestEffort")
    assert not r0.field_frame_published and r1.field_frame_published
    assert disabled.capture_current_macroscopic_field()
    a, b = disabled.snapshot(), observed.snapshot()
    assert a.step == b.step == 6 and a.time == b.time
    assert bytes(a.body) == bytes(b.body) and bytes(a.loads) == bytes(b.loads)
    ra, va = disabled.lattice.fields()
    rb, vb = observed.lattice.fields()
    assert np.max(np.abs(ra - rb)) < 1e-6
    assert np.max(np.linalg.norm(va - vb, axis=1)) < 1e-6
    # copyMacroscopicFields reports m/s
    _, vphys = observed.copy_macroscopic_fields()
    assert np.array_equal(vphys, (vb * np.float32(config.scaling.velocity_to_physical)).astype(np.float32))
    disabled.close()
    observed.close()


def test_exhausted_viewer_slots_drop_without_waiting():
    """ObservationAndCheckpointTests.swift:62-87."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird()
    sim = BirdFlowSimulation(config, bird, state, observation_buffer_count=3)
    first = sim.acquire_latest_gpu_field_frame()
    assert first is not None and first.step == 0
    sim.advance(1, field_capture="bestEffort")
    second = sim.acquire_latest_gpu_field_frame()
    sim.advance(1, field_capture="bestEffort")
    third = sim.acquire_latest_gpu_field_frame()
    assert second is not None and third is not None
    result = sim.advance(1, field_capture="bestEffort")
    assert not result.field_frame_published
    assert result.dropped_field_frame_count == 1
    assert sim.field_capture_wait_count == 0
    assert sim.step_index == 3
    first.release()
    second.release()
    third.release()
    assert sim.advance(1, field_capture="bestEffort").field_frame_published
    sim.close()


def test_field_frame_lease_holds_its_frame():
    """A leased frame keeps its step's fields while later captures publish
    into the other slots; afterStep filters; the metadata carries the
    snapshot and the prepared geometry frame of that step; the device views
    read the same bytes as the host copy."""
    import torch
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird()
    sim = BirdFlowSimulation(config, bird, state, observation_buffer_count=2)
    sim.advance(3, field_capture="required")
    rho3, vel3 = sim.lattice.fields()
    snap3 = sim.snapshot()
    lease = sim.acquire_latest_gpu_field_frame()
    assert lease is not None and lease.step == 3
    assert lease.metadata["grid"] == (config.grid.x, config.grid.y, config.grid.z)
    assert lease.metadata["time_seconds"] == snap3.time
    assert bytes(lease.metadata["body"]) == bytes(snap3.body)
    assert lease.metadata["geometry"]["body_position"][:3] == pytest.approx(list(snap3.body.position), abs=1e-5)
    assert lease.metadata["pressure_scale_pascals"] > 0 and lease.metadata["reference_dynamic_pressure_pascals"] > 0
    sim.advance(2, field_capture="required")
    rho5, vel5 = sim.lattice.fields()
    assert not np.array_equal(rho3, rho5)
    r, v = lease.copy()
    assert np.array_equal(r, rho3) and np.array_equal(v, vel3)
    d, u = lease.device_views()
    td = torch.as_tensor(d, device="cuda")
    tu = torch.as_tensor(u, device="cuda")
    assert np.array_equal(td.cpu().numpy().ravel(), rho3)
    assert np.array_equal(tu.cpu().numpy().reshape(-1, 4)[:, :3], vel3)
    assert sim.acquire_latest_gpu_field_frame(after_step=5) is None
    newer = sim.acquire_latest_gpu_field_frame(after_step=4)
    assert newer is not None and newer.step == 5
    lease.release()
    lease.release()  # a no-op
    newer.release()
    sim.close()


def test_required_capture_waits_for_a_lease_release():
    """A required capture with every slot leased waits until another thread
    releases one (fieldCaptureWaitCount counts it); with a wait limit it
    fails with a timeout instead, runs no step, and the handle stays usable."""
    import threading
    import time
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird()
    sim = BirdFlowSimulation(config, bird, state, observation_buffer_count=1, field_wait_limit_ms=20000)
    lease = sim.acquire_latest_gpu_field_frame()
    t = threading.Thread(target=lambda: (time.sleep(0.3), lease.release()))
    t.start()
    res = sim.advance(2, field_capture="required")
    t.join()
    assert res.field_frame_published and sim.field_capture_wait_count >= 1
    sim.close()
    lat = lattice(cases.shear_wave(n=16, axis="y")[0])
    lat.set_observation_buffers(1, 200)
    held = lat.acquire_field_frame()
    with pytest.raises(BirdFlowError) as e:
        lat.advance(1, capture_fields="required")
    assert e.value.status == 11
    assert lat.step_index()[0] == 0
    held.release()
    lat.advance(1, capture_fields="required")
    assert lat.step_index()[0] == 1
    lat.close()


def test_release_after_stream_completion_and_restore_republishes():
    """releaseAfterCompletion(of:) on a torch stream frees the slot once the
    stream's work is done; a restore republishes slot 0 from the restored
    populations at the restored step."""
    import torch
    cfg, _, _, _ = cases.shear_wave(n=16, viscosity=0.03, magic=3.0 / 16.0, axis="y")
    lat = lattice(cfg)
    lat.advance(3, capture_fields=True)
    state = lat.save_state()
    rho3, vel3 = lat.fields()
    lease = lat.acquire_field_frame()
    d, _ = lease.device_views()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        total = torch.as_tensor(d, device="cuda").sum()
    lease.release_after(stream)
    stream.synchronize()
    assert float(total) == pytest.approx(float(rho3.astype(np.float64).sum()), rel=1e-5)
    res, _ = lat.advance(1, capture_fields="bestEffort")
    assert res.field_frame_published
    lat.advance(2)
    lat.restore_state(state)
    frame = lat.acquire_field_frame()
    assert frame is not None and frame.step == 3
    r, v = frame.copy()
    assert np.max(np.abs(r - rho3)) < 1e-6 and np.max(np.abs(v - vel3)) < 1e-6
    frame.release()
    lat.close()


def _flow_diagnostics_numpy(vel, mask, nx, ny, nz, cell_size, time_step):
    """deriveFlowDiagnostics (Visualization.metal:270-308) restated in NumPy
    float32 with the kernel's operation order."""
    f32 = np.float32
    u = vel.reshape(nz, ny, nx, 3).astype(f32)
    m = mask.reshape(nz, ny, nx) & 0x3F
    v2p = f32(cell_size) / f32(time_step)
    scale = f32(0.5) * v2p / f32(cell_size)
    ok = np.zeros((nz, ny, nx), bool)
    ok[1:-1, 1:-1, 1:-1] = True
    near = m.copy()
    near[:, :, 1:] |= m[:, :, :-1]
    near[:, :, :-1] |= m[:, :, 1:]
    near[:, 1:, :] |= m[:, :-1, :]
    near[:, :-1, :] |= m[:, 1:, :]
    near[1:, :, :] |= m[:-1, :, :]
    near[:-1, :, :] |= m[1:, :, :]
    ok &= near == 0
    c = (slice(1, -1),) * 3
    dx = (u[1:-1, 1:-1, 2:] - u[1:-1, 1:-1, :-2]) * scale
    dy = (u[1:-1, 2:, 1:-1] - u[1:-1, :-2, 1:-1]) * scale
    dz = (u[2:, 1:-1, 1:-1] - u[:-2, 1:-1, 1:-1]) * scale
    cx = dy[..., 2] - dz[..., 1]
    cy = dz[..., 0] - dx[..., 2]
    cz = dx[..., 1] - dy[..., 0]
    ts = (dx[..., 0] * dx[..., 0] + dy[..., 1] * dy[..., 1] + dz[..., 2] * dz[..., 2]
          + f32(2.0) * (dx[..., 1] * dy[..., 0] + dx[..., 2] * dz[..., 0] + dy[..., 2] * dz[..., 1]))
    vort = np.zeros((nz, ny, nx, 4), f32)
    q = np.zeros((nz, ny, nx), f32)
    vort[c] = np.stack([cx, cy, cz, np.sqrt(cx * cx + cy * cy + cz * cz)], axis=-1)
    q[c] = f32(-0.5) * ts
    vort[~ok] = 0.0
    q[~ok] = 0.0
    return vort.reshape(-1, 4), q.ravel(), ok.ravel().astype(np.uint8)


def test_flow_diagnostics_of_a_leased_frame_match_numpy():
    """Vorticity, Q criterion and validity of a leased frame of the flapping
    compact bird against the NumPy restatement of the same operations; the
    body of the captured step (held with the slot) is excluded, so a later
    step's motion does not change an older frame's diagnostics."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird()
    sim = BirdFlowSimulation(config, bird, state, observation_buffer_count=2)
    sim.advance(8, field_capture="required")
    lat = sim.lattice
    mask8 = lat.mask()
    lease = sim.acquire_latest_gpu_field_frame()
    _, vel = lease.copy()
    c = lat.config
    want = _flow_diagnostics_numpy(vel, mask8, c.nx, c.ny, c.nz, c.cell_size, c.time_step)
    # the wings move on; the leased frame keeps the occupancy of its own step
    for _ in range(40):
        sim.advance(10, field_capture="required")
        if not np.array_equal(lat.mask(), mask8):
            break
    assert not np.array_equal(lat.mask(), mask8)
    vort, q, valid = lease.flow_diagnostics()
    assert np.array_equal(valid, want[2])
    assert 0 < int(valid.sum()) < valid.size
    scale = float(np.max(np.abs(want[0][:, 3])))
    assert scale > 0.0
    np.testing.assert_allclose(vort, want[0], rtol=1e-6, atol=1e-6 * scale)
    qs = float(np.max(np.abs(want[1])))
    np.testing.assert_allclose(q, want[1], rtol=1e-6, atol=1e-6 * qs)
    print("exact:", np.array_equal(vort, want[0]), np.array_equal(q, want[1]))
    lease.release()
    sim.close()


def test_staged_kernel_wait_timeout_invalidates_the_handle():
    """The staged 16-bit kernel's bounded pipeline waits, made to run out by
    the test hook (one tile's loads withheld, a short wait limit): the advance
    fails with BFX_ERR_KERNEL, the handle refuses every later call with
    BFX_ERR_INVALIDATED (the reference's terminal command-buffer failure,
    BirdFlowSimulation.swift:2059-2095), and fresh handles on the same GPU
    step normally and agree bit for bit."""
    cfg, _, _, _ = cases.shear_wave(n=64, viscosity=0.02, amplitude=0.02, storage=L.STORAGE_F16_DEVIATION)
    lat = lattice(cfg)
    lat.advance(2)
    lib = lat.lib
    assert lib.bfx_test_stall_staged_kernel(lat.handle, 0, 1 << 14) == 0
    assert lib.bfx_advance(lat.handle, 1, 1, 0, None, 0, None) == 4  # BFX_ERR_KERNEL
    assert "timed out" in L.last_error(lat.handle)
    assert lib.bfx_advance(lat.handle, 1, 1, 0, None, 0, None) == 6  # BFX_ERR_INVALIDATED
    lat.close()
    runs = []
    for _ in range(2):
        fresh = lattice(cfg)
        fresh.advance(5)
        runs.append(fresh.populations())
        fresh.close()
    assert np.all(np.isfinite(runs[0])) and np.array_equal(runs[0], runs[1])
    # a handle without the staged kernel has no such hook
    cfg32, _, _, _ = cases.shear_wave(n=16, storage=L.STORAGE_F32)
    plain = lattice(cfg32)
    assert lib.bfx_test_stall_staged_kernel(plain.handle, 0, 1 << 14) == 10  # BFX_ERR_UNSUPPORTED
    plain.close()


def test_ledger_terms_match_the_oracle_restatement():
    """Each source term of the coupled momentum ledger (measureFluidMassMomentumChange
    and captureExternalFluidSources, BF.metal:4322-4552) per step on the
    compact free-flight bird, against the oracle's restatement on the same
    populations: fluid momentum before and after, the open far-field faces,
    the sponge, the persistent cut-link exchange and every count.  Both form
    each cell's terms in FP64 from the same FP32 populations and sum in FP64
    in different orders, so each term agrees to 1e-12 of its gross size (the
    sum of the magnitudes it cancels, bounded from the term's count) plus
    1e-9 of its value; the counts are equal."""
    from bfx.simulation import BirdFlowSimulation
    config, bird, state = cases.compact_bird(free_flight=True)
    sim = BirdFlowSimulation(config, bird, state)
    lat = sim.lattice
    cfg = lat.config
    rows = bird.packed()
    body = (state.position_meters, state.orientation_body_to_world, state.linear_velocity_meters_per_second,
            state.angular_velocity_body_radians_per_second)
    osim = oracle_twin(cfg, rows, body)
    mscale = float(cfg.force_to_physical) * float(cfg.time_step)
    terms = {"fluid_momentum_before": slice(1, 4), "fluid_momentum_after": slice(5, 8),
             "far_field_impulse": slice(9, 12), "link_exchange_impulse": slice(13, 16),
             "sponge_impulse": slice(17, 20)}
    n = int(cfg.nx) * int(cfg.ny) * int(cfg.nz)
    # gross size per term (lattice units): every population and |f + f'| here is below 1
    gross_of = {"fluid_momentum_before": lambda o: 19.0 * n, "fluid_momentum_after": lambda o: 19.0 * n,
                "far_field_impulse": lambda o: o[20], "link_exchange_impulse": lambda o: o[22],
                "sponge_impulse": lambda o: 19.0 * o[21]}
    seen = {k: 0.0 for k in terms}
    for step in range(12):
        sample = lat.advance_ledger(1)[0]
        osim.step(ledger=True)
        o = osim.ledger
        for name, sl in terms.items():
            g = np.array(getattr(sample, name), np.float64)
            ref = o[sl] * mscale
            seen[name] = max(seen[name], float(np.max(np.abs(ref))))
            tol = 1e-12 * gross_of[name](o) * mscale + 1e-9 * np.abs(ref)
            assert np.all(np.abs(g - ref) <= tol), (step + 1, name, g, ref)
        assert sample.far_field_links == int(o[20]), step + 1
        assert sample.sponge_cells == int(o[21]), step + 1
        assert sample.boundary_links == int(o[22]), step + 1
        assert sample.topology_cells == int(o[23]), step + 1
    # every term was exercised
    assert all(v > 0.0 for v in seen.values()), seen
    sim.close()
