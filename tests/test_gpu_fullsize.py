"""Full-size GPU parity on the benchmark configurations, step by step against
the CPU oracle (the reference's gate pattern of GPU against CPU per step,
Sources/BirdFlowMetal/MetalShearWaveValidation.swift:282-345):

  C2  256x128x128 RR3 channel past the ellipsoid, interpolated links, 50 steps
  C3  512x256x256 flapping plates (2 x 8,192 triangles), ray-root links, FP32, 10 steps
  C5  768x384x384 articulated bird (~145k triangles), RR3, free 6-DOF body, FP32, 3 steps

Every step: masks and cut-link sets bit-exact, loads within 1e-5 relative.
Populations within 1e-6 relative per value at the first, a middle and the
last step (each test also prints whether they were bit-identical).  The
comparisons run direction by direction so the host holds one extra
direction-sized FP64 buffer at a time.
"""
from __future__ import annotations

import ctypes as ct

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


def host_memory_gb() -> float:
    try:
        import psutil
        return psutil.virtual_memory().available / 1e9
    except Exception:
        return float("inf")


def make_pair(cfg, rows, body, mesh=None):
    lat = Lattice(cfg, bird_struct(rows), body_struct_from_tuple(body), mesh)
    osim = oracle_twin(cfg, rows, body, mesh)
    return lat, osim


def compare_pops_chunked(lat, osim, what):
    """Max relative difference per value and whether every value is equal."""
    g = lat.populations().reshape(19, -1)
    o = osim.pa.reshape(19, -1)
    worst, exact = 0.0, True
    for q in range(19):
        gq, oq = g[q], o[q]
        assert np.all(np.isfinite(gq)), f"{what}: non-finite populations in direction {q}"
        if np.array_equal(gq, oq):
            continue
        exact = False
        d = np.abs(gq.astype(np.float64) - oq.astype(np.float64))
        worst = max(worst, float(np.max(d / np.maximum(np.abs(oq.astype(np.float64)), 1e-12))))
    assert worst <= POP_RTOL, f"{what}: max relative population difference {worst:.3e}"
    return worst, exact


def compare_loads(lat, osim, what):
    ld = lat.loads()
    gf, of = np.array(ld.force), np.array(osim.loads.f64_force)
    gt, ot = np.array(ld.torque), np.array(osim.loads.f64_torque)
    fscale = max(np.max(np.abs(of)), 1e-30)
    tscale = max(np.max(np.abs(ot)), 1e-30)
    assert np.max(np.abs(gf - of)) <= LOAD_RTOL * fscale, f"{what}: force {gf} vs {of}"
    assert np.max(np.abs(gt - ot)) <= LOAD_RTOL * tscale, f"{what}: torque {gt} vs {ot}"
    assert ld.covered_count == osim.loads.covered_count and ld.uncovered_count == osim.loads.uncovered_count, what


def oracle_link_set(osim):
    """Sorted (cell * 32 + direction) keys of the oracle's cut links, counted first."""
    L2 = O.lib()
    n = L2.or_enumerate_links(ct.byref(osim.p), O.u8ptr(osim.mnext), O.u8ptr(osim.mcur), None, None, 0)
    cell = np.zeros(max(n, 1), np.uint32)
    d = np.zeros(max(n, 1), np.uint8)
    m = L2.or_enumerate_links(ct.byref(osim.p), O.u8ptr(osim.mnext), O.u8ptr(osim.mcur),
                              cell.ctypes.data_as(ct.POINTER(ct.c_uint32)), O.u8ptr(d), n)
    assert m == n
    return np.sort(cell[:n].astype(np.uint64) * 32 + d[:n].astype(np.uint64))


def gpu_link_set(lat):
    cell, d, q = lat.links()
    return np.sort(cell.astype(np.uint64) * 32 + d.astype(np.uint64)), cell, d, q


def test_c2_ellipsoid_channel_full_size_50_steps():
    cfg, rows, body, _ = cases.ellipsoid_channel()  # 256x128x128, RR3, interpolated links
    lat, osim = make_pair(cfg, rows, body)
    assert np.array_equal(lat.mask(), osim.mcur)
    gl, cell, d, q = gpu_link_set(lat)
    exact_all = True
    for step in range(1, 51):
        lat.advance(1)
        osim.step()
        compare_loads(lat, osim, f"C2 step {step}")
        if step in (1, 25, 50):
            _, exact = compare_pops_chunked(lat, osim, f"C2 step {step}")
            exact_all &= exact
    gl, cell, d, q = gpu_link_set(lat)
    assert np.array_equal(gl, oracle_link_set(osim))
    assert len(gl) > 1000
    # link fractions: the oracle's bisection for a sample of links
    c, _, _ = O.lattice()
    nx, ny = cfg.nx, cfg.ny
    for i in range(0, len(cell), max(1, len(cell) // 300)):
        g = int(cell[i])
        x, y, z = g % nx, (g // nx) % ny, g // (nx * ny)
        qq = int(d[i])
        oq = O.lib().or_ellipsoid_link_fraction(ct.byref(osim.p), ct.byref(osim.bird), ct.byref(osim.prep),
                                                x, y, z, x - c[qq][0], y - c[qq][1], z - c[qq][2])
        assert q[i] == np.float32(oq)
    print(f"C2 populations bit-identical at steps 1, 25, 50: {exact_all}")
    lat.close()


def test_c3_flapping_plates_full_size_10_steps():
    cfg, rows, body, mesh = cases.flapping_plates(storage=L.STORAGE_F32)  # 512x256x256, ray-root links, TRT
    lat, osim = make_pair(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    exact_all = True
    events = 0
    for step in range(1, 11):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"C3 mask step {step}"
        gl, cell, d, q = gpu_link_set(lat)
        assert np.array_equal(gl, oracle_link_set(osim)), f"C3 links step {step}"
        compare_loads(lat, osim, f"C3 step {step}")
        events += osim.loads.covered_count + osim.loads.uncovered_count
        if step in (1, 5, 10):
            _, exact = compare_pops_chunked(lat, osim, f"C3 step {step}")
            exact_all &= exact
    assert events > 0
    # sampled ray-root fractions of the last step, bit for bit
    tris = mesh["tris"].astype(np.uint32).ravel()
    c, _, _ = O.lattice()
    nx, ny = cfg.nx, cfg.ny
    sampled = range(0, len(cell), max(1, len(cell) // 300))
    for i in sampled:
        g = int(cell[i])
        x, y, z = g % nx, (g // nx) % ny, g // (nx * ny)
        qq = int(d[i])
        oq = O.lib().or_mesh_ray_root(ct.byref(osim.p), O.fptr(osim.mesh_pos),
                                      tris.ctypes.data_as(ct.POINTER(ct.c_uint32)), mesh["tris"].shape[0],
                                      cfg.mesh_half_thickness, osim.keys.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                      x, y, z, x - c[qq][0], y - c[qq][1], z - c[qq][2])
        assert q[i] == np.float32(oq), (i, float(q[i]), oq)
    print(f"C3 populations bit-identical at steps 1, 5, 10: {exact_all}")
    lat.close()


def test_c5_articulated_bird_full_size_3_steps():
    if host_memory_gb() < 60.0:
        pytest.skip(f"the oracle twin of the 768x384x384 lattice needs ~45 GB of host memory "
                    f"({host_memory_gb():.0f} GB available)")
    cfg, rows, body, mesh = cases.articulated_bird(storage=L.STORAGE_F32)  # 768x384x384, RR3, free flight
    lat, osim = make_pair(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    exact_all = True
    for step in range(1, 4):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"C5 mask step {step}"
        gl, _, _, _ = gpu_link_set(lat)
        assert np.array_equal(gl, oracle_link_set(osim)), f"C5 links step {step}"
        compare_loads(lat, osim, f"C5 step {step}")
        b = lat.body()
        assert rel_diff(list(b.position), list(osim.body64.position)) < 1e-12
        assert np.allclose(list(b.velocity), list(osim.body64.velocity), rtol=1e-9, atol=1e-12)
    _, exact = compare_pops_chunked(lat, osim, "C5 step 3")
    exact_all &= exact
    print(f"C5 populations bit-identical at step 3: {exact_all}")
    lat.close()
