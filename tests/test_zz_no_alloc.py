"""The allocation-free mass/momentum entry point against the allocating one.

bfx_fluid_mass_momentum_noalloc serves callers that cannot allocate device
memory when they need the global fluid mass and momentum (an application
whose device memory is reserved by its own allocator, or a loop that must not
stall on cudaMalloc's device synchronisation).  Here the test itself
allocates the device input and output with torch, calls the entry point
through the C ABI twice in a row on a lattice with solid cells, and compares
each result with bfx_fluid_mass_momentum on the same state.  Both are FP64 sums of the same
FP32 values in different orders, so they agree to 1e-12 relative (the
tolerance of the other FP64 reduction tests).  This file is collected last.
"""
from __future__ import annotations

import numpy as np
import pytest

import bfx._lib as L
import bfx.cases as cases
from bfx.simulation import Lattice, bird_struct
from helpers import body_struct_from_tuple

pytestmark = pytest.mark.gpu


def _call(lib, pops, mask, nx, ny, nz, out):
    return lib.bfx_fluid_mass_momentum_noalloc(pops.data_ptr(), mask.data_ptr() if mask is not None else None,
                                               nx, ny, nz, out.data_ptr())


def test_no_alloc_mass_momentum_matches_allocating_entry_point():
    import torch
    cfg, rows, body, _ = cases.ellipsoid_channel(nx=64, ny=32, nz=32, radii=(9.0, 5.0, 4.5), inflow=0.05,
                                                 viscosity=0.02)
    lat = Lattice(cfg, bird_struct(rows), body_struct_from_tuple(body))
    lib = L.load()
    for call in range(2):
        lat.advance(3 + call)
        ref = lat.mass_momentum()
        pops = torch.from_numpy(lat.populations().ravel().copy()).cuda()
        mask = torch.from_numpy(lat.mask().copy()).cuda()
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _call(lib, pops, mask, cfg.nx, cfg.ny, cfg.nz, out)
        assert rc == 0, L.last_error(None)
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= 1e-12 * abs(ref[0]), (call, got, ref)
    lat.close()


def test_no_alloc_rejects_lattices_beyond_its_scratch():
    import torch
    lib = L.load()
    pops = torch.zeros(19, dtype=torch.float32, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = _call(lib, pops, None, 2048, 2048, 4, out)  # 16.8M cells > 8,388,608
    assert rc == 9  # BFX_ERR_CAPACITY
    assert "exceeds" in L.last_error(None)
