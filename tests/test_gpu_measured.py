"""GPU keyframe replay of a measured bird surface sequence against the
oracle: the reference's committed dove surface (ValidationInputs/
deetjen-ob-f03-surface-v1, 2,157 vertices, 3,968 triangles in four parts, 144
frames at 1 kHz) when BFX_MEASURED_SURFACE_DIR points at it, else skipped.

Frames 60-63 (three keyframe intervals, 20 steps each) at 4 mm cells with the
validator's 0.75-cell half thickness and linear link fractions: masks, cut-link
sets and covered / uncovered counts bit-exact every step, loads within 1e-5,
populations within 1e-6 relative after the 60 steps.  The reference's own
archived Metal-versus-CPU envelope for this surface is an occupancy mismatch of
0 cells (Docs/BUILD_REPORT.md:155)."""
from __future__ import annotations

import os

import numpy as np
import pytest

import bfx.cases as cases
import bfx.measured as M
from test_gpu_parity import compare_loads, compare_pops, link_set, make_pair, oracle_links

pytestmark = pytest.mark.gpu


def test_measured_dove_surface_replay_matches_oracle():
    d = os.environ.get("BFX_MEASURED_SURFACE_DIR")
    if not d:
        pytest.skip("BFX_MEASURED_SURFACE_DIR is not set")
    surface = M.load(d)
    cfg, rows, body, mesh = cases.measured_surface_replay(surface, first=60, frames=4, steps_per_frame=20)
    lat, osim = make_pair(cfg, rows, body, mesh)
    assert np.array_equal(lat.mask(), osim.mcur)
    events = 0
    for step in range(60):
        lat.advance(1)
        osim.step()
        assert np.array_equal(lat.mask(), osim.mcur), f"mask step {step + 1}"
        cell, dd, _ = lat.links()
        oc, od = oracle_links(osim)
        assert np.array_equal(link_set(cell, dd), link_set(oc, od)), f"links step {step + 1}"
        ld = lat.loads()
        assert ld.covered_count == osim.loads.covered_count and ld.uncovered_count == osim.loads.uncovered_count
        events += ld.covered_count + ld.uncovered_count
        compare_loads(lat, osim, f"measured step {step + 1}")
    compare_pops(lat, osim, "measured surface after 60 steps")
    assert events > 0
    assert set(np.unique(lat.mask()).tolist()) >= {0, 1, 2, 3, 4}
    lat.close()
