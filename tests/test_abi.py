"""The C-ABI library loads without a GPU, exports every symbol include/bfx.h
declares, and its structures have the layout the ctypes mirror assumes."""
from __future__ import annotations

import ctypes as ct
import os
import re
import subprocess
import tempfile

import pytest

import bfx._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bfx.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^BFX_API\s+[\w\s\*]+?\b(bfx_\w+)\s*\(", text, re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.load()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(L.EXPORTED)
    assert lib.bfx_abi_version() == 3


def test_no_device_reports_unavailable_not_crash():
    lib = L.load()
    n = ct.c_int(-1)
    rc = lib.bfx_device_count(ct.byref(n))
    assert rc in (0, 1)
    if rc == 1:
        assert n.value == 0


def test_struct_layout_matches_c_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "bfx.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(bfx_config), sizeof(bfx_bird),
         sizeof(bfx_body_state), sizeof(bfx_mesh), sizeof(bfx_loads), sizeof(bfx_run_sample),
         sizeof(bfx_safety_record), sizeof(bfx_snapshot_data), sizeof(bfx_advance_result),
         offsetof(bfx_config, mesh_half_thickness), sizeof(bfx_adjoint_objective), sizeof(bfx_adjoint_result),
         sizeof(bfx_ledger_sample), offsetof(bfx_ledger_sample, far_field_links), sizeof(bfx_field_frame),
         offsetof(bfx_field_frame, geometry), offsetof(bfx_field_frame, density), sizeof(bfx_flapping_wing));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    sizes = [int(x) for x in out]
    mine = [ct.sizeof(L.Config), ct.sizeof(L.Bird), ct.sizeof(L.BodyState), ct.sizeof(L.Mesh), ct.sizeof(L.Loads),
            ct.sizeof(L.RunSample), ct.sizeof(L.SafetyRecord), ct.sizeof(L.Snapshot), ct.sizeof(L.AdvanceResult),
            L.Config.mesh_half_thickness.offset, ct.sizeof(L.AdjointObjective), ct.sizeof(L.AdjointResult),
            ct.sizeof(L.LedgerSample), L.LedgerSample.far_field_links.offset, ct.sizeof(L.FieldFrame),
            L.FieldFrame.geometry.offset, L.FieldFrame.density.offset, ct.sizeof(L.FlappingWing)]
    assert sizes == mine
    # GPUBirdParameters is 13 float4, GPUFlappingWingParameters 4 (GPUDataLayoutTests.swift:5-40)
    assert ct.sizeof(L.Bird) == 13 * 16
    assert ct.sizeof(L.FlappingWing) == 4 * 16


def test_create_without_device_fails_cleanly():
    from bfx.simulation import BirdFlowError, Lattice, default_config
    lib = L.load()
    n = ct.c_int(0)
    if lib.bfx_device_count(ct.byref(n)) == 0 and n.value > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(BirdFlowError) as e:
        Lattice(default_config(16, 16, 16, omega_plus=1.0, omega_minus=1.0))
    assert e.value.status == 1


def test_invalid_configurations_are_rejected_before_any_device_work():
    from bfx.simulation import BirdFlowError, Lattice, default_config
    bad = [
        default_config(2, 16, 16),                                         # grid too small
        default_config(16, 16, 16, omega_plus=2.5),                        # unstable relaxation
        default_config(16, 16, 16, face_bc=[1, 0, 0, 0, 0, 0]),            # half-periodic axis
        default_config(16, 16, 16, far_field=[0.2, 0, 0, 1]),              # Mach > 0.15
        default_config(16, 16, 16, geometry=1),                            # geometry without bird
    ]
    for cfg in bad:
        with pytest.raises(BirdFlowError) as e:
            Lattice(cfg)
        assert e.value.status == 7
