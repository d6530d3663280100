"""Checkpoint archive layout on the host (bfx.checkpoint): manifest with byte
counts and SHA-256 digests, atomic replacement, and the refusals of the
reference's CheckpointArchive.read (CheckpointArchive.swift:82-110): unsupported
schema, empty numerical state, checksum mismatch."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import bfx.checkpoint as C


def files(seed=0):
    rng = np.random.default_rng(seed)
    return {C.POPULATIONS: rng.random(19 * 64, dtype=np.float32).tobytes(),
            C.SOLID_MASK: rng.integers(0, 3, 64, dtype=np.uint8).tobytes(),
            C.RESTART_STATE: rng.integers(0, 255, 4096, dtype=np.uint8).tobytes()}


def test_round_trip_and_manifest(tmp_path):
    path = str(tmp_path / "a")
    fs = files()
    C.write_archive(path, {"step": 12, "timeSeconds": 0.5}, fs)
    manifest, got = C.read_archive(path)
    assert got == fs
    assert manifest["schema"] == C.SCHEMA_VERSION and manifest["step"] == 12
    assert manifest["populationBytes"] == len(fs[C.POPULATIONS])
    assert manifest["solidMaskSHA256"] == C.sha256(fs[C.SOLID_MASK])
    # the reference's manifest keys are sorted and pretty-printed
    text = open(os.path.join(path, C.MANIFEST)).read()
    assert text == json.dumps(manifest, indent=2, sort_keys=True)


def test_replaces_the_destination_atomically(tmp_path):
    path = str(tmp_path / "a")
    C.write_archive(path, {"step": 1}, files(1))
    C.write_archive(path, {"step": 2}, files(2))
    manifest, got = C.read_archive(path)
    assert manifest["step"] == 2 and got == files(2)
    assert sorted(os.listdir(tmp_path)) == ["a"]  # no temporary directory left behind


@pytest.mark.parametrize("name", [C.POPULATIONS, C.SOLID_MASK, C.RESTART_STATE])
def test_refuses_a_flipped_byte(tmp_path, name):
    path = str(tmp_path / "a")
    C.write_archive(path, {}, files())
    f = os.path.join(path, name)
    data = bytearray(open(f, "rb").read())
    data[len(data) // 2] ^= 0x80
    open(f, "wb").write(bytes(data))
    with pytest.raises(C.CheckpointError, match="checksum"):
        C.read_archive(path)


def test_refuses_schema_size_and_missing_files(tmp_path):
    path = str(tmp_path / "a")
    C.write_archive(path, {}, files())
    m = json.load(open(os.path.join(path, C.MANIFEST)))
    m["schema"] = 2
    json.dump(m, open(os.path.join(path, C.MANIFEST), "w"))
    with pytest.raises(C.CheckpointError, match="schema"):
        C.read_archive(path)
    m["schema"] = 1
    m["solidMaskBytes"] = 0
    json.dump(m, open(os.path.join(path, C.MANIFEST), "w"))
    with pytest.raises(C.CheckpointError, match="empty"):
        C.read_archive(path)
    C.write_archive(path, {}, files())
    os.remove(os.path.join(path, C.RESTART_STATE))
    with pytest.raises(C.CheckpointError):
        C.read_archive(path)
    with pytest.raises(C.CheckpointError, match="manifest"):
        C.read_archive(str(tmp_path / "missing"))


def test_ledger_report_gates_on_the_relative_residuals():
    """The ledger report's RMS arithmetic and gates (CoupledMomentumLedger.swift:36-60)
    on synthetic samples: 1 % boundary residual fails a 0.5 % gate, 0.1 % passes."""
    import bfx._lib as L
    from bfx.simulation import ledger_report

    def sample(step, residual):
        s = L.LedgerSample()
        s.step = step
        s.aerodynamic_impulse[:] = [0.0, 0.0, 2.0]
        s.boundary_residual[:] = [0.0, 0.0, 2.0 * residual]
        s.external_impulse[:] = [0.0, 0.0, 1.0]
        s.system_residual[:] = [0.0, 0.0, 1.0e-4]
        return s

    bad = ledger_report([sample(i, 0.01) for i in range(4)], 1e-4, 0.005)
    good = ledger_report([sample(i, 0.001) for i in range(4)], 1e-4, 0.005)
    assert not bad["passed"] and good["passed"]
    assert abs(good["relative_rms_boundary_closure_residual"] - 0.001) < 1e-12
    assert abs(good["rms_aerodynamic_impulse"] - 2.0) < 1e-12
