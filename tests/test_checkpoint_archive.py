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


def test_struct_dict_round_trip():
    """struct_from_dict inverts struct_dict for the structures an archive's
    manifest holds (configuration, bird, body), nested arrays included."""
    import json
    import bfx._lib as L
    import bfx.cases as cases
    import bfx.checkpoint as C
    from bfx.simulation import bird_struct
    from helpers import body_struct_from_tuple
    cfg, rows, body, _ = cases.flapping_plates(nx=96, ny=64, nz=64)
    for s in (cfg, bird_struct(rows), body_struct_from_tuple(body)):
        d = json.loads(json.dumps(C.struct_dict(s)))
        back = C.struct_from_dict(type(s), d)
        assert bytes(back) == bytes(s)


def test_from_archive_rebuilds_a_valid_configuration(tmp_path):
    """Lattice.from_archive rebuilds the configuration from the manifest: the
    rebuilt configuration passes the library's checks and the call stops at
    device creation on a machine without a GPU (deviceUnavailable, not
    invalidConfiguration); a mesh configuration without its mesh is refused."""
    import ctypes as ct
    import bfx._lib as L
    import bfx.cases as cases
    import bfx.checkpoint as C
    from bfx.simulation import BirdFlowError, Lattice, bird_struct
    from helpers import body_struct_from_tuple
    lib = L.load()
    n = ct.c_int(0)
    if lib.bfx_device_count(ct.byref(n)) == 0 and n.value > 0:
        pytest.skip("a CUDA device is present")
    cfg, rows, body, _ = cases.ellipsoid_channel(nx=64, ny=32, nz=32, radii=(8.0, 4.0, 4.0))
    manifest = {"configuration": C.struct_dict(cfg), "bird": C.struct_dict(bird_struct(rows)),
                "body": C.struct_dict(body_struct_from_tuple(body)), "step": 0, "timeSeconds": 0.0}
    files = {C.POPULATIONS: b"\\0" * 16, C.SOLID_MASK: b"\\0" * 16, C.RESTART_STATE: b"\\0" * 16}
    C.write_archive(str(tmp_path / "a"), manifest, files)
    with pytest.raises(BirdFlowError) as e:
        Lattice.from_archive(str(tmp_path / "a"))
    assert e.value.status == 1
    mcfg, mrows, mbody, _ = cases.flapping_plates(nx=96, ny=64, nz=64)
    manifest["configuration"] = C.struct_dict(mcfg)
    C.write_archive(str(tmp_path / "m"), manifest, files)
    with pytest.raises(C.CheckpointError, match="mesh"):
        Lattice.from_archive(str(tmp_path / "m"))
