"""Measured bird surface sequences (bfx.measured): the reference's loader
checks (MeasuredBirdSurfaceSequence.load, MeasuredBirdSurfaceSequence.swift:
280-534) on small synthetic sequences written here, the keyframe mesh a
window of frames becomes, and - when BFX_MEASURED_SURFACE_DIR points at a
sequence directory such as the reference's committed dove surface
(ValidationInputs/deetjen-ob-f03-surface-v1) - that it loads."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

import bfx.measured as M


def write_sequence(d, frames=3, mutate=None):
    """Four components of one triangle each (3 vertices per component)."""
    nv, nt = 12, 4
    rng = np.random.default_rng(1)
    pos = rng.uniform(-0.1, 0.1, (frames, nv, 3)).astype("<f4")
    tris = np.arange(12, dtype="<u2").reshape(4, 3)
    comps = [{"name": n, "partIdentifier": p, "evidenceClass": "synthetic", "vertexOffset": 3 * i, "vertexCount": 3,
              "triangleOffset": i, "triangleCount": 1} for i, (n, p) in enumerate(M.CANONICAL_COMPONENTS)]
    m = {"schemaVersion": 1, "scientificTier": "derived-measured-complete-surface", "datasetIdentifier": "synthetic",
         "coordinateFrame": {"units": "meters"},
         "frames": {"count": frames, "frameNumbers": list(range(frames)), "timesSeconds": [0.001 * k for k in range(frames)],
                    "sampleRateHertz": 1000.0, "interpolation": "piecewise-linear-nonperiodic",
                    "endpointVelocity": "one-sided-adjacent-frame", "periodic": False},
         "topology": {"vertexCount": nv, "triangleCount": nt, "indexType": "uint16-little-endian",
                      "fixedAcrossFrames": True, "metalTriangleIdentifierLimit": 4096, "components": comps},
         "readiness": {"completeBirdSurfaceReady": True, "cpuParityRequired": True,
                       "quantitativeForceAcceptanceReady": False},
         "binary": {}}
    blobs = {"positions": ("positions.f32le", pos.tobytes(), "float32-little-endian", "frame-major, vertex-major, xyz"),
             "triangles": ("triangles.u16le", tris.tobytes(), "uint16-little-endian",
                           "triangle-major, three global vertex indices")}
    if mutate:
        mutate(m, blobs)
    for key, (name, data, fmt, layout) in blobs.items():
        open(os.path.join(d, name), "wb").write(data)
        m["binary"].setdefault(key, {"file": name, "bytes": len(data), "sha256": hashlib.sha256(data).hexdigest(),
                                     "format": fmt, "layout": layout})
    json.dump(m, open(os.path.join(d, "manifest.json"), "w"))
    return pos, tris


def test_synthetic_sequence_loads_and_becomes_a_keyframe_mesh(tmp_path):
    pos, tris = write_sequence(str(tmp_path), frames=4)
    s = M.load(str(tmp_path))
    assert s.frame_count == 4 and s.vertex_count == 12
    assert np.array_equal(s.positions, pos) and np.array_equal(s.triangles, tris.astype(np.uint32))
    assert s.triangle_parts.tolist() == [1, 2, 3, 4]
    mesh = s.keyframe_mesh(1, 3)
    assert np.allclose(mesh["kf_times"], [0.0, 0.001, 0.002])
    assert mesh["kf_points"].shape == (3, 36) and np.array_equal(mesh["local"], pos[1])
    assert not mesh["segment"].any()
    with pytest.raises(M.MeasuredSurfaceError):
        s.keyframe_mesh(3, 2)


def _mutations():
    def times(m, b):
        m["frames"]["timesSeconds"][1] = m["frames"]["timesSeconds"][0]

    def parts(m, b):
        m["topology"]["components"][1]["partIdentifier"] = 5

    def crossing(m, b):
        t = np.arange(12, dtype="<u2").reshape(4, 3)
        t[0, 0] = 5
        b["triangles"] = (b["triangles"][0], t.tobytes(), b["triangles"][2], b["triangles"][3])

    def lock(m, b):
        m["binary"]["positions"] = {"file": "positions.f32le", "bytes": len(b["positions"][1]), "sha256": "0" * 64,
                                    "format": "float32-little-endian", "layout": "frame-major, vertex-major, xyz"}

    def units(m, b):
        m["coordinateFrame"]["units"] = "millimeters"

    def ready(m, b):
        m["readiness"]["quantitativeForceAcceptanceReady"] = True

    def path(m, b):
        m["binary"]["positions"] = {"file": "../positions.f32le", "bytes": 0, "sha256": "",
                                    "format": "float32-little-endian", "layout": "frame-major, vertex-major, xyz"}
    return {"times": (times, "strictly increasing"), "parts": (parts, "canonical"),
            "crossing": (crossing, "crosses a component"), "lock": (lock, "lock mismatch"),
            "units": (units, "meters"), "ready": (ready, "readiness"), "path": (path, "unsafe")}


@pytest.mark.parametrize("name", sorted(_mutations()))
def test_loader_refuses_what_the_reference_refuses(tmp_path, name):
    mutate, message = _mutations()[name]
    write_sequence(str(tmp_path), mutate=mutate)
    with pytest.raises(M.MeasuredSurfaceError) as e:
        M.load(str(tmp_path))
    assert message in str(e.value)


def test_measured_dove_sequence_loads_when_present():
    d = os.environ.get("BFX_MEASURED_SURFACE_DIR")
    if not d:
        pytest.skip("BFX_MEASURED_SURFACE_DIR is not set")
    s = M.load(d)
    assert s.frame_count >= 2 and s.triangles.shape[0] > 0
    assert set(np.unique(s.triangle_parts).tolist()) == {1, 2, 3, 4}
    assert np.all(np.diff(s.times) > 0)
