"""Measured bird surface sequences: the reference's on-disk format for an
indexed, keyframed bird surface and its replay through the keyframe mesh.

The format and its checks follow MeasuredBirdSurfaceSequence.load
(Sources/BirdFlowMetal/MeasuredBirdSurfaceSequence.swift:280-534): a
``manifest.json`` (schema 1, a complete derived surface in metres, strictly
increasing frame times, fixed indexed topology, readiness flags) next to two
SHA-256-locked binaries, ``positions.f32le`` (frame-major, vertex-major,
xyz float32) and ``triangles.u16le`` (triangle-major uint16 indices), and four
canonical components (body, leftWing, rightWing, tail = parts 1-4) whose
vertex and triangle ranges tile the topology.  The reference caps the
triangle count at 4,096 for its 12-bit triangle identifiers; the library's
64-bit raster keys have no such cap, so that bound is not enforced here.

``MeasuredSurface.keyframe_mesh`` turns a window of frames into the
``bfx_mesh`` keyframe replay (prepareIndexedBirdSurface, BF.metal:1585-1622):
all vertices on the body segment, the frames' positions as body-frame
offsets relative to the body origin, times relative to the first frame.
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import dataclass

import numpy as np

CANONICAL_COMPONENTS = (("body", 1), ("leftWing", 2), ("rightWing", 3), ("tail", 4))


class MeasuredSurfaceError(ValueError):
    """invalidMeasuredSurface (MeasuredBirdSurfaceSequence.swift:534-540)."""


@dataclass
class MeasuredSurface:
    dataset: str
    times: np.ndarray          # (frames,) seconds
    positions: np.ndarray      # (frames, vertices, 3) float32 metres
    triangles: np.ndarray      # (triangles, 3) uint32
    triangle_parts: np.ndarray  # (triangles,) uint8, 1 body, 2 left wing, 3 right wing, 4 tail
    sample_rate_hz: float
    manifest_sha256: str

    @property
    def frame_count(self) -> int:
        return int(self.positions.shape[0])

    @property
    def vertex_count(self) -> int:
        return int(self.positions.shape[1])

    def keyframe_mesh(self, first: int, count: int) -> dict:
        """The mesh dict of bfx.simulation.Lattice for a replay of frames
        first ... first + count - 1, with times counted from the first."""
        if count < 2 or first < 0 or first + count > self.frame_count:
            raise MeasuredSurfaceError(f"frame window [{first}, {first + count}) outside 0..{self.frame_count}")
        pts = np.ascontiguousarray(self.positions[first:first + count], np.float32)
        times = (self.times[first:first + count] - self.times[first]).astype(np.float32)
        return {"local": pts[0].copy(), "segment": np.zeros(self.vertex_count, np.uint8),
                "tris": self.triangles.astype(np.uint32), "tri_part": self.triangle_parts.astype(np.uint8),
                "kf_times": times, "kf_points": pts.reshape(count, -1)}


def _fail(msg: str):
    raise MeasuredSurfaceError(msg)


def _locked(directory: str, record: dict, fmt: str, layout: str) -> bytes:
    name = record.get("file", "")
    if not name or os.path.basename(name) != name or name in (".", ".."):
        _fail(f"unsafe binary member path: {name}")
    if record.get("format") != fmt or record.get("layout") != layout:
        _fail(f"binary {name} is not {fmt} / {layout}")
    try:
        with open(os.path.join(directory, name), "rb") as fh:
            data = fh.read()
    except OSError as e:
        _fail(f"unable to read {name}: {e}")
    if record.get("bytes") != len(data) or record.get("sha256") != hashlib.sha256(data).hexdigest():
        _fail(f"binary lock mismatch for {name}")
    return data


def load(directory: str) -> MeasuredSurface:
    """Reads and checks a measured surface sequence directory."""
    path = os.path.join(directory, "manifest.json")
    try:
        raw = open(path, "rb").read()
        m = json.loads(raw)
    except (OSError, ValueError) as e:
        _fail(f"unable to decode manifest.json: {e}")
    if m.get("schemaVersion") != 1:
        _fail("schemaVersion must be 1")
    if m.get("scientificTier") != "derived-measured-complete-surface":
        _fail("scientificTier is not a complete derived surface")
    if m.get("coordinateFrame", {}).get("units") != "meters":
        _fail("coordinate units must be meters")
    fr = m.get("frames", {})
    times = np.asarray(fr.get("timesSeconds", []), np.float64)
    rate = fr.get("sampleRateHertz")
    if not (fr.get("count", 0) >= 2 and fr["count"] == len(fr.get("frameNumbers", [])) == len(times)
            and isinstance(rate, (int, float)) and np.isfinite(rate) and rate > 0
            and fr.get("interpolation") == "piecewise-linear-nonperiodic"
            and fr.get("endpointVelocity") == "one-sided-adjacent-frame" and not fr.get("periodic", True)):
        _fail("frame timing contract is invalid")
    if not (np.all(np.isfinite(times)) and np.all(np.diff(times) > 0)):
        _fail("frame times must be finite and strictly increasing")
    topo = m.get("topology", {})
    nv, nt = int(topo.get("vertexCount", 0)), int(topo.get("triangleCount", 0))
    if not (0 < nv <= 65535 and nt > 0 and topo.get("indexType") == "uint16-little-endian"
            and topo.get("fixedAcrossFrames")):
        _fail("indexed topology is not a fixed uint16 topology")
    ready = m.get("readiness", {})
    if not (ready.get("completeBirdSurfaceReady") and ready.get("cpuParityRequired")
            and not ready.get("quantitativeForceAcceptanceReady")):
        _fail("scientific readiness boundary is inconsistent")
    b = m.get("binary", {})
    pos = _locked(directory, b.get("positions", {}), "float32-little-endian", "frame-major, vertex-major, xyz")
    tri = _locked(directory, b.get("triangles", {}), "uint16-little-endian",
                  "triangle-major, three global vertex indices")
    frames = len(times)
    if len(pos) != frames * nv * 3 * 4 or len(tri) != nt * 3 * 2:
        _fail("binary scalar count does not match manifest topology")
    positions = np.frombuffer(pos, "<f4").reshape(frames, nv, 3).astype(np.float32)
    if not np.all(np.isfinite(positions)):
        _fail("position stream contains a nonfinite value")
    triangles = np.frombuffer(tri, "<u2").reshape(nt, 3).astype(np.uint32)
    if np.any(triangles >= nv):
        _fail("triangle stream contains an out-of-range vertex")
    comps = topo.get("components", [])
    if [(c.get("name"), c.get("partIdentifier")) for c in comps] != list(CANONICAL_COMPONENTS):
        _fail("component names and part identifiers must be canonical")
    parts = np.zeros(nt, np.uint8)
    next_v = next_t = 0
    for c in comps:
        vo, vc, to, tc = c["vertexOffset"], c["vertexCount"], c["triangleOffset"], c["triangleCount"]
        if vo != next_v or to != next_t or vc <= 0 or tc <= 0:
            _fail("component ranges must be positive and contiguous")
        if vo + vc > nv or to + tc > nt:
            _fail("component range exceeds topology")
        corners = triangles[to:to + tc]
        if np.any(corners < vo) or np.any(corners >= vo + vc):
            _fail("triangle crosses a component vertex range")
        parts[to:to + tc] = c["partIdentifier"]
        next_v, next_t = vo + vc, to + tc
    if next_v != nv or next_t != nt:
        _fail("component ranges do not cover the topology exactly")
    return MeasuredSurface(dataset=str(m.get("datasetIdentifier", "")), times=times, positions=positions,
                           triangles=triangles, triangle_parts=parts, sample_rate_hz=float(rate),
                           manifest_sha256=hashlib.sha256(raw).hexdigest())
