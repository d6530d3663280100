"""Keyframe replay of a mesh (MeasuredBirdSurfaceSequence; prepareIndexedBirdSurface,
BF.metal:1585-1622) on the CPU: the oracle's interval rule and linear
interpolation against values worked by hand, and the configuration checks the
library runs before any device work."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

import bfx._lib as L
import bfx.cases as cases
import oracle as O


def _prepare(times, points, t):
    prep = O.Prepared()
    prep.orientation.v[:] = [0.0, 0.0, 0.0, 1.0]
    nv = points.shape[1]
    pos = np.zeros(4 * nv, np.float32)
    vel = np.zeros(4 * nv, np.float32)
    tt = np.ascontiguousarray(times, np.float32)
    pp = np.ascontiguousarray(points, np.float32).ravel()
    O.lib().or_mesh_prepare_keyframes(ct.byref(prep), O.fptr(tt), len(tt), O.fptr(pp), nv, t, 1.0, O.fptr(pos),
                                      O.fptr(vel))
    return pos.reshape(-1, 4)[:, :3], vel.reshape(-1, 4)[:, :3]


def test_keyframe_interval_rule_and_interpolation():
    times = [0.0, 1.0, 3.0]
    pts = np.array([[[0.0, 0.0, 0.0]], [[1.0, 0.0, 0.0]], [[3.0, 2.0, 0.0]]])
    # inside the first interval
    p, v = _prepare(times, pts, 0.5)
    assert np.array_equal(p[0], [0.5, 0.0, 0.0]) and np.array_equal(v[0], [1.0, 0.0, 0.0])
    # an exact interior keyframe opens the following interval
    p, v = _prepare(times, pts, 1.0)
    assert np.array_equal(p[0], [1.0, 0.0, 0.0]) and np.array_equal(v[0], [1.0, 1.0, 0.0])
    # past the last keyframe: the last interval, blend clamped to 1
    p, v = _prepare(times, pts, 5.0)
    assert np.array_equal(p[0], [3.0, 2.0, 0.0]) and np.array_equal(v[0], [1.0, 1.0, 0.0])
    # before the first: the first interval, blend clamped to 0
    p, v = _prepare(times, pts, -1.0)
    assert np.array_equal(p[0], [0.0, 0.0, 0.0]) and np.array_equal(v[0], [1.0, 0.0, 0.0])


def test_keyframed_case_is_a_body_mesh():
    cfg, rows, body, mesh = cases.keyframed_plates()
    nv = mesh["local"].shape[0]
    assert mesh["kf_points"].shape == (24, nv, 3) and mesh["kf_times"].shape == (24,)
    assert np.all(np.diff(mesh["kf_times"]) > 0) and not np.any(mesh["segment"])


@pytest.mark.parametrize("defect", ["unsorted", "joints", "segment", "single"])
def test_invalid_keyframes_are_rejected_before_device_work(defect):
    from bfx.simulation import BirdFlowError, Lattice, bird_struct
    from helpers import body_struct_from_tuple
    cfg, rows, body, mesh = cases.keyframed_plates()
    mesh = dict(mesh)
    if defect == "unsorted":
        t = mesh["kf_times"].copy()
        t[3], t[4] = t[4], t[3]
        mesh["kf_times"] = t
    elif defect == "joints":
        mesh["joints"] = [dict(origin=(0.0, 4.0, 0.0), axis=(1.0, 0.0, 0.0), bias=0.0, amplitude=0.1, phase=0.0)]
    elif defect == "segment":
        seg = mesh["segment"].copy()
        seg[0] = 1
        mesh["segment"] = seg
    else:
        mesh["kf_times"] = mesh["kf_times"][:1]
        mesh["kf_points"] = mesh["kf_points"][:1]
    with pytest.raises(BirdFlowError) as e:
        Lattice(cfg, bird_struct(rows), body_struct_from_tuple(body), mesh)
    assert e.value.status == 7
