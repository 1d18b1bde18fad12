"""Concave polygon decomposition on the host (PhysicsGeometry::preparePolygonOutline, decomposeConcave with the
Bayazit method and its ear-clipping fallback, limitConvexPieceVertexCount with the fan split:
PhysicsGeometry.cpp:175-212, PolygonDecomposition.cpp:704-831) against the reference engine's own functions,
compiled from its sources (oracle/_ref): for stars, combs, spirals, convex outlines above the 16-vertex limit and
refused outlines, the same pieces in the same order with the same vertices, bit for bit. No device is needed:
ag2d_decompose_polygon runs on the host."""
import ctypes
import math

import numpy as np
import pytest

ag2d = pytest.importorskip("ag2d")
from oracle import refapi  # noqa: E402


def _ours(xy):
    v = np.ascontiguousarray(np.asarray(xy, np.float32).reshape(-1))
    out = np.zeros(8192, np.float32)
    counts = np.zeros(1024, np.uint32)
    k = ctypes.c_uint32(0)
    f = ctypes.POINTER(ctypes.c_float)
    code = ag2d.lib.ag2d_decompose_polygon(v.ctypes.data_as(f), v.size // 2, out.ctypes.data_as(f), out.size // 2,
                                           counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), counts.size,
                                           ctypes.byref(k))
    if code == ag2d.ERR_INVALID_ARG:
        return None
    assert code == 0, ag2d.lib.ag2d_last_error_string()
    pieces, at = [], 0
    for c in counts[:k.value].tolist():
        pieces.append(out[2 * at:2 * (at + c)].reshape(-1, 2).copy())
        at += c
    return pieces


def _star(rng, n):
    t = np.sort(rng.uniform(0, 2 * math.pi, n))
    r = rng.uniform(0.3, 2.0, n)
    return np.stack([r * np.cos(t), r * np.sin(t)], 1) + rng.uniform(-3, 3, 2)


def _comb(teeth, depth=1.5, width=0.4):
    top = [(0.0, 0.0), (teeth * 2 * width, 0.0)]
    for k in range(teeth, 0, -1):
        x = (2 * k - 1) * width
        top += [(x + width, depth), (x, depth), (x, 0.5), (x - width, 0.5)][: 4 if k > 1 else 2]
    return np.array(top, np.float32)


def _spiral(turns=1.6, n=40, w=0.35):
    t = np.linspace(0.2, turns * 2 * math.pi, n)
    outer = np.stack([(1 + t) * np.cos(t), (1 + t) * np.sin(t)], 1)
    inner = np.stack([(1 + t - w * 4) * np.cos(t), (1 + t - w * 4) * np.sin(t)], 1)[::-1]
    return np.concatenate([outer, inner]).astype(np.float32)


def _cases():
    rng = np.random.default_rng(7)
    cases = [_star(rng, int(n)) for n in rng.integers(5, 40, 150)]
    cases += [_comb(k) for k in (2, 3, 5, 9)]
    cases.append(_spiral())
    cases.append(_spiral(turns=2.4, n=60, w=0.2))
    t = np.arange(23) * 2 * math.pi / 23
    cases.append(np.stack([np.cos(t), np.sin(t)], 1))                               # convex, 23 vertices: fans
    t = np.arange(60) * 2 * math.pi / 60
    cases.append(np.stack([3 * np.cos(t), np.sin(t)], 1))                           # convex, 60 vertices
    cases.append(np.array([(0, 0), (4, 0), (4, 3), (2, 1), (0, 3)], np.float32))    # one notch
    cases.append(np.array([(0, 0), (2, 2), (0, 2), (2, 0)], np.float32))            # bow tie: refused
    cases.append(np.array([(0, 0), (1, 0), (2, 0)], np.float32))                    # collinear: refused
    cases.append(np.array([(0, 0), (3, 0), (3, 3), (0, 3), (0, 3), (1.5, 1.5)], np.float32))   # duplicate vertex
    return cases


@pytest.mark.skipif(not refapi.available(), reason="the compiled reference (oracle/_ref) is not present")
def test_decomposition_matches_the_reference():
    split = refused = 0
    for i, xy in enumerate(_cases()):
        theirs, ours = refapi.decompose(xy), _ours(xy)
        assert (theirs is None) == (ours is None), i
        if theirs is None:
            refused += 1
            continue
        assert len(ours) == len(theirs), i
        for a, b in zip(ours, theirs):
            assert a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32)), i
        split += len(theirs) > 1
    assert split > 100 and refused >= 2


def test_pieces_are_convex_and_cover_the_outline():
    rng = np.random.default_rng(11)
    for _ in range(60):
        xy = _star(rng, int(rng.integers(6, 30)))
        pieces = _ours(xy)
        if pieces is None:
            continue
        area = 0.0
        for p in pieces:
            assert 3 <= p.shape[0] <= 16
            d = np.roll(p, -1, 0) - p
            turns = d[:, 0] * np.roll(d, -1, 0)[:, 1] - d[:, 1] * np.roll(d, -1, 0)[:, 0]
            assert (turns > -1e-5).all()
            area += 0.5 * float(np.sum(p[:, 0] * np.roll(p, -1, 0)[:, 1] - np.roll(p, -1, 0)[:, 0] * p[:, 1]))
        x, y = xy[:, 0], xy[:, 1]
        whole = 0.5 * abs(float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)))
        assert abs(area - whole) <= 1e-4 * max(whole, 1.0)


def test_capacity_and_refusals():
    sq = np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32)
    k = ctypes.c_uint32(0)
    f = ctypes.POINTER(ctypes.c_float)
    out = np.zeros(2, np.float32)
    counts = np.zeros(1, np.uint32)
    code = ag2d.lib.ag2d_decompose_polygon(sq.ctypes.data_as(f), 4, out.ctypes.data_as(f), 1,
                                           counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 1,
                                           ctypes.byref(k))
    assert code == ag2d.ERR_CAPACITY and k.value == 1
    assert _ours(sq[:2]) is None
