"""Parity helpers shared by the oracle checks (CPU) and the CUDA parity tests (GPU)."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PHASE_FIXTURES = ("c1_n256_s0_step300.npz", "c2_n2000_s1_step240.npz", "c3_n1500_s0_step0.npz",
                  "c2_n20000_s2_step420.npz")
# Capsules with every other shape (all ten shape pairs): the CUDA path is compared with the reference's own taps;
# the C restatement does not restate the capsule routines, so the CPU oracle checks leave this fixture out.
CAPSULE_FIXTURES = ("capsules_n1500_s0_step300.npz",)
GPU_PHASE_FIXTURES = PHASE_FIXTURES + CAPSULE_FIXTURES

# Solver impulses against the FP64 replay of the same order (the FP32 replay of the same order is bit-exact; this is
# the precision contract), on the active contacts' normal and friction impulses:
#  - at least 1 - IMPULSE_SHARE_OVER of them within IMPULSE_RTOL relative, with an absolute floor IMPULSE_ATOL
#    (1e-4 N s, about a thousandth of the impulse gravity gives a 1 kg body in one 1/60 s step) for impulses near
#    zero, where a relative bound means nothing;
#  - every one within IMPULSE_CEIL_RTOL relative + IMPULSE_CEIL_ATOL.
# Why a share: in a deep pile the block solver's case tests (BodyCollisionSolver.cpp:623-700) can fall either way
# on a rounding difference, and eight Gauss-Seidel sweeps carry that to neighbouring contacts. The reference's own
# FP32 solve in its own order shows it: on the 20,000-body pile 24 of 93,654 impulses miss FP64 by more than 1e-4
# relative (worst 0.0074 N s on 1.73 N s), and a colour-major order does the same (23-26). tests/test_oracle_golden.py
# checks the reference's order against this contract; the GPU tests check the coloured order against it.
IMPULSE_RTOL = 1e-4
IMPULSE_ATOL = 1e-4
IMPULSE_SHARE_OVER = 5e-3
IMPULSE_CEIL_RTOL = 1e-3
IMPULSE_CEIL_ATOL = 1e-2


def impulse_errors(m, imp64):
    """(got, fp64, active) as float64 arrays [n, 4] (jn0, jt0, jn1, jt1) for a manifold record array m."""
    got = np.stack([m["jn"][:, 0], m["jt"][:, 0], m["jn"][:, 1], m["jt"][:, 1]], 1).astype(np.float64)
    cnt = np.asarray(m["count"])
    active = np.stack([cnt > 0, cnt > 0, cnt > 1, cnt > 1], 1)
    return got, np.asarray(imp64, np.float64), active


def impulses_within_contract(m, imp64) -> tuple:
    """(ok, message): the impulse contract above for manifold records m against FP64 impulses imp64 [n, 4]."""
    got, ref, active = impulse_errors(m, imp64)
    err, mag = np.abs(got - ref)[active], np.abs(ref)[active]
    if err.size == 0:
        return True, "no active contacts"
    over = int(np.count_nonzero(err > IMPULSE_RTOL * mag + IMPULSE_ATOL))
    ceil = float(np.max(err / (IMPULSE_CEIL_RTOL * mag + IMPULSE_CEIL_ATOL)))
    ok = over <= IMPULSE_SHARE_OVER * err.size and ceil <= 1.0
    return ok, (f"{over} of {err.size} impulses beyond 1e-4 relative of FP64 (allowed {IMPULSE_SHARE_OVER:.1%}); "
                f"worst at {ceil:.2f} of the ceiling; largest error {err.max():.3g} N s")


def load(name: str) -> dict:
    """A fixture as a dict of arrays; arrays stored once for several names (meta.aliases "name=stored") are
    expanded."""
    with np.load(os.path.join(GOLDEN, name)) as z:
        d = {k: z[k] for k in z.files}
    for entry in d.pop("meta.aliases", np.array([], dtype=str)).tolist():
        dst, src = entry.split("=", 1)
        d[dst] = d[src]
    return d


def bits(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a)
    if a.dtype == np.float32:
        return a.view(np.uint32)
    return a


def mismatches(a, b) -> int:
    """Number of elements whose bit patterns differ (floats compared bit-exactly, -0 != +0)."""
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    return int(np.count_nonzero(bits(a) != bits(b)))


def canonical_pairs(pairs: np.ndarray, dyn_begin: int) -> np.ndarray:
    """Canonical pair set: dynamic-dynamic pairs as (min, max), cross pairs as (dynamic, other), sorted."""
    p = np.asarray(pairs, dtype=np.uint32).reshape(-1, 2)
    both = (p[:, 0] >= dyn_begin) & (p[:, 1] >= dyn_begin)
    c = np.where(both[:, None], np.sort(p, axis=1), p)
    return c[np.lexsort((c[:, 1], c[:, 0]))]


def sort_manifolds(m: np.ndarray) -> np.ndarray:
    return m[np.lexsort((m["b"], m["a"]))]


def active_points(m: np.ndarray, field: str) -> np.ndarray:
    return np.where(m["count"][:, None] > np.arange(2)[None, :], m[field], 0)


def partition_labels(ids: np.ndarray) -> np.ndarray:
    """Relabels a set partition by first occurrence, so two labelings of the same partition compare equal."""
    _, inv = np.unique(np.asarray(ids), return_inverse=True)
    first = {}
    return np.array([first.setdefault(int(v), len(first)) for v in inv], dtype=np.int64)


def query_leaf_test(mnx, mny, mxx, mxy, tree_bits, shape, params, trees):
    """Colliders a shape query finds, restated from the reference's query shapes (CollisionDetection/Broad/
    QueryShapes.h:8-86) in float32 without fused multiply-add: AABB (shape 0, params min_x, min_y, max_x, max_y) -
    strict overlap on both axes (AABBQuery::simdOverlap); circle (shape 1, params x, y, r) - dx = fmax(min_x - x,
    fmax(0, x - max_x)), dy alike, found when dx*dx + dy*dy <= fmax(0, r)^2 (CircleQuery::simdOverlap). tree_bits:
    each collider's tree (1 dynamic, 2 static, 4 sleeping); trees: the selected bits. Returns ascending indices."""
    f32 = np.float32
    mnx, mny, mxx, mxy = (np.asarray(a, f32) for a in (mnx, mny, mxx, mxy))
    sel = (np.asarray(tree_bits) & trees) != 0
    if shape == 0:
        qx0, qy0, qx1, qy1 = (f32(v) for v in params)
        hit = (mnx < qx1) & (mxx > qx0) & (mny < qy1) & (mxy > qy0)
    else:
        x, y, r = (f32(v) for v in params)
        r = np.fmax(f32(0), r)
        rr = f32(r * r)
        dx = np.fmax(mnx - x, np.fmax(f32(0), x - mxx)).astype(f32)
        dy = np.fmax(mny - y, np.fmax(f32(0), y - mxy)).astype(f32)
        hit = (dx * dx + dy * dy).astype(f32) <= rr
    return np.nonzero(sel & hit)[0].astype(np.uint32)
