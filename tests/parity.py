"""Parity helpers shared by the oracle checks (CPU) and the CUDA parity tests (GPU)."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PHASE_FIXTURES = ("c1_n256_s0_step300.npz", "c2_n2000_s1_step240.npz", "c3_n1500_s0_step0.npz")


def load(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


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
