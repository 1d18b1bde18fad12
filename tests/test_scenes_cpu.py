"""The seeded workload generators the bench and the tests share (CPU only).

c4 worlds and c5 requests built in a spawned process pool equal the ones built in order; the c5 request stream is
the sequence make_c5_request draws; the bench's Poisson arrival times are increasing with the stated mean gap.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "physicssimulation-agony_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from ag2d import scenes  # noqa: E402

FIELDS = ("kind", "px", "py", "rot", "vx", "vy", "w", "mass", "radius", "width", "height", "poly_xy")


def _same(a, b):
    assert a.n == b.n and a.name == b.name
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_pool_builds_the_same_worlds():
    serial = scenes.make_c4_worlds(worlds=6, seed=7, lo=16, hi=200, processes=1)
    pooled = scenes.make_c4_worlds(worlds=6, seed=7, lo=16, hi=200, processes=2)
    for a, b in zip(serial, pooled):
        _same(a, b)
    req_serial = scenes.make_c5_requests(5, seed=3, lo=8, hi=300, processes=1)
    req_pooled = scenes.make_c5_requests(5, seed=3, lo=8, hi=300, processes=2)
    for a, b in zip(req_serial, req_pooled):
        _same(a, b)


def test_request_stream_is_the_sequential_draw():
    rng = np.random.default_rng(11)
    one_by_one = [scenes.make_c5_request(rng, k, lo=8, hi=300) for k in range(4)]
    for a, b in zip(one_by_one, scenes.make_c5_requests(4, seed=11, lo=8, hi=300)):
        _same(a, b)
    # 5 % of the bodies (never the ground) are small fast circles.
    big = scenes.make_c5_requests(1, seed=5, lo=2000, hi=2000)[0]
    fast = (big.kind == scenes.CIRCLE) & (np.hypot(big.vx, big.vy) > 100)
    assert not fast[0] and 0.02 < fast.mean() < 0.08


def test_poisson_arrivals():
    import bench
    t = bench.poisson_arrivals(20000, 2000.0, 0)
    assert np.all(np.diff(t) > 0)
    assert abs(np.diff(t).mean() - 1.0 / 2000.0) < 0.05 / 2000.0
    assert np.array_equal(t, bench.poisson_arrivals(20000, 2000.0, 0))
