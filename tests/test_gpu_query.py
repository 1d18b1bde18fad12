"""Spatial queries (BroadPhaseCollisionDetector::queryCollidersInShape with the AABBQuery and CircleQuery shapes of
CollisionDetection/Broad/QueryShapes.h:8-86) through the C ABI, against a float32 restatement of the shapes' leaf
tests over the colliders' AABBs read back from the same world.

The checker below restates the reference's tests with numpy float32 (no fused multiply-add, as the reference is
built): AABB - strict overlap on both axes; circle - dx = fmax(min_x - x, fmax(0, x - max_x)) (and dy alike),
found when dx*dx + dy*dy <= fmax(0, r)^2. A collider belongs to the dynamic, static or sleeping tree by its body's
state. Found sets must be equal, index for index.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402


def _expected(w, shape, params, trees):
    f32 = np.float32
    mnx, mny = w.read(ag2d.COL_AABB_MIN_X), w.read(ag2d.COL_AABB_MIN_Y)
    mxx, mxy = w.read(ag2d.COL_AABB_MAX_X), w.read(ag2d.COL_AABB_MAX_Y)
    state = w.read(ag2d.BODY_STATE)   # one collider per body, in body order, in these scenes
    assert state.size == mnx.size
    bit = np.where(state == 2, 1, np.where(state == 0, 2, 4))
    sel = (bit & trees) != 0
    if shape == ag2d.QUERY_AABB:
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


@pytest.fixture(scope="module")
def world():
    w = ag2d.World.from_scene(scenes.make_c1(600, seed=5, width=60.0, height=40.0))
    assert w.query_aabb((-1e6, -1e6), (1e6, 1e6)).size == 0   # before the first step: nothing
    w.step(240)   # settled enough that some bodies sleep: all three trees are populated
    states = w.read(ag2d.BODY_STATE)
    assert (states == 0).any() and (states == 2).any()
    return w


def test_queries_match_the_restated_leaf_tests(world):
    rng = np.random.default_rng(3)
    checked = found = 0
    for _ in range(40):
        cx, cy = rng.uniform(-35, 35), rng.uniform(-5, 30)
        hw, hh = rng.uniform(0.1, 15), rng.uniform(0.1, 15)
        r = rng.uniform(-1, 12)
        for trees in (ag2d.TREE_ALL, ag2d.TREE_DYNAMIC, ag2d.TREE_STATIC, ag2d.TREE_SLEEPING,
                      ag2d.TREE_DYNAMIC | ag2d.TREE_SLEEPING):
            got = world.query_aabb((cx - hw, cy - hh), (cx + hw, cy + hh), trees)
            want = _expected(world, ag2d.QUERY_AABB, (cx - hw, cy - hh, cx + hw, cy + hh), trees)
            assert np.array_equal(got, want), ("aabb", trees)
            got = world.query_circle((cx, cy), r, trees)
            want = _expected(world, ag2d.QUERY_CIRCLE, (cx, cy, r), trees)
            assert np.array_equal(got, want), ("circle", trees, r)
            checked += 2
            found += got.size
    assert checked == 400 and found > 0


def test_query_capacity_and_counts(world):
    everything = world.query_aabb((-1e6, -1e6), (1e6, 1e6))
    assert everything.size == world.read(ag2d.BODY_STATE).size
    assert world.query_circle((0.0, 0.0), -3.0).size <= everything.size   # a negative radius is clamped at 0
    with pytest.raises(ag2d.Ag2dError):
        world._query(7, [0, 0, 1, 1], ag2d.TREE_ALL)
