"""Spatial queries (BroadPhaseCollisionDetector::queryCollidersInShape with the AABBQuery and CircleQuery shapes of
CollisionDetection/Broad/QueryShapes.h:8-86) through the C ABI, against the restated leaf tests
(parity.query_leaf_test) over the colliders' AABBs read back from the same world. The restatement is pinned to the
reference's own trees by tests/test_oracle_golden.py::test_query_restatement_matches_the_reference. A collider
belongs to the dynamic, static or sleeping tree by its body's state. Found sets must be equal, index for index.
"""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402


def _expected(w, shape, params, trees):
    state = w.read(ag2d.BODY_STATE)   # one collider per body, in body order, in these scenes
    mnx = w.read(ag2d.COL_AABB_MIN_X)
    assert state.size == mnx.size
    tree_bits = np.where(state == 2, 1, np.where(state == 0, 2, 4))
    return parity.query_leaf_test(mnx, w.read(ag2d.COL_AABB_MIN_Y), w.read(ag2d.COL_AABB_MAX_X),
                                  w.read(ag2d.COL_AABB_MAX_Y), tree_bits, shape, params, trees)


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


@pytest.fixture(scope="module", params=["contacts_c2_n1500_step300.npz", "contacts_capsules_n1500_step300.npz"])
def loaded(request):
    """A world holding the reference's own state of a mixed-shape pile (circles, boxes, polygons in a U container;
    in the second fixture capsules too, 1,500 bodies after 300 steps), collider poses and AABBs included, with the
    reference's query answers."""
    g = parity.load(request.param)
    w = ag2d.World()
    w.load_state(g, "q.", g["meta.materials"], with_poses=True)
    return w, g


def test_shape_queries_match_the_reference(loaded):
    w, g = loaded
    for k in range(g["s.shape"].size):
        shape, trees = int(g["s.shape"][k]), int(g["s.trees"][k])
        params = g["s.params"][k][:4] if shape == 0 else g["s.params"][k][:3]
        want = g["s.idx"][g["s.offsets"][k]:g["s.offsets"][k + 1]]
        assert np.array_equal(w._query(shape, params, trees), want), (k, shape, trees)


def test_circle_contacts_match_the_reference(loaded):
    """Same colliders as NarrowPhaseCollisionDetector::findCollisionsInCircle over the reference's circle query;
    signed distances within 1e-5 relative (the narrow-phase bar for depths)."""
    w, g = loaded
    total = 0
    for k in range(g["c.trees"].size):
        x, y, r = (float(v) for v in g["c.params"][k])
        idx, dist = w.query_circle_contacts((x, y), r, int(g["c.trees"][k]))
        lo, hi = g["c.offsets"][k], g["c.offsets"][k + 1]
        assert np.array_equal(idx, g["c.idx"][lo:hi]), k
        want = g["c.sdf"][lo:hi]
        assert np.allclose(dist, want, rtol=1e-5, atol=1e-6), (k, np.abs(dist - want).max())
        total += idx.size
    assert total > 1000
