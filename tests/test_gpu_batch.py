"""Batched worlds against the same worlds stepped alone, through the C ABI.

A batch packs several worlds into one world-segmented engine instance. Each world's Morton bounds, tree, manifold
order, colouring and solving order are those it has when stepped alone, so the comparison is bit-exact: body state,
sleep state and manifolds (with their impulses) of every world equal the alone run's.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402

BODY_FIELDS = [ag2d.BODY_COM_X, ag2d.BODY_COM_Y, ag2d.BODY_VEL_X, ag2d.BODY_VEL_Y, ag2d.BODY_ROTATION,
               ag2d.BODY_ANGULAR_VELOCITY, ag2d.BODY_ROT_COS, ag2d.BODY_ROT_SIN, ag2d.BODY_WRAP_COUNT,
               ag2d.BODY_SLEEP_TIMER, ag2d.BODY_STATE, ag2d.BODY_SLEEP_ISLAND]
COL_FIELDS = [ag2d.COL_WORLD_X, ag2d.COL_WORLD_Y, ag2d.COL_AABB_MIN_X, ag2d.COL_AABB_MAX_Y]


def _scene_list(seed=3):
    out = scenes.make_c4_worlds(worlds=7, seed=seed, lo=16, hi=600)
    out.append(scenes.make_c1(1, seed=seed + 50, width=20.0, height=10.0))    # one body over its ground
    out.append(scenes.make_c1(9, seed=seed + 51, width=20.0, height=10.0))    # a SIMD body of 8 and a tail
    return out


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _assert_world_equal(batch, k, alone):
    for f in BODY_FIELDS + COL_FIELDS:
        got, want = batch.read(k, f), alone.read(f)
        assert got.shape == want.shape, (k, f)
        bad = np.nonzero(_bits(got) != _bits(want))[0]
        assert bad.size == 0, f"world {k} field {f}: {bad.size} mismatches, first at {bad[:5]}"
    mg, mw = batch.read(k, ag2d.PREV_MANIFOLDS), alone.read(ag2d.PREV_MANIFOLDS)
    assert mg.shape == mw.shape, (k, mg.shape, mw.shape)
    assert np.array_equal(mg.view(np.uint8), mw.view(np.uint8)), f"world {k}: manifolds differ"


def test_batch_equals_alone_from_rest():
    sc = _scene_list()
    alone = [ag2d.World.from_scene(s) for s in sc]
    packed = [ag2d.World.from_scene(s) for s in sc]
    batch = ag2d.Batch(packed)
    assert batch.n_worlds == len(sc)
    steps = 240
    for w in alone:
        w.step(steps)
    batch.step(steps)
    for k, w in enumerate(alone):
        _assert_world_equal(batch, k, w)
    c = batch.counters()
    assert c["status"] == 0
    # The scenes settle far enough that some bodies sleep: the sleep path runs in both forms.
    states = np.concatenate([w.read(ag2d.BODY_STATE) for w in alone])
    assert (states == 1).any() or steps < 200


def test_batch_packed_mid_run_keeps_warm_start():
    sc = _scene_list(seed=11)
    alone = [ag2d.World.from_scene(s) for s in sc]
    packed = [ag2d.World.from_scene(s) for s in sc]
    for w in alone + packed:
        w.step(45)
    batch = ag2d.Batch(packed)
    for w in alone:
        w.step(60)
    batch.step(60)
    for k, w in enumerate(alone):
        _assert_world_equal(batch, k, w)
    # The source worlds were copied: they did not advance with the batch.
    for w_src, w_alone in zip(packed, alone):
        assert not np.array_equal(w_src.read(ag2d.BODY_COM_Y), w_alone.read(ag2d.BODY_COM_Y)) or \
            np.all(w_alone.read(ag2d.BODY_STATE) != 2)


def test_batch_pair_counts_add_up():
    sc = _scene_list(seed=5)
    alone = [ag2d.World.from_scene(s) for s in sc]
    batch = ag2d.Batch([ag2d.World.from_scene(s) for s in sc])
    for w in alone:
        w.step(100)
    batch.step(100)
    assert batch.counters()["pairs"] == sum(w.counters()["pairs"] for w in alone)
    assert batch.counters()["manifolds"] == sum(w.counters()["manifolds"] for w in alone)


def test_batch_errors():
    a = ag2d.World.from_scene(scenes.make_c1(8, seed=1, width=20.0, height=10.0))
    b = ag2d.World(dt=1.0 / 120.0)
    with pytest.raises(ag2d.Ag2dError):
        ag2d.Batch([a, b])
    batch = ag2d.Batch([a])
    with pytest.raises(ag2d.Ag2dError):
        batch.read(1, ag2d.BODY_COM_X)
    with pytest.raises(ag2d.Ag2dError):
        batch.read(0, ag2d.PAIRS)


def test_autotune_does_not_change_results():
    """The autotuner times real steps under different launch shapes; the world must come out as if stepped plainly."""
    sc = _scene_list(seed=17)
    tuned = ag2d.Batch([ag2d.World.from_scene(s) for s in sc])
    plain = ag2d.Batch([ag2d.World.from_scene(s) for s in sc])
    t = tuned.engine.autotune(1)
    assert t["team_colliders"] in (128, 256, 512, 1024, 2048) and t["team_threads"] in (64, 128, 256, 512)
    assert t["query_threads"] in (64, 128, 256) and t["narrow_threads"] in (128, 256, 512)
    assert t["team_cons_on_chip"] in (0, 1)
    # One step, then per candidate one untimed and one timed step; the worlds larger than the chosen team size add
    # the four large-team modes. The tuned engine's own step count says how many ran.
    plain.step(int(tuned.counters()["steps"]))
    for k in range(len(sc)):
        for f in BODY_FIELDS:
            assert np.array_equal(_bits(tuned.read(k, f)), _bits(plain.read(k, f))), (k, f)


@pytest.mark.parametrize("on_chip,colliders,threads", [(0, 1024, 128), (1, 128, 64), (1, 512, 256), (1, 2048, 512)])
def test_set_tuning_does_not_change_results(on_chip, colliders, threads):
    """Team solver with its constraint records in global or shared memory (and teams too large for the shared-memory
    records, which fall back to global memory): the same results as the default launch shapes."""
    sc = _scene_list(seed=23)
    tuned = ag2d.Batch([ag2d.World.from_scene(s) for s in sc])
    plain = ag2d.Batch([ag2d.World.from_scene(s) for s in sc])
    tuned.engine.set_tuning({"team_colliders": colliders, "team_threads": threads, "query_threads": 64,
                             "narrow_threads": 512, "team_cons_on_chip": on_chip})
    tuned.step(150)
    plain.step(150)
    for k in range(len(sc)):
        _assert_world_equal(tuned, k, _Alone(plain, k))


class _Alone:
    """A world of a batch read through the single-world interface (for _assert_world_equal)."""

    def __init__(self, batch, k):
        self.batch, self.k = batch, k

    def read(self, field):
        return self.batch.read(self.k, field)
