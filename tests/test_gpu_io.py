"""Host transfers through the C ABI: packed reads, asynchronous reads and batch checkpoints.

- ag2d_world_read / ag2d_batch_read pack a field on the device and copy only its bytes; the values must equal the
  same field assembled from the full records (bit for bit), into pageable and page-locked destinations alike.
- ag2d_world_read_async returns the values as they stood when the read was queued, although the steps queued after
  it overwrite the arrays; several reads in flight (more than the ring of staging slots) stay ordered.
- ag2d_batch_save / ag2d_batch_restore: a restored batch steps on bit for bit as the saved one, for every world,
  including the warm-start manifolds, sleep state and colours carried across steps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402

BODY_FIELDS = [ag2d.BODY_COM_X, ag2d.BODY_COM_Y, ag2d.BODY_VEL_X, ag2d.BODY_VEL_Y, ag2d.BODY_ROTATION,
               ag2d.BODY_ANGULAR_VELOCITY, ag2d.BODY_ROT_COS, ag2d.BODY_ROT_SIN, ag2d.BODY_WRAP_COUNT,
               ag2d.BODY_SLEEP_TIMER, ag2d.BODY_STATE, ag2d.BODY_SLEEP_ISLAND, ag2d.BODY_INV_MASS,
               ag2d.BODY_INV_INERTIA, ag2d.BODY_POSE]
COL_FIELDS = [ag2d.COL_WORLD_X, ag2d.COL_WORLD_Y, ag2d.COL_WORLD_COS, ag2d.COL_WORLD_SIN,
              ag2d.COL_WORLD_ROTATION, ag2d.COL_AABB_MIN_X, ag2d.COL_AABB_MIN_Y, ag2d.COL_AABB_MAX_X,
              ag2d.COL_AABB_MAX_Y]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _worlds(n=12, seed=21):
    return [ag2d.World.from_scene(s) for s in scenes.make_c4_worlds(worlds=n, seed=seed, lo=16, hi=700)]


def test_packed_read_matches_components():
    w = ag2d.World.from_scene(scenes.make_c1(700, seed=4))
    w.step(90)
    x, y, r = w.read(ag2d.BODY_COM_X), w.read(ag2d.BODY_COM_Y), w.read(ag2d.BODY_ROTATION)
    pose = w.read(ag2d.BODY_POSE).reshape(-1, 3)
    assert np.array_equal(_bits(pose[:, 0]), _bits(x))
    assert np.array_equal(_bits(pose[:, 1]), _bits(y))
    assert np.array_equal(_bits(pose[:, 2]), _bits(r))
    # Page-locked and pageable destinations give the same bytes; a larger destination is filled at its front.
    for f in BODY_FIELDS + COL_FIELDS:
        plain = w.read(f)
        pinned = ag2d.host_empty(plain.nbytes + 64)
        got = w.read(f, out=pinned)
        assert np.array_equal(got.view(np.uint8), plain.view(np.uint8)), f


def test_large_pageable_read_crosses_chunks():
    # 12 bytes x 800k bodies is above the 8 MiB bounce chunks: the chunked copy must reassemble in order.
    sc = scenes.make_c3(800_000, 0, extent=4000.0 * 0.8 ** 0.5)
    w = ag2d.World.from_scene(sc)
    w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    pose = w.read(ag2d.BODY_POSE).reshape(-1, 3)
    assert pose.shape[0] == sc.n
    assert np.array_equal(_bits(pose[:, 0]), _bits(w.read(ag2d.BODY_COM_X)))
    assert np.array_equal(_bits(pose[:, 1]), _bits(w.read(ag2d.BODY_COM_Y)))
    circles = np.asarray(sc.kind) == scenes.CIRCLE   # a circle's centre of mass is its scene position
    assert np.array_equal(_bits(pose[circles, 0]), _bits(np.asarray(sc.px, np.float32)[circles]))


def test_async_reads_hold_the_state_they_were_queued_at():
    w = ag2d.World.from_scene(scenes.make_c1(900, seed=8))
    w.step(30)
    expected, bufs, views = [], [], []
    for k in range(6):   # more reads than staging slots: the ring wraps while copies are in flight
        expected.append(w.read(ag2d.BODY_POSE).copy())
        buf = ag2d.host_empty(w.field_bytes(ag2d.BODY_POSE))
        views.append(w.read_async(ag2d.BODY_POSE, buf))
        bufs.append(buf)
        w.step(2)
    w.read_wait()
    for k in range(6):
        assert np.array_equal(views[k].view(np.uint8), expected[k].view(np.uint8)), k
    with pytest.raises(ag2d.Ag2dError):
        w.read_async(ag2d.BODY_POSE, np.empty(w.field_bytes(ag2d.BODY_POSE), np.uint8))   # pageable: refused
    with pytest.raises(ag2d.Ag2dError):
        w.read_async(ag2d.PAIRS, ag2d.host_empty(1 << 20))   # phase taps are read synchronously only


def test_batch_read_of_one_world_matches_slices_of_the_engine():
    batch = ag2d.Batch(_worlds())
    batch.step(80)
    e = batch.engine
    starts_b = np.cumsum([0] + [batch.read(k, ag2d.BODY_COM_X).size for k in range(batch.n_worlds)])
    starts_c = np.cumsum([0] + [batch.read(k, ag2d.COL_WORLD_X).size for k in range(batch.n_worlds)])
    for f in BODY_FIELDS + COL_FIELDS:
        full = e.read(f)
        per = 3 if f == ag2d.BODY_POSE else 1
        st = starts_c if f in COL_FIELDS else starts_b
        for k in (0, 5, batch.n_worlds - 1):
            got = batch.read(k, f)
            want = full[per * st[k]:per * st[k + 1]].copy()
            if f == ag2d.BODY_SLEEP_ISLAND:
                want = np.where(want == 0xFFFFFFFF, want, want - st[k]).astype(np.uint32)
            assert np.array_equal(_bits(got), _bits(want)), (f, k)


@pytest.mark.parametrize("pinned", [True, False])
def test_checkpoint_restore_steps_on_bit_exact(pinned):
    batch = ag2d.Batch(_worlds(seed=33))
    batch.step(140)   # settled enough that some bodies sleep and colours carry over
    blob = batch.save() if pinned else batch.save(out=np.empty(batch.save().nbytes, np.uint8))
    restored = ag2d.Batch.restore(blob)
    assert restored.n_worlds == batch.n_worlds
    # Right after restoring, every field equals the saved batch's.
    for k in range(batch.n_worlds):
        for f in BODY_FIELDS + COL_FIELDS:
            assert np.array_equal(_bits(restored.read(k, f)), _bits(batch.read(k, f))), (k, f)
    batch.step(60)
    restored.step(60)
    for k in range(batch.n_worlds):
        for f in BODY_FIELDS + COL_FIELDS:
            assert np.array_equal(_bits(restored.read(k, f)), _bits(batch.read(k, f))), (k, f)
        mg, mw = restored.read(k, ag2d.PREV_MANIFOLDS), batch.read(k, ag2d.PREV_MANIFOLDS)
        assert np.array_equal(mg.view(np.uint8), mw.view(np.uint8)), k
    assert restored.counters()["status"] == 0
    # A damaged blob is refused, not trusted.
    bad = np.array(blob, copy=True)
    bad[:8] = 0
    with pytest.raises(ag2d.Ag2dError):
        ag2d.Batch.restore(bad)
    with pytest.raises(ag2d.Ag2dError):
        ag2d.Batch.restore(blob[:blob.nbytes // 2])


def test_checkpoint_loaded_into_a_running_batch_steps_on_bit_exact():
    """ag2d_batch_load: a batch that has run on loads another state of the same worlds and steps on exactly as the
    batch the checkpoint came from, without allocating device memory when its buffers are large enough."""
    batch = ag2d.Batch(_worlds(seed=34))
    batch.step(150)
    blob = batch.save()
    other = ag2d.Batch.restore(blob)
    other.step(37)                  # a different state, buffers warm
    allocs = ag2d.device_allocs()
    other.load(blob)
    assert ag2d.device_allocs() == allocs
    batch.step(40)
    other.step(40)
    for k in range(batch.n_worlds):
        for f in BODY_FIELDS + COL_FIELDS:
            assert np.array_equal(_bits(other.read(k, f)), _bits(batch.read(k, f))), (k, f)
        mg, mw = other.read(k, ag2d.PREV_MANIFOLDS), batch.read(k, ag2d.PREV_MANIFOLDS)
        assert np.array_equal(mg.view(np.uint8), mw.view(np.uint8)), k
    assert other.counters()["status"] == 0
