"""The request server against the same worlds stepped alone, through the C ABI.

Requests join and leave the resident batch between rounds (a device-side repack of the world-segmented arrays).
Each request's world keeps its own Morton bounds, trees, manifold order and colouring whatever else is resident, so
its final body state equals the alone run's bit for bit: with other requests admitted before, after and beside it,
with a memory budget that admits one request at a time, and with continuous collision detection on.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402

FIELDS = [ag2d.BODY_COM_X, ag2d.BODY_COM_Y, ag2d.BODY_ROTATION, ag2d.BODY_VEL_X, ag2d.BODY_VEL_Y,
          ag2d.BODY_ANGULAR_VELOCITY, ag2d.BODY_STATE]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _alone(scene, steps, ccd, pre_steps=0):
    w = ag2d.World.from_scene(scene, ccd=ccd)
    w.step(pre_steps + steps)
    return w


def _assert_same(server, rid, alone, tag):
    for f in FIELDS:
        got, want = server.read(rid, f), alone.read(f)
        assert got.shape == want.shape, (tag, f, got.shape, want.shape)
        bad = np.nonzero(_bits(got) != _bits(want))[0]
        assert bad.size == 0, f"{tag} field {f}: {bad.size} mismatches, first at {bad[:5]}"


def _requests(n, seed, hi=400):
    return scenes.make_c5_requests(n, seed=seed, lo=8, hi=hi)


@pytest.mark.parametrize("ccd", [False, True])
def test_server_mix_equals_alone(ccd):
    sc = _requests(9, seed=11)
    steps = [7, 30, 19, 45, 3, 30, 12, 26, 40]
    server = ag2d.Server(memory_budget_bytes=1 << 30, steps_per_round=8, ccd=ccd)
    ids = []
    # Staggered arrivals: some requests join a batch that has already stepped, others leave before they arrive.
    for k, s in enumerate(sc):
        ids.append(server.submit(ag2d.World.from_scene(s, ccd=ccd), steps[k]))
        if k % 3 == 2:
            time.sleep(0.05)
    server.wait_all(120_000)
    st = server.stats()
    assert st["completed"] == len(sc) and st["waiting"] == 0 and st["resident"] == 0
    assert st["body_steps"] == sum(s.n * n for s, n in zip(sc, steps))
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["peak_resident"] > 1
    for k, s in enumerate(sc):
        state, lat = server.poll(ids[k])
        assert state == ag2d.REQUEST_DONE and lat > 0
        _assert_same(server, ids[k], _alone(s, steps[k], ccd), f"request {k}")
    server.close()


def test_server_budget_admits_one_at_a_time():
    sc = _requests(4, seed=12, hi=200)
    steps = [10, 5, 17, 9]
    server = ag2d.Server(memory_budget_bytes=1, steps_per_round=4, ccd=True)
    worlds = [ag2d.World.from_scene(s, ccd=True) for s in sc]
    ids = [server.submit(w, n) for w, n in zip(worlds, steps)]
    # With the budget below every request, the queue is served in order, one resident world at a time.
    server.wait_all(120_000)
    st = server.stats()
    assert st["peak_resident"] == 1
    assert st["rounds"] == sum((n + 3) // 4 for n in steps)
    for k, s in enumerate(sc):
        _assert_same(server, ids[k], _alone(s, steps[k], True), f"request {k}")
        server.release(ids[k])
    with pytest.raises(ag2d.Ag2dError):
        server.read(ids[0], ag2d.BODY_COM_X)
    server.close()


def test_server_request_from_stepped_world():
    # A world that already stepped joins with its state, warm-start manifolds and collider poses (the sweep start of
    # continuous collision detection), and continues as it would alone.
    sc = _requests(3, seed=13, hi=300)
    server = ag2d.Server(memory_budget_bytes=1 << 30, steps_per_round=16, ccd=True)
    ids = []
    for k, s in enumerate(sc):
        w = ag2d.World.from_scene(s, ccd=True)
        w.step(5 + k)
        ids.append(server.submit(w, 20))
    server.wait_all(120_000)
    for k, s in enumerate(sc):
        _assert_same(server, ids[k], _alone(s, 20, True, pre_steps=5 + k), f"request {k}")
    server.close()


def test_server_rejects_mismatched_settings():
    server = ag2d.Server(memory_budget_bytes=1 << 30, ccd=True)
    w = ag2d.World.from_scene(_requests(1, seed=14, hi=50)[0], ccd=False)
    with pytest.raises(ag2d.Ag2dError):
        server.submit(w, 5)
    server.wait_all(10_000)
    server.close()
