"""Edge cases of the batch and the request server, and batching invariance at the full c4 size.

- Degenerate worlds in a batch: a ground box alone, a single body, no ground at all (free fall), next to ordinary
  worlds; each comes out bit-identical to the same world stepped alone.
- Server requests with zero steps (the state comes back unchanged), worlds without dynamic bodies, and a server
  reused after it drained.
- The full c4 workload (4,096 worlds, 1.69 M bodies) as one batch: a stratified sample of worlds is bit-identical
  to the same worlds stepped alone, so the size-independent property that the parity tests check at small sizes
  holds at the measured size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402

FIELDS = [ag2d.BODY_COM_X, ag2d.BODY_COM_Y, ag2d.BODY_ROTATION, ag2d.BODY_VEL_X, ag2d.BODY_VEL_Y,
          ag2d.BODY_ANGULAR_VELOCITY, ag2d.BODY_STATE]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _free_fall_world(n=5):
    w = ag2d.World()
    for k in range(n):
        w.add_circle(0.5, float(k) * 1.5, 10.0 + k, vx=0.3 * k)
    return w


def _degenerate_worlds():
    return [
        ("ground only", lambda: ag2d.World.from_scene(scenes.make_c1(0, seed=1, width=20.0, height=10.0))),
        ("one body", lambda: ag2d.World.from_scene(scenes.make_c1(1, seed=2, width=20.0, height=10.0))),
        ("no ground", lambda: _free_fall_world()),
        ("ordinary", lambda: ag2d.World.from_scene(scenes.make_c1(40, seed=3, width=20.0, height=10.0))),
        ("nine", lambda: ag2d.World.from_scene(scenes.make_c1(9, seed=4, width=20.0, height=10.0))),
    ]


def test_batch_with_degenerate_worlds():
    cases = _degenerate_worlds()
    batch = ag2d.Batch([make() for _, make in cases])
    alone = [make() for _, make in cases]
    batch.step(90)
    for w in alone:
        w.step(90)
    for k, (name, _) in enumerate(cases):
        for f in FIELDS:
            got, want = batch.read(k, f), alone[k].read(f)
            assert got.shape == want.shape, (name, f)
            assert np.array_equal(_bits(got), _bits(want)), (name, f)


def test_server_edge_requests():
    server = ag2d.Server(memory_budget_bytes=1 << 30, steps_per_round=8)
    cases = _degenerate_worlds()
    steps = [0, 13, 20, 0, 7]
    ids = [server.submit(make(), n) for (_, make), n in zip(cases, steps)]
    server.wait_all(120_000)
    for k, ((name, make), n) in enumerate(zip(cases, steps)):
        w = make()
        w.step(n)
        for f in FIELDS:
            got, want = server.read(ids[k], f), w.read(f)
            assert got.shape == want.shape, (name, f)
            assert np.array_equal(_bits(got), _bits(want)), (name, f, n)
    # The drained server takes new requests.
    w = ag2d.World.from_scene(scenes.make_c1(30, seed=9, width=20.0, height=10.0))
    rid = server.submit(w, 25)
    server.wait_all(120_000)
    alone = ag2d.World.from_scene(scenes.make_c1(30, seed=9, width=20.0, height=10.0))
    alone.step(25)
    assert np.array_equal(_bits(server.read(rid, ag2d.BODY_POSE)), _bits(alone.read(ag2d.BODY_POSE)))
    st = server.stats()
    assert st["completed"] == len(cases) + 1 and st["resident"] == 0
    server.close()


def test_full_c4_batch_sample_equals_alone():
    sc = scenes.make_c4_worlds(worlds=4096, seed=0, processes=16)
    worlds = []
    for s in sc:
        w = ag2d.World(dt=s.dt, gravity=s.gravity)
        w.add_scene(s)
        worlds.append(w)
    batch = ag2d.Batch(worlds)
    steps = 60
    batch.step(steps)
    order = np.argsort([s.n for s in sc])
    sample = [int(order[k]) for k in np.linspace(0, len(sc) - 1, 8).astype(int)]   # smallest to largest world
    for k in sample:
        w = ag2d.World.from_scene(sc[k])
        w.step(steps)
        for f in FIELDS:
            assert np.array_equal(_bits(batch.read(k, f)), _bits(w.read(f))), (k, sc[k].n, f)
    assert batch.counters()["status"] == 0
