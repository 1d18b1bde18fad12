"""Collision events through the C ABI (Simulation::createCollisionCallback / destroyCollisionCallback /
setColliderCollisionCallback, Simulation.cpp:130-171; recorded in BodyCollisionSolver::computeConstraintData,
Solving/BodyCollisionSolver.cpp:320-387; dispatched at the end of the step, Simulation.cpp:174-180, 450).

- Full steps against the reference's own events (tests/golden/events_c2_n1200.npz): a world loaded with the
  reference's state before each of four steps of a 1,200-body drop, its colliders opted in as the reference's were
  (two callbacks; thresholds 0, 0.5, 3 and never), steps once. Its events are the reference's as a set (colliders and
  bodies by handle slot, callback id, point, normal and impulse bit for bit), and the callbacks receive exactly the
  recorded events, in order, each from its own id.
- The event kernel against the oracle's restatement on every phase fixture, the 20,000-body pile included (more
  events than the ring's first size, so the ring grows): the same events in the same order, bit for bit.
- The callback table and the switches: ids from 1 with the last destroyed id reused first, a destroyed id's
  colliders cleared, the reference's rejected arguments, events off or without callbacks record nothing, a
  callback cannot step the world, and body handles in the events are the creation handles.
"""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from oracle import oraapi  # noqa: E402

FLOAT_FIELDS = ("point_x", "point_y", "normal_x", "normal_y", "impulse")
REF_FLOAT = ("px", "py", "nx", "ny", "impulse")


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _from_oracle(m):
    out = np.zeros(m.shape[0], ag2d.MANIFOLD_DTYPE)
    for f in ("a", "b", "nx", "ny", "depth", "count"):
        out[f] = m[f]
    for f, k in (("px", 0), ("px", 1), ("py", 0), ("py", 1), ("id", 0), ("id", 1), ("jn", 0), ("jn", 1), ("jt", 0),
                 ("jt", 1)):
        out[f"{f}{k}"] = m[f][:, k]
    return out


def _loaded_world(d, prefix):
    it, g = d["meta.iters"], d["meta.gravity"]
    w = ag2d.World(dt=float(d["meta.dt"][0]), velocity_iterations=int(it[0]), position_iterations=int(it[1]),
                   gravity=(float(g[0]), float(g[1])), sleep_time=float(d["meta.sleep_time"][0]))
    w.load_state(d, prefix, [tuple(r) for r in d["meta.materials"]])
    return w


def test_events_of_full_steps_match_the_reference():
    d = parity.load("events_c2_n1200.npz")
    total = 0
    for k in d["meta.steps"].tolist():
        p = f"s{k}."
        w = _loaded_world(d, p)
        calls = []
        ids = [w.create_collision_callback(lambda e, i=i: calls.append((i, e.self, e.other, e.impulse)))
               for i in (1, 2)]
        assert ids == [1, 2]
        cb, thr = d[p + "col.callbackId"], d[p + "col.eventThreshold"]
        for c in np.nonzero(cb)[0].tolist():
            w.set_collider_collision_callback(c, int(cb[c]), float(thr[c]))
        w.step(1)
        ev = w.collision_events()
        assert w.counters()["events"] == ev.size
        slot, bslot = d[p + "col.handleSlot"], d[p + "body.handleSlot"]
        ours = sorted(zip(slot[ev["self"]].tolist(), slot[ev["other"]].tolist(), bslot[ev["self_body"]].tolist(),
                          bslot[ev["other_body"]].tolist(), ev["callback_id"].astype(np.uint32).tolist(),
                          *(_bits(ev[f]).tolist() for f in FLOAT_FIELDS)))
        want = sorted(zip(*(d[f"e{k}.ev.{f}"].tolist() for f in ("self", "other", "selfBody", "otherBody",
                                                                  "callback")),
                          *(_bits(d[f"e{k}.ev.{f}"]).tolist() for f in REF_FLOAT)))
        assert ours == want, k
        # Dispatch: every recorded event once, in the recorded order, to the callback of its id.
        assert [(c[0], c[1], c[2]) for c in calls] == list(zip(ev["callback_id"].tolist(), ev["self"].tolist(),
                                                               ev["other"].tolist()))
        assert _bits([c[3] for c in calls]).tolist() == _bits(ev["impulse"]).tolist()
        # Events come in manifold order with side a first: the two sides of one manifold are adjacent.
        pairs = list(zip(ev["self"].tolist(), ev["other"].tolist()))
        for i, (a, b) in enumerate(pairs):
            if (b, a) in pairs:
                j = pairs.index((b, a))
                assert abs(i - j) == 1
        total += ev.size
        assert w.counters()["status"] == 0
        w.close()
    assert total > 300


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES)
def test_event_kernel_matches_the_oracle(name):
    d = parity.load(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    mats = [tuple(r) for r in d["meta.materials"]]
    it, g = d["meta.iters"], d["meta.gravity"]
    w = ag2d.World(dt=float(d["meta.dt"][0]), velocity_iterations=int(it[0]), position_iterations=int(it[1]),
                   gravity=(float(g[0]), float(g[1])))
    w.load_state(d, "svin.", mats)
    m_in = oraapi.manifolds_from_dump(d, "svin.man.")
    w.write(ag2d.MANIFOLDS, _from_oracle(m_in))
    n = d["svin.col.bodyIndex"].size
    ids = [w.create_collision_callback(lambda e: None) for _ in range(2)]
    # Opt-ins by collider index: id 1 at 0, id 2 at 0.05, none, id 1 at 1.
    pattern = [(ids[0], 0.0), (ids[1], 0.05), None, (ids[0], 1.0)]
    cb = np.zeros(n, np.uint32)
    thr = np.full(n, ag2d.NO_COLLISION_EVENT_THRESHOLD, np.float32)
    for c in range(n):
        p = pattern[c % len(pattern)]
        if p is not None:
            cb[c], thr[c] = p
            w.set_collider_collision_callback(c, *p)
    w.run_phase(ag2d.PHASE_EVENTS)
    ev = w.collision_events()
    ref = oraapi.OraWorld(d, "svin.", mats).collision_events(m_in, cb, thr)
    assert ev.size == ref.size and ref.size > 0
    for ours, theirs in (("self", "self"), ("other", "other"), ("self_body", "selfBody"),
                         ("other_body", "otherBody")):
        assert np.array_equal(ev[ours], ref[theirs]), ours
    assert np.array_equal(ev["callback_id"].astype(np.uint32), ref["callback"])
    for ours, theirs in zip(FLOAT_FIELDS, REF_FLOAT):
        assert parity.mismatches(ev[ours], ref[theirs]) == 0, ours
    if m_in.size > 10_000:
        assert ev.size > 1024   # beyond the ring's first size: the ring grew and the pass ran again


def _ball_on_ground(w, height=3.0, vy=-6.0):
    """A ball dropped onto a static ground box without restitution: after its impact it rests on the ground, and
    gravity gives the resting contact a positive impact impulse every step."""
    mat = w.add_material(0.0, 0.5, 0.4)
    ground = w.add_box(40.0, 2.0, 0.0, -1.0, mass=0.0, material=mat)
    ball = w.add_circle(0.5, 0.0, height, vy=vy, mass=1.0, material=mat)
    return ground, ball


def test_callback_table_and_switches():
    w = ag2d.World(dt=1.0 / 60.0)
    ground, ball = _ball_on_ground(w)
    got = []
    a = w.create_collision_callback(lambda e: got.append(("a", e.self, e.self_body_handle, e.other_body_handle)))
    b = w.create_collision_callback(lambda e: got.append(("b", e.self, e.self_body_handle, e.other_body_handle)))
    assert (a, b) == (1, 2)
    w.destroy_collision_callback(a)
    a2 = w.create_collision_callback(lambda e: got.append(("a2", e.self, e.self_body_handle, e.other_body_handle)))
    assert a2 == 1   # the last destroyed id is reused first
    with pytest.raises(ag2d.Ag2dError):
        w.destroy_collision_callback(0)
    with pytest.raises(ag2d.Ag2dError):
        w.destroy_collision_callback(7)
    with pytest.raises(ag2d.Ag2dError):
        w.set_collider_collision_callback(2, a2, 0.0)          # collider out of range
    with pytest.raises(ag2d.Ag2dError):
        w.set_collider_collision_callback(1, a2, -1.0)         # negative threshold
    with pytest.raises(ag2d.Ag2dError):
        w.set_collider_collision_callback(1, a2, float("nan"))
    with pytest.raises(ag2d.Ag2dError):
        w.set_collider_collision_callback(1, 9, 0.0)           # dead id
    ball_col = 1 if w.read(ag2d.COL_BODY)[1] == w.body_index(ball) else 0
    ground_col = 1 - ball_col
    w.set_collider_collision_callback(ball_col, a2, 0.0)
    w.set_collider_collision_callback(ground_col, b, 0.0)
    steps = 0
    while not got and steps < 120:
        w.step(1)
        steps += 1
    assert got, "the ball never touched the ground"
    # The impact step: one event per side, each to its collider's callback, with the creation handles.
    assert sorted(g[0] for g in got) == ["a2", "b"]
    for tag, col, self_h, other_h in got:
        if tag == "a2":
            assert (col, self_h, other_h) == (ball_col, ball, ground)
        else:
            assert (col, self_h, other_h) == (ground_col, ground, ball)
    ev = w.collision_events()
    assert ev.size == 2 and ev["impulse"][0] > 0 and ev["impulse"][0] == ev["impulse"][1]
    assert np.allclose(ev["normal_x"][0], -ev["normal_x"][1]) and np.allclose(ev["normal_y"][0], -ev["normal_y"][1])
    # A threshold above the impulse silences that side.
    w.set_collider_collision_callback(ground_col, b, float(ev["impulse"][0]) * 1e6)
    got.clear()
    w.step(1)
    assert all(g[0] == "a2" for g in got)
    # Events off: nothing recorded or called; back on: recorded again.
    w.set_collision_events(False)
    got.clear()
    w.step(2)
    assert not got and w.collision_events().size == 0 and w.counters()["events"] == 0
    w.set_collision_events(True)
    w.step(1)
    assert got
    # Destroying an id clears its colliders: no callback left, nothing recorded.
    w.destroy_collision_callback(a2)
    w.destroy_collision_callback(b)
    got.clear()
    w.step(2)
    assert not got and w.collision_events().size == 0
    # A new id is not attached to any collider.
    c = w.create_collision_callback(lambda e: got.append(e.self))
    w.step(1)
    assert not got
    w.set_collider_collision_callback(ball_col, c, 0.0)
    w.step(1)
    assert got == [ball_col]
    assert w.counters()["status"] == 0


def test_a_callback_cannot_step_the_world():
    w = ag2d.World(dt=1.0 / 60.0)
    _, ball = _ball_on_ground(w, height=0.6, vy=-2.0)
    codes = []

    def fn(e):
        codes.append(int(ag2d.lib.ag2d_world_step(w.h, 1)))
        w.set_body_velocity(ball, 0.0, 5.0)   # a queued command is fine: applied at the next step

    cid = w.create_collision_callback(fn)
    col = int(np.nonzero(w.read(ag2d.COL_BODY) == w.body_index(ball))[0][0])
    w.set_collider_collision_callback(col, cid, 0.0)
    for _ in range(30):
        w.step(1)
        if codes:
            break
    assert codes and all(c != 0 for c in codes)
    steps = w.counters()["steps"]
    w.step(1)   # the queued velocity applies
    assert w.read(ag2d.BODY_VEL_Y)[w.body_index(ball)] > 4.0
    assert w.counters()["steps"] == steps + 1
