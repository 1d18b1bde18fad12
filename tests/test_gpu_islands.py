"""Manifolds of sleeping islands kept on the device (the reference's islandManifolds: NarrowPhaseCollisionDetector::
sleepContactData / wakeContactData, CollisionDetection/Narrow/NarrowPhaseCollisionDetector.cpp:299-414), against the
reference's own taps of a scene of 40 three-box towers (tests/golden/towers_s0_step*.npz, from the compiled
reference).

- Wake (step 141: four towers woken by falling circles): loaded with the reference's state, warm-start list and
  store, the narrow phase and the wake pass give exactly the reference's solver input: the fresh manifolds plus the
  12 stored records of the woken islands, bit for bit (geometry, ids, impulses), matched by collider handle slots
  (the reference moves woken bodies between its dense groups; here they keep their index).
- Sleep (step 34: 36 towers fall asleep): one full step from the reference's state moves the manifolds of the bodies
  now asleep into the store. The same records (by slots), the same island partition, geometry and ids bit for bit,
  impulses within the solver contract (the solving order differs); the warm-start list keeps the rest.
- Batches: a batch of tower worlds with staggered drops (islands sleeping and waking in different steps, records
  merged into the world-grouped list) steps bit for bit as each world alone, store included, and a checkpoint
  carries the store.
"""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402
from oracle import oraapi  # noqa: E402


def _from_oracle(m):
    out = np.zeros(m.shape[0], ag2d.MANIFOLD_DTYPE)
    for f in ("a", "b", "nx", "ny", "depth", "count"):
        out[f] = m[f]
    out["px0"], out["px1"] = m["px"][:, 0], m["px"][:, 1]
    out["py0"], out["py1"] = m["py"][:, 0], m["py"][:, 1]
    out["id0"], out["id1"] = m["id"][:, 0], m["id"][:, 1]
    out["jn0"], out["jn1"] = m["jn"][:, 0], m["jn"][:, 1]
    out["jt0"], out["jt1"] = m["jt"][:, 0], m["jt"][:, 1]
    return out


def _world(d, body_prefix=None):
    it, g = d["meta.iters"], d["meta.gravity"]
    w = ag2d.World(dt=float(d["meta.dt"][0]), velocity_iterations=int(it[0]), position_iterations=int(it[1]),
                   gravity=(float(g[0]), float(g[1])))
    w.load_state(d, "pre.", [tuple(r) for r in d["meta.materials"]], body_prefix)
    return w


def _load_store(w, d, prefix="pre."):
    """The reference's store, its island ids (FIRST_SLEEP_ISLAND_ID-based) turned into this library's island roots:
    the smallest dense index of a sleeping body of the island, as the state loader numbers them."""
    w.write(ag2d.PREV_MANIFOLDS, _from_oracle(oraapi.manifolds_from_dump(d, prefix + "man.")))
    store = oraapi.manifolds_from_dump(d, prefix + "isle.")
    starts = d[prefix + "body.groupStarts"]
    sleep_id = d[prefix + "body.sleepIslandId"]
    root = {}
    for i in range(int(starts[1]), int(starts[2])):
        root.setdefault(int(sleep_id[i]), i)
    ids = np.array([root[int(x)] for x in d[prefix + "isle.islandId"]], np.uint32)
    w.write(ag2d.ISLAND_MANIFOLDS, _from_oracle(store))
    w.write(ag2d.ISLAND_IDS, ids)
    return ids


def _by_slots(m, slot):
    """{(slot of a, slot of b): record} for our records (dense collider indices mapped through 'slot')."""
    return {(int(slot[r["a"]]), int(slot[r["b"]])): r for r in m}


def _ref_by_slots(d, prefix):
    m = oraapi.manifolds_from_dump(d, prefix)
    return {(int(a), int(b)): r for a, b, r in zip(d[prefix + "slotA"], d[prefix + "slotB"], m)}


def _same_geometry(ours, ref, impulses=True):
    n = int(ref["count"])
    assert int(ours["count"]) == n
    got = np.array([ours["nx"], ours["ny"], ours["depth"]], np.float32)
    assert parity.mismatches(got, np.array([ref["nx"], ref["ny"], ref["depth"]], np.float32)) == 0
    pts = np.array([ours["px0"], ours["py0"], ours["px1"], ours["py1"]], np.float32)[:2 * n]
    rpts = np.array([ref["px"][0], ref["py"][0], ref["px"][1], ref["py"][1]], np.float32)[:2 * n]
    assert parity.mismatches(pts, rpts) == 0
    assert [int(ours["id0"]), int(ours["id1"])][:n] == [int(x) for x in ref["id"][:n]]
    if impulses:
        imp = np.array([ours["jn0"], ours["jt0"], ours["jn1"], ours["jt1"]], np.float32)
        rimp = np.array([ref["jn"][0], ref["jt"][0], ref["jn"][1], ref["jt"][1]], np.float32)
        assert parity.mismatches(imp, rimp) == 0


def _states_by_slot(d, prefix):
    starts, slots = d[prefix + "body.groupStarts"], d[prefix + "body.handleSlot"]
    idx = np.arange(slots.size)
    state = np.where(idx < starts[1], ag2d.STATE_STATIC, np.where(idx < starts[2], ag2d.STATE_SLEEPING,
                                                                    ag2d.STATE_DYNAMIC))
    return dict(zip(slots.tolist(), state.tolist()))


def test_woken_islands_bring_their_manifolds_back():
    d = parity.load("towers_s0_step140.npz")
    w = _world(d, body_prefix="int.")
    w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    if not bool(d["sp.spatialDirty"][0]):
        w.run_phase(ag2d.PHASE_SPATIAL_DYNAMIC)
    w.write(ag2d.PAIRS, d["bp.pairs"].reshape(-1, 2))
    _load_store(w, d)
    w.run_phase(ag2d.PHASE_NARROW)
    w.run_phase(ag2d.PHASE_WAKE)
    slot = d["pre.col.handleSlot"]
    ours = _by_slots(w.read(ag2d.MANIFOLDS), slot)
    ref = _ref_by_slots(d, "svin.man.")
    assert len(ref) == 16 and set(ours) == set(ref)
    for k, r in ref.items():
        _same_geometry(ours[k], r)
    assert w.counters()["restored"] == 12
    # The woken towers' bodies are awake, the other sleepers still asleep.
    want = _states_by_slot(d, "svin.")
    state = w.read(ag2d.BODY_STATE)
    for i, s in enumerate(d["pre.body.handleSlot"].tolist()):
        assert int(state[i]) == want[s], i


def test_islands_falling_asleep_store_their_manifolds():
    d = parity.load("towers_s0_step33.npz")
    w = _world(d)
    _load_store(w, d)
    w.step(1)
    assert w.counters()["status"] == 0
    slot = d["pre.col.handleSlot"]
    bslot = d["pre.body.handleSlot"]
    want = _states_by_slot(d, "post.")
    state = w.read(ag2d.BODY_STATE)
    assert all(int(state[i]) == want[s] for i, s in enumerate(bslot.tolist()))
    store = w.read(ag2d.ISLAND_MANIFOLDS)
    ids = w.read(ag2d.ISLAND_IDS)
    ours = _by_slots(store, slot)
    ref = _ref_by_slots(d, "post.isle.")
    assert len(ref) == 108 and set(ours) == set(ref)
    got, fp = [], []
    for k, r in ref.items():
        _same_geometry(ours[k], r, impulses=False)
        got.append(ours[k])
        fp.append(r)
    # Impulses: the colour order against the reference's order, within the solver contract.
    mine = np.array([(g["jn0"], g["jt0"], g["jn1"], g["jt1"]) for g in got], np.float64)
    theirs = np.array([(r["jn"][0], r["jt"][0], r["jn"][1], r["jt"][1]) for r in fp], np.float64)
    cnt = np.array([int(r["count"]) for r in fp])
    active = np.stack([cnt > 0, cnt > 0, cnt > 1, cnt > 1], 1)
    err = np.abs(mine - theirs)[active]
    assert np.all(err <= parity.IMPULSE_CEIL_RTOL * np.abs(theirs[active]) + parity.IMPULSE_CEIL_ATOL)
    # Same island partition of the records.
    order = list(ref)
    rec_island = {k: int(i) for k, i in zip(((int(slot[r["a"]]), int(slot[r["b"]])) for r in store), ids)}
    ref_island = dict(zip(zip(d["post.isle.slotA"].tolist(), d["post.isle.slotB"].tolist()),
                          d["post.isle.islandId"].tolist()))
    assert np.array_equal(parity.partition_labels([rec_island[k] for k in order]),
                          parity.partition_labels([ref_island[k] for k in order]))
    # The warm-start list keeps the manifolds of the towers still awake.
    prev = _by_slots(w.read(ag2d.PREV_MANIFOLDS), slot)
    assert set(prev) == set(_ref_by_slots(d, "post.man."))


def _tower_scenes():
    # Different drop heights and groupings: islands fall asleep and wake in different steps in each world.
    return [scenes.make_towers(towers=t, levels=lv, drops=dr, seed=s, drop_height=h, group=g)
            for t, lv, dr, s, h, g in ((12, 3, 4, 1, 12.0, 2), (7, 2, 3, 2, 9.0, 1), (20, 4, 7, 3, 15.0, 3),
                                       (5, 3, 2, 4, 6.0, 2))]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def test_batch_keeps_each_worlds_store_as_alone():
    sc = _tower_scenes()
    alone = [ag2d.World.from_scene(s) for s in sc]
    batch = ag2d.Batch([ag2d.World.from_scene(s) for s in sc])
    restored = 0
    for _ in range(6):   # 6 x 40 steps: towers sleep, circles hit, woken towers settle and sleep again
        for w in alone:
            w.step(40)
            restored += w.counters()["restored"]
        batch.step(40)
        for k, w in enumerate(alone):
            for f in (ag2d.BODY_COM_X, ag2d.BODY_COM_Y, ag2d.BODY_VEL_Y, ag2d.BODY_STATE, ag2d.BODY_SLEEP_ISLAND):
                assert np.array_equal(_bits(batch.read(k, f)), _bits(w.read(f))), (k, f)
            for f in (ag2d.PREV_MANIFOLDS, ag2d.ISLAND_MANIFOLDS, ag2d.ISLAND_IDS):
                assert np.array_equal(_bits(batch.read(k, f)), _bits(w.read(f))), (k, f)
    assert batch.counters()["status"] == 0
    stored = sum(w.read(ag2d.ISLAND_MANIFOLDS).size for w in alone)
    assert stored > 0
    # Restores happened in the single worlds (counted on the steps that ended a 40-step call): the wake path ran.
    woke = any(int((w.read(ag2d.BODY_STATE) == ag2d.STATE_DYNAMIC).sum()) > 0 for w in alone)
    assert woke or restored > 0


def test_checkpoint_carries_the_store():
    batch = ag2d.Batch([ag2d.World.from_scene(s) for s in _tower_scenes()])
    batch.step(60)   # towers asleep, circles still falling
    assert sum(batch.read(k, ag2d.ISLAND_MANIFOLDS).size for k in range(batch.n_worlds)) > 0
    restored = ag2d.Batch.restore(batch.save())
    batch.step(150)
    restored.step(150)
    for k in range(batch.n_worlds):
        for f in (ag2d.BODY_COM_Y, ag2d.BODY_STATE, ag2d.PREV_MANIFOLDS, ag2d.ISLAND_MANIFOLDS, ag2d.ISLAND_IDS):
            assert np.array_equal(_bits(restored.read(k, f)), _bits(batch.read(k, f))), (k, f)


def _platform_scene():
    """Six towers on the ground and two on a static platform (scene body 1), all asleep after 60 steps."""
    rng = np.random.default_rng(9)
    b = scenes._Builder([scenes.FRICTION_MATERIAL])
    b.add(scenes.BOX, 0.0, -1.0, width=80.0, height=2.0, mass=0.0, material=1)
    b.add(scenes.BOX, 25.0, 0.5, width=8.0, height=1.0, mass=0.0, material=1)
    bases = [(-15.0 + 3.0 * k, 0.0) for k in range(6)] + [(23.5, 1.0), (26.5, 1.0)]
    for x, y0 in bases:
        y = y0
        for _ in range(3):
            s = rng.uniform(0.8, 1.0)
            b.add(scenes.BOX, x + rng.uniform(-0.05, 0.05), y + 0.5 * s + 0.005, width=s, height=s, mass=s * s,
                  material=1)
            y += s + 0.01
    return b.build("platform_towers")


def _pairs_by_scene_body(col_body, body_to_scene, m):
    return {tuple(sorted((body_to_scene[int(col_body[r["a"]])], body_to_scene[int(col_body[r["b"]])]))) for r in m}


def test_commands_wake_islands_and_return_their_manifolds_like_the_reference():
    from oracle import refapi
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    sc = _platform_scene()
    ref = refapi.RefSim(sc)
    w = ag2d.World(dt=sc.dt, gravity=sc.gravity)
    hs = w.add_scene(sc)
    ref.update(60)
    w.step(60)
    # A kick on the top box of the third ground tower (its island wakes) and the platform set to its own position
    # (a static edit: the islands resting on it wake, their stored manifolds with the platform are dropped).
    top = 2 + 2 * 3 + 2
    ref.set_body(top, refapi.RefSim.SET_VELOCITY, 0.0, 2.0)
    ref.set_body(1, refapi.RefSim.SET_POSITION, 25.0, 0.5)
    w.set_body_velocity(int(hs[top]), 0.0, 2.0)
    w.set_body_position(int(hs[1]), 25.0, 0.5)
    for when in ("asleep", "flushed"):
        if when == "flushed":
            ref.flush_commands()
            w.flush_commands()
        ref.dump_state("c.")
        ours_b2s = {w.body_index(int(h)): i for i, h in enumerate(hs)}
        ref_b2s = {ref.body_index(i): i for i in range(sc.n)}
        state = w.read(ag2d.BODY_STATE)
        starts = ref.blob("c.body.groupStarts")
        for i in range(sc.n):
            ri = ref.body_index(i)
            rs = 0 if ri < starts[1] else (1 if ri < starts[2] else 2)
            assert int(state[w.body_index(int(hs[i]))]) == rs, (when, i)
        cb = w.read(ag2d.COL_BODY)
        rcb = ref.blob("c.col.bodyIndex")
        ours_store = _pairs_by_scene_body(cb, ours_b2s, w.read(ag2d.ISLAND_MANIFOLDS))
        ref_store = {tuple(sorted((ref_b2s[int(rcb[a])], ref_b2s[int(rcb[b])])))
                     for a, b in zip(ref.blob("c.isle.colA"), ref.blob("c.isle.colB"))}
        assert ours_store == ref_store, when
        ours_prev = _pairs_by_scene_body(cb, ours_b2s, w.read(ag2d.PREV_MANIFOLDS))
        ref_prev = {tuple(sorted((ref_b2s[int(rcb[a])], ref_b2s[int(rcb[b])])))
                    for a, b in zip(ref.blob("c.man.colA"), ref.blob("c.man.colB"))}
        assert ours_prev == ref_prev, when
        if when == "asleep":
            assert len(ours_store) == 8 * 3 and not ours_prev
        else:
            # The kicked tower's three records are back in the warm-start list; the platform towers' records
            # with the platform are gone, their box-on-box records back in the list.
            assert len(ours_store) == 5 * 3 and len(ours_prev) == 3 + 2 * 2
    ref.update(30)
    w.step(30)
    assert w.counters()["status"] == 0
    ref.close()
