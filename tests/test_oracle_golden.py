"""The oracle (CPU restatement in oracle/) against golden vectors produced by the reference engine itself.

These pin the oracle before it is trusted as the checker of the CUDA path: every phase must reproduce the
reference's output bit for bit on the same inputs.
"""
import numpy as np
import pytest

import parity
from oracle import oraapi


def _fixture(name):
    d = parity.load(name)
    mats = [tuple(r) for r in d["meta.materials"]]
    return d, mats


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_integration_wrap_cossin(oracle_lib, name):
    d, mats = _fixture(name)
    w = oraapi.OraWorld(d, "pre.", mats)
    g = d["meta.gravity"]
    w.integrate(float(d["meta.dt"][0]), float(g[0]), float(g[1]))
    for ours, theirs in [("comX", "comX"), ("comY", "comY"), ("velX", "velocityX"), ("velY", "velocityY"),
                         ("rot", "rotation"), ("angVel", "angularVelocity"), ("rotCos", "rotationCos"),
                         ("rotSin", "rotationSin"), ("wrapCount", "renderRotationWrapCount")]:
        assert parity.mismatches(w.a[ours], d["int.body." + theirs]) == 0, theirs


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_poses_aabbs_morton_sort(oracle_lib, name):
    d, mats = _fixture(name)
    w = oraapi.OraWorld(d, "pre.", mats)
    g = d["meta.gravity"]
    w.integrate(float(d["meta.dt"][0]), float(g[0]), float(g[1]))
    w.spatial(bool(d["sp.spatialDirty"][0]))
    for ours, theirs in oraapi.OraWorld.COL_F.items():
        assert parity.mismatches(w.a[ours], d["sp.col." + theirs]) == 0, theirs
    codes, sorted_c, sorted_k, _ = w.morton(2)
    assert parity.mismatches(sorted_c, d["dyn.sorted"]) == 0
    assert parity.mismatches(sorted_k, d["dyn.morton"]) == 0


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_broad_pair_set(oracle_lib, name):
    d, mats = _fixture(name)
    w = oraapi.OraWorld(d, "sp.", mats, body_prefix="int.")
    ours = w.broad_pairs()
    dyn_begin = int(d["sp.col.groupStarts"][2])
    ref = parity.canonical_pairs(d["bp.pairs"], dyn_begin)
    assert ours.shape == ref.shape
    assert parity.mismatches(ours, ref) == 0


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_narrow_and_warm_start(oracle_lib, name):
    d, mats = _fixture(name)
    w = oraapi.OraWorld(d, "sp.", mats, body_prefix="int.")
    pairs = d["bp.pairs"].reshape(-1, 2)
    m = w.narrow(pairs)
    prev = oraapi.manifolds_from_dump(d, "pre.man.")
    prev_slots = np.stack([d["pre.man.slotA"], d["pre.man.slotB"]], 1)
    slot = d["sp.col.handleSlot"]
    m = oraapi.warm_start(prev, prev_slots, m, np.stack([slot[m["a"]], slot[m["b"]]], 1))
    ref = parity.sort_manifolds(oraapi.manifolds_from_dump(d, "np."))
    m = parity.sort_manifolds(m)
    assert m.shape == ref.shape
    for f in ("a", "b", "nx", "ny", "depth", "count", "jn", "jt"):
        assert parity.mismatches(m[f], ref[f]) == 0, f
    for f in ("px", "py", "id"):
        assert parity.mismatches(parity.active_points(m, f), parity.active_points(ref, f)) == 0, f


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_solver_reference_order_fp32(oracle_lib, name):
    """The FP32 restatement, run in the reference's own constraint order, matches it bit for bit."""
    d, mats = _fixture(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    iters = d["meta.iters"]
    w = oraapi.OraWorld(d, "svin.", mats)
    m = oraapi.manifolds_from_dump(d, "svin.man.")
    out = w.solve(m, None, int(iters[0]), int(iters[1]))
    ref = oraapi.manifolds_from_dump(d, "sv.man.")
    assert parity.mismatches(out["jn"], ref["jn"]) == 0
    assert parity.mismatches(out["jt"], ref["jt"]) == 0
    for ours, theirs in [("velX", "velocityX"), ("velY", "velocityY"), ("angVel", "angularVelocity"),
                         ("comX", "comX"), ("comY", "comY")]:
        assert parity.mismatches(w.a[ours], d["sv.body." + theirs]) == 0, theirs


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_solver_fp64_replay_close_to_fp32(oracle_lib, name):
    """The FP32 restatement in the reference's own order (bit-exact with the reference) meets the impulse contract of
    tests/parity.py against the FP64 replay: this is the precision FP32 arithmetic itself reaches, and the same
    contract is then asked of the GPU's coloured order."""
    d, mats = _fixture(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    iters = d["meta.iters"]
    w32 = oraapi.OraWorld(d, "svin.", mats)
    w64 = oraapi.OraWorld(d, "svin.", mats)
    m = oraapi.manifolds_from_dump(d, "svin.man.")
    out = w32.solve(m, None, int(iters[0]), int(iters[1]))
    vel, pos, imp = w64.solve_f64(m, None, int(iters[0]), int(iters[1]))
    ok, msg = parity.impulses_within_contract(out, imp)
    assert ok, msg


@pytest.mark.parametrize("name", parity.PHASE_FIXTURES)
def test_islands_partition(oracle_lib, name):
    d, mats = _fixture(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    w = oraapi.OraWorld(d, "svin.", mats)
    m = oraapi.manifolds_from_dump(d, "svin.man.")
    body = d["svin.col.bodyIndex"]
    ids, _ = w.islands(np.stack([body[m["a"]], body[m["b"]]], 1))
    assert np.array_equal(parity.partition_labels(ids), parity.partition_labels(d["is.islandId"]))


def test_fastcossin_edges(oracle_lib):
    d = parity.load("cossin_edge.npz")
    c, s = oraapi.fastcossin(d["angles"])
    assert parity.mismatches(c, d["cos"]) == 0
    assert parity.mismatches(s, d["sin"]) == 0


def test_wrap_edges_simd_body_and_tail(oracle_lib):
    d = parity.load("wrap_edge.npz")
    w = oraapi.OraWorld(d, "pre.")
    g = d["meta.gravity"]
    w.integrate(float(d["meta.dt"][0]), float(g[0]), float(g[1]))
    for ours, theirs in [("rot", "rotation"), ("wrapCount", "renderRotationWrapCount"), ("rotCos", "rotationCos"),
                         ("rotSin", "rotationSin")]:
        assert parity.mismatches(w.a[ours], d["int.body." + theirs]) == 0, theirs
    w.spatial(bool(True))
    for ours, theirs in [("worldRot", "worldRotation"), ("worldCos", "worldRotationCos"),
                         ("worldSin", "worldRotationSin"), ("minX", "aabbMinX"), ("maxY", "aabbMaxY")]:
        assert parity.mismatches(w.a[ours], d["sp.col." + theirs]) == 0, theirs


def test_oracle_detects_a_planted_fault(oracle_lib):
    """A restatement with one operation changed must fail the same comparison (the check has teeth)."""
    d, mats = _fixture("c1_n256_s0_step300.npz")
    w = oraapi.OraWorld(d, "sp.", mats, body_prefix="int.")
    m = w.narrow(d["bp.pairs"].reshape(-1, 2))
    w.a["worldX"][int(m["a"][0])] += np.float32(1e-3)
    m2 = w.narrow(d["bp.pairs"].reshape(-1, 2))
    assert parity.mismatches(parity.sort_manifolds(m)["depth"], parity.sort_manifolds(m2)["depth"]) > 0 or \
        m.shape != m2.shape


def test_query_restatement_matches_the_reference():
    """The restated query-shape leaf tests (parity.query_leaf_test, which the GPU query test checks the kernel
    against) find exactly the colliders the reference's own trees return (queryCollidersInShape), for AABB and
    circle shapes and every tree selection, on a settled pile with sleeping bodies."""
    g = parity.load("query_c1_n600_step700.npz")
    starts = g["q.col.groupStarts"]   # BodyGroup order: static, sleeping, dynamic
    n = g["q.col.aabbMinX"].size
    idx = np.arange(n)
    tree_bits = np.where(idx < starts[1], 2, np.where(idx < starts[2], 4, 1))
    assert (tree_bits == 4).any() and (tree_bits == 2).any()
    nonempty = 0
    for k in range(g["shape"].size):
        shape, trees = int(g["shape"][k]), int(g["trees"][k])
        params = g["params"][k][:4] if shape == 0 else g["params"][k][:3]
        got = parity.query_leaf_test(g["q.col.aabbMinX"], g["q.col.aabbMinY"], g["q.col.aabbMaxX"],
                                     g["q.col.aabbMaxY"], tree_bits, shape, params, trees)
        want = g["found"][g["offsets"][k]:g["offsets"][k + 1]]
        assert np.array_equal(got, want), (k, shape, trees)
        nonempty += want.size > 0
    assert nonempty > 20


def test_query_restatement_matches_the_reference_on_mixed_shapes():
    """The same restatement against the reference's shape queries on the mixed-shape pile of the circle-contact
    fixture (circles, boxes, polygons)."""
    g = parity.load("contacts_c2_n1500_step300.npz")
    starts = g["q.col.groupStarts"]
    idx = np.arange(g["q.col.aabbMinX"].size)
    tree_bits = np.where(idx < starts[1], 2, np.where(idx < starts[2], 4, 1))
    for k in range(g["s.shape"].size):
        shape, trees = int(g["s.shape"][k]), int(g["s.trees"][k])
        params = g["s.params"][k][:4] if shape == 0 else g["s.params"][k][:3]
        got = parity.query_leaf_test(g["q.col.aabbMinX"], g["q.col.aabbMinY"], g["q.col.aabbMaxX"],
                                     g["q.col.aabbMaxY"], tree_bits, shape, params, trees)
        assert np.array_equal(got, g["s.idx"][g["s.offsets"][k]:g["s.offsets"][k + 1]]), (k, shape, trees)


def _event_keys(ev, col_slot, body_slot):
    """Events as sorted tuples: handle slots of the colliders and bodies, callback id and the float fields' bits."""
    bits = {k: np.ascontiguousarray(ev[k], dtype=np.float32).view(np.uint32) for k in ("px", "py", "nx", "ny",
                                                                                       "impulse")}
    return sorted(zip(col_slot[ev["self"]].tolist(), col_slot[ev["other"]].tolist(),
                      body_slot[ev["selfBody"]].tolist(), body_slot[ev["otherBody"]].tolist(),
                      np.asarray(ev["callback"]).tolist(), *(bits[k].tolist() for k in bits)))


def test_collision_events_restatement_matches_the_reference(oracle_lib):
    """The restated event records (oraapi.collision_events over the oracle's own integrate, poses, broad and
    narrow phase of the step) are the reference's dispatched events, bit for bit: four steps of a 1,200-body drop
    with two callbacks and colliders opted in at thresholds 0, 0.5, 3 and never."""
    d, mats = _fixture("events_c2_n1200.npz")
    g, dt = d["meta.gravity"], float(d["meta.dt"][0])
    total = 0
    for k in d["meta.steps"].tolist():
        p = f"s{k}."
        w = oraapi.OraWorld(d, p, mats)
        w.integrate(dt, float(g[0]), float(g[1]))
        w.spatial(True)
        m = w.narrow(w.broad_pairs())
        ev = w.collision_events(m, d[p + "col.callbackId"], d[p + "col.eventThreshold"])
        ref = {f: d[f"e{k}.ev.{f}"] for f in ("px", "py", "nx", "ny", "impulse")}
        slot = d[p + "col.handleSlot"]
        bslot = d[p + "body.handleSlot"]
        want = sorted(zip(d[f"e{k}.ev.self"].tolist(), d[f"e{k}.ev.other"].tolist(), d[f"e{k}.ev.selfBody"].tolist(),
                          d[f"e{k}.ev.otherBody"].tolist(), d[f"e{k}.ev.callback"].tolist(),
                          *(np.ascontiguousarray(ref[f], dtype=np.float32).view(np.uint32).tolist() for f in ref)))
        assert _event_keys(ev, slot, bslot) == want, k
        total += len(want)
    assert total > 300
