"""CUDA path against the reference's golden taps and the oracle, phase by phase, through the C ABI.

Tolerances (from the path's parity contract): integration, poses, AABBs, Morton keys, the sorted order and the
candidate pair set are bit-exact; narrow-phase manifolds are bit-exact on the same pair list (the arithmetic is the
reference's, contraction off); solver impulses are bit-exact against the FP32 oracle replay of the GPU's own colour
order and within the impulse contract of tests/parity.py against the FP64 replay (1e-4 relative, absolute floor
1e-4 N s, for at least 99.5 % of impulses; 1e-3 relative + 1e-2 N s for every one; the reference's own FP32 solve
meets the same bound).
"""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from oracle import oraapi  # noqa: E402


def _fixture(name):
    d = parity.load(name)
    return d, [tuple(r) for r in d["meta.materials"]]


def _world(d, mats, prefix, body_prefix=None):
    it = d["meta.iters"] if "meta.iters" in d else np.array([8, 3])
    g = d["meta.gravity"]
    w = ag2d.World(dt=float(d["meta.dt"][0]), velocity_iterations=int(it[0]), position_iterations=int(it[1]),
                   gravity=(float(g[0]), float(g[1])))
    w.load_state(d, prefix, mats, body_prefix)
    return w


def _to_oracle(m):
    out = np.zeros(m.shape[0], oraapi.MANIFOLD_DTYPE)
    for f in ("a", "b", "nx", "ny", "depth", "count"):
        out[f] = m[f]
    out["px"] = np.stack([m["px0"], m["px1"]], 1)
    out["py"] = np.stack([m["py0"], m["py1"]], 1)
    out["id"] = np.stack([m["id0"], m["id1"]], 1)
    out["jn"] = np.stack([m["jn0"], m["jn1"]], 1)
    out["jt"] = np.stack([m["jt0"], m["jt1"]], 1)
    return out


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


BODY_FIELDS = [(ag2d.BODY_COM_X, "comX"), (ag2d.BODY_COM_Y, "comY"), (ag2d.BODY_VEL_X, "velocityX"),
               (ag2d.BODY_VEL_Y, "velocityY"), (ag2d.BODY_ROTATION, "rotation"),
               (ag2d.BODY_ANGULAR_VELOCITY, "angularVelocity"), (ag2d.BODY_ROT_COS, "rotationCos"),
               (ag2d.BODY_ROT_SIN, "rotationSin"), (ag2d.BODY_WRAP_COUNT, "renderRotationWrapCount")]
COL_FIELDS = [(ag2d.COL_WORLD_X, "worldPosX"), (ag2d.COL_WORLD_Y, "worldPosY"),
              (ag2d.COL_WORLD_ROTATION, "worldRotation"), (ag2d.COL_WORLD_COS, "worldRotationCos"),
              (ag2d.COL_WORLD_SIN, "worldRotationSin"), (ag2d.COL_AABB_MIN_X, "aabbMinX"),
              (ag2d.COL_AABB_MIN_Y, "aabbMinY"), (ag2d.COL_AABB_MAX_X, "aabbMaxX"), (ag2d.COL_AABB_MAX_Y, "aabbMaxY")]


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES + ("wrap_edge.npz",))
def test_integrate_bit_exact(name):
    d, mats = _fixture(name) if name != "wrap_edge.npz" else (parity.load(name), None)
    w = _world(d, mats, "pre.")
    w.run_phase(ag2d.PHASE_INTEGRATE)
    for field, ref in BODY_FIELDS:
        assert parity.mismatches(w.read(field), d["int.body." + ref]) == 0, ref


def _spatial(w, d):
    w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    if not bool(d["sp.spatialDirty"][0]):
        w.run_phase(ag2d.PHASE_SPATIAL_DYNAMIC)


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES + ("wrap_edge.npz",))
def test_poses_and_aabbs_bit_exact(name):
    d, mats = _fixture(name) if name != "wrap_edge.npz" else (parity.load(name), None)
    w = _world(d, mats, "pre.", body_prefix="int.")
    if name == "wrap_edge.npz":
        w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    else:
        _spatial(w, d)
    for field, ref in COL_FIELDS:
        assert parity.mismatches(w.read(field), d["sp.col." + ref]) == 0, ref


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES)
def test_broad_morton_sort_pairs_bit_exact(name):
    d, mats = _fixture(name)
    w = _world(d, mats, "pre.", body_prefix="int.")
    _spatial(w, d)
    w.run_phase(ag2d.PHASE_BROAD)
    assert parity.mismatches(w.read(ag2d.DYN_SORTED), d["dyn.sorted"]) == 0
    assert parity.mismatches(w.read(ag2d.DYN_MORTON), d["dyn.morton"]) == 0
    dyn_begin = int(d["sp.col.groupStarts"][2])
    ours = parity.canonical_pairs(w.read(ag2d.PAIRS), dyn_begin)
    ref = parity.canonical_pairs(d["bp.pairs"], dyn_begin)
    assert ours.shape == ref.shape
    assert parity.mismatches(ours, ref) == 0
    # Orientation: dynamic-dynamic pairs lead with the lower Morton rank, cross pairs with the dynamic collider.
    p = w.read(ag2d.PAIRS)
    rank = np.empty(int(d["sp.col.groupStarts"][3]), np.int64)
    rank[d["dyn.sorted"]] = np.arange(d["dyn.sorted"].size)
    both = (p[:, 0] >= dyn_begin) & (p[:, 1] >= dyn_begin)
    assert np.all(rank[p[both, 0]] < rank[p[both, 1]])
    assert np.all(p[~both, 0] >= dyn_begin)


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES)
def test_narrow_and_warm_start_bit_exact(name):
    d, mats = _fixture(name)
    w = _world(d, mats, "pre.", body_prefix="int.")
    _spatial(w, d)
    w.write(ag2d.PAIRS, d["bp.pairs"].reshape(-1, 2))
    w.write(ag2d.PREV_MANIFOLDS, _from_oracle(oraapi.manifolds_from_dump(d, "pre.man.")))
    w.run_phase(ag2d.PHASE_NARROW)
    ours = parity.sort_manifolds(_to_oracle(w.read(ag2d.MANIFOLDS)))
    ref = parity.sort_manifolds(oraapi.manifolds_from_dump(d, "np."))
    assert ours.shape == ref.shape
    for f in ("a", "b", "nx", "ny", "depth", "count", "jn", "jt"):
        assert parity.mismatches(ours[f], ref[f]) == 0, f
    for f in ("px", "py", "id"):
        assert parity.mismatches(parity.active_points(ours, f), parity.active_points(ref, f)) == 0, f


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES)
def test_solver_against_replays_of_the_colour_order(name):
    d, mats = _fixture(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    iters = d["meta.iters"]
    w = _world(d, mats, "svin.")
    m_in = oraapi.manifolds_from_dump(d, "svin.man.")
    w.write(ag2d.MANIFOLDS, _from_oracle(m_in))
    w.run_phase(ag2d.PHASE_SOLVE)
    order = w.read(ag2d.SOLVE_ORDER).astype(np.int64)
    starts = w.read(ag2d.COLOR_STARTS)
    assert np.array_equal(np.sort(order), np.arange(m_in.size))
    # Colours are independent sets over dynamic bodies.
    body = d["svin.col.bodyIndex"]
    inv_mass = d["svin.body.invMass"]
    for c in range(starts.size - 1):
        ms = order[starts[c]:starts[c + 1]]
        bodies = np.concatenate([body[m_in["a"][ms]], body[m_in["b"][ms]]])
        dyn = bodies[inv_mass[bodies] > 0]
        assert np.unique(dyn).size == dyn.size, f"colour {c} shares a dynamic body"
    ours = _to_oracle(w.read(ag2d.MANIFOLDS))
    # FP32 replay of the same order: bit-exact.
    o32 = oraapi.OraWorld(d, "svin.", mats)
    rep = o32.solve(m_in, order, int(iters[0]), int(iters[1]))
    assert parity.mismatches(ours["jn"], rep["jn"]) == 0
    assert parity.mismatches(ours["jt"], rep["jt"]) == 0
    for field, ref in [(ag2d.BODY_VEL_X, "velX"), (ag2d.BODY_VEL_Y, "velY"), (ag2d.BODY_ANGULAR_VELOCITY, "angVel"),
                       (ag2d.BODY_COM_X, "comX"), (ag2d.BODY_COM_Y, "comY")]:
        assert parity.mismatches(w.read(field), o32.a[ref]) == 0, ref
    # FP64 replay of the same order: the impulse contract of tests/parity.py (1e-4 relative for all but a stated
    # share, and a hard ceiling for every impulse), the bound the reference's own FP32 solve meets.
    o64 = oraapi.OraWorld(d, "svin.", mats)
    _, _, imp = o64.solve_f64(m_in, order, int(iters[0]), int(iters[1]))
    ok, msg = parity.impulses_within_contract(ours, imp)
    assert ok, msg


@pytest.mark.parametrize("name", parity.GPU_PHASE_FIXTURES)
def test_islands_partition(name):
    d, mats = _fixture(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    w = _world(d, mats, "svin.")
    m_in = oraapi.manifolds_from_dump(d, "svin.man.")
    w.write(ag2d.MANIFOLDS, _from_oracle(m_in))
    w.run_phase(ag2d.PHASE_ISLANDS)
    state = w.read(ag2d.BODY_STATE)
    ora = oraapi.OraWorld(d, "svin.", mats)
    body = d["svin.col.bodyIndex"]
    ids, k = ora.islands(np.stack([body[m_in["a"]], body[m_in["b"]]], 1))
    sleep = ora.update_sleeping(ids, k, float(d["meta.dt"][0]))
    assert np.array_equal(state == 1, sleep.astype(bool) | (d["svin.body.groupStarts"][1] <= np.arange(state.size)) &
                          (np.arange(state.size) < d["svin.body.groupStarts"][2]))


def test_pair_set_at_scale_matches_oracle():
    """200k circles and 4-6-gons (the broad+narrow stress scene at reduced size): exact pair set and sorted keys."""
    from ag2d import scenes
    sc = scenes.make_c3(200_000, 5, extent=1800.0)
    w = ag2d.World.from_scene(sc)
    w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    w.run_phase(ag2d.PHASE_BROAD)
    keys = w.read(ag2d.DYN_MORTON)
    assert np.all(keys[1:] >= keys[:-1])
    srt = w.read(ag2d.DYN_SORTED)
    assert np.array_equal(np.sort(srt), np.arange(srt.size))
    state = {"body.groupStarts": np.array([0, 0, 0, sc.n], np.uint32),
             "col.groupStarts": np.array([0, 0, 0, sc.n], np.uint32)}
    minx, miny = w.read(ag2d.COL_AABB_MIN_X), w.read(ag2d.COL_AABB_MIN_Y)
    maxx, maxy = w.read(ag2d.COL_AABB_MAX_X), w.read(ag2d.COL_AABB_MAX_Y)
    ours = parity.canonical_pairs(w.read(ag2d.PAIRS), 0)
    # Oracle sweep over the same AABBs.
    lib = oraapi.lib()
    c = oraapi.OraWorldC()
    c.n_bodies = sc.n
    c.n_colliders = sc.n
    for k in range(4):
        c.col_starts[k] = int(state["col.groupStarts"][k])
    keep = []
    for name, arr in (("minX", minx), ("minY", miny), ("maxX", maxx), ("maxY", maxy),
                      ("bodyIndex", np.arange(sc.n, dtype=np.uint32))):
        a = np.ascontiguousarray(arr)
        keep.append(a)
        setattr(c, name, a.ctypes.data_as(oraapi._U if a.dtype == np.uint32 else oraapi._F))
    cap = 16 * sc.n
    out = np.zeros((cap, 2), np.uint32)
    import ctypes
    n = lib.ora_broad_pairs(ctypes.byref(c), out.ctypes.data, cap)
    assert n >= 0
    ref = out[:n]
    assert ours.shape == ref.shape
    assert parity.mismatches(ours, ref) == 0


def test_full_steps_run_and_count():
    from ag2d import scenes
    w = ag2d.World.from_scene(scenes.make_c1(256, 0))
    w.step(120)
    c = w.counters()
    assert c["status"] == 0
    assert c["steps"] == 120
    assert c["manifolds"] > 0 and c["pairs"] >= c["manifolds"]
    vy = w.read(ag2d.BODY_VEL_Y)
    assert np.all(np.isfinite(vy))


def test_collision_pass_replayed_as_a_graph_gives_the_same_results():
    """AG2D_PHASE_COLLIDE: the first pass of a launch shape runs as it is, the second is captured into a CUDA graph,
    later ones replay it. With the bodies unmoved every pass finds the same pairs and manifolds, bit for bit, and
    the replays count the graph's launches."""
    from ag2d import scenes
    sc = scenes.make_c3(100_000, 7, extent=1300.0)
    w = ag2d.World.from_scene(sc)
    w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    results, launches = [], []
    for _ in range(5):
        before = w.counters()["launches"]
        w.run_phase(ag2d.PHASE_COLLIDE)
        launches.append(w.counters()["launches"] - before)
        results.append((parity.canonical_pairs(w.read(ag2d.PAIRS), 0),
                        parity.sort_manifolds(_to_oracle(w.read(ag2d.MANIFOLDS)))))
    p0, m0 = results[0]
    assert p0.shape[0] > 1000 and m0.size > 100
    for p, m in results[1:]:
        assert np.array_equal(p, p0)
        assert m.tobytes() == m0.tobytes()
    assert len(set(launches[1:])) == 1 and launches[1] > 5
    assert w.counters()["status"] == 0
