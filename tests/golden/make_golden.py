"""Generates the golden vectors in tests/golden/ from the reference engine itself.

The reference (PS_AGONY2D) ships no tests, fixtures or known-answer vectors, so its behaviour is pinned by running
it: oracle/ref_build.sh compiles the reference's own sources on the CPU (oracle/_ref/libagony_ref.so) and this
script drives them through oracle/refapi.py on seeded synthetic scenes (ag2d.scenes), saving per-phase taps.

Run from the repository root (needs the reference checkout, so only in the build container):
    oracle/ref_build.sh && python tests/golden/make_golden.py

Fixtures:
    c1_n256_s0_step300.npz  polygons on a ground box, phase taps of step 301 (contacts, warm start, solver)
    c2_n2000_s1_step240.npz circles/boxes/polygons in a U container, phase taps of step 241
    c3_n1500_s0_step0.npz   circles and 4-6-gons, no gravity, the first step (full spatial rebuild)
    cossin_edge.npz         FastCosSin over edge angles (quadrant boundaries, values just below 2 pi)
    wrap_edge.npz           body rotations around wrap boundaries (SIMD body and scalar tail)
    traj_c1_n256.npz        600-step trajectory statistics of a 256-polygon scene
    traj_c1_n2048.npz       the same statistics of the full c1 configuration (2,048 polygons, seed 0, 600 steps)
    contacts_capsules_n1500_step300.npz  circle contacts and shape queries on a 1,500-body pile with capsules among
                            circles, boxes and polygons (findCollisionsInCircle's capsule branch)
    events_c2_n1200.npz     collision events of four steps of a 1,200-body mixed-shape drop (two callbacks, colliders
                            opted in at several thresholds), with the reference's state before each step
    towers_s0_step33.npz    40 three-box towers: the step in which 36 of them fall asleep (their manifolds go to
                            the sleeping-island store), with the store after the step
    towers_s0_step140.npz   the same scene: the step in which four towers wake and their stored manifolds return
    capsules_n1500_s0_step300.npz  capsules with circles, boxes and polygons in a U container (every shape pair),
                               phase taps of step 301
    c2_n20000_s2_step420.npz   20,000 bodies of the c2 mix (500 columns x 40 rows) in a U container, phase taps of step 421 (the
                               narrow phase and the solver compared at scale)
    c5_ccd_hit.npz          the first continuous-collision hit of a serving-style request (fast circles)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "physicssimulation-agony_b200"))

from ag2d import scenes  # noqa: E402
from oracle import refapi  # noqa: E402

PHASE_PREFIXES = ("pre.", "int.body.", "sp.col.", "sp.spatialDirty", "dyn.", "bp.pairs", "np.", "svin.", "sv.",
                  "is.islandId", "post.body.", "post.man.")
DROP_SUFFIXES = (".localOffsetX", ".localOffsetY", ".mass", ".inertia", ".localCenterOfMassX",
                 ".localCenterOfMassY", ".minExtent", ".maxExtent")


def dedupe(blobs):
    """Stores each distinct array once: a later array equal to an earlier one (same dtype, shape and bytes)
    becomes an entry "later=earlier" of meta.aliases, which tests/parity.py load() expands."""
    seen, out, aliases = {}, {}, []
    for k in sorted(blobs):
        v = np.ascontiguousarray(blobs[k])
        key = (v.dtype.str, v.shape, v.tobytes())
        if key in seen and not k.startswith("meta."):
            aliases.append(f"{k}={seen[key]}")
        else:
            seen.setdefault(key, k)
            out[k] = v
    if aliases:
        out["meta.aliases"] = np.array(aliases)
    return out


def phase_fixture(scene, steps, path, prefixes=PHASE_PREFIXES, store_once=False):
    r = refapi.RefSim(scene)
    r.update(steps)
    r.phase_step()
    blobs = {k: v for k, v in r.blobs().items()
             if k.startswith(prefixes) and not k.endswith(DROP_SUFFIXES)}
    blobs["meta.dt"] = np.array([scene.dt], np.float32)
    blobs["meta.gravity"] = np.array(scene.gravity, np.float32)
    blobs["meta.iters"] = np.array([scene.velocity_iterations, scene.position_iterations], np.uint32)
    blobs["meta.materials"] = np.array([(1.0, 0.0, 0.0)] + list(scene.materials), np.float32)
    np.savez_compressed(path, **(dedupe(blobs) if store_once else blobs))
    r.close()
    print(f"{os.path.basename(path)}: {len(blobs)} arrays, pairs {blobs['bp.pairs'].size // 2}, "
          f"manifolds {blobs.get('np.count', np.zeros(0)).size}")


def cossin_fixture(path):
    two_pi = np.float32(2.0 * np.pi)
    half_pi = np.float32(0.5 * np.pi)
    edges = []
    for base in (np.float32(0.0), half_pi, np.float32(np.pi), np.float32(1.5 * np.pi), two_pi):
        b = np.float32(base)
        v = b
        for _ in range(6):
            v = np.nextafter(v, np.float32(-1.0), dtype=np.float32)
            edges.append(v)
        v = b
        for _ in range(6):
            edges.append(v)
            v = np.nextafter(v, np.float32(10.0), dtype=np.float32)
    rng = np.random.default_rng(7)
    angles = np.concatenate([np.asarray(edges, np.float32), rng.uniform(0, 2 * np.pi, 971).astype(np.float32)])
    angles = angles[(angles >= 0) & (angles <= two_pi)]
    c, s = refapi.fastcossin(angles)
    np.savez_compressed(path, angles=angles, cos=c, sin=s)
    print(f"{os.path.basename(path)}: {angles.size} angles")


def wrap_fixture(path):
    """21 bodies (ground + 20 dynamic): the dynamic range splits into a SIMD body of 16 and a scalar tail of 4."""
    scene = scenes.make_c1(20, 3)
    r = refapi.RefSim(scene)
    n = refapi.lib().agref_body_count(r.h)
    rng = np.random.default_rng(11)
    two_pi = np.float32(2.0 * np.pi)
    special = np.array([-1e-7, -two_pi, two_pi, np.nextafter(two_pi, np.float32(0), dtype=np.float32),
                        np.nextafter(two_pi, np.float32(10), dtype=np.float32), 100.0, -100.0, 1e4, -1e4,
                        3 * two_pi, -3 * two_pi], np.float32)
    rot = rng.uniform(-50, 50, n).astype(np.float32)
    rot[1:1 + special.size] = special
    rot[n - 4:] = special[-4:]
    r.set_body_field("rotation", rot)
    r.set_body_field("angularVelocity", rng.uniform(-30, 30, n).astype(np.float32))
    r.phase_step()
    keep = {k: v for k, v in r.blobs().items() if k.startswith(("pre.", "int.body.", "sp.col."))
            and not k.endswith(DROP_SUFFIXES)}
    keep["meta.dt"] = np.array([scene.dt], np.float32)
    keep["meta.gravity"] = np.array(scene.gravity, np.float32)
    np.savez_compressed(path, **keep)
    r.close()
    print(f"{os.path.basename(path)}: {n} bodies")


def trajectory_stats(sim, steps):
    """Per-step: momentum (sum m v), kinetic energy, max manifold depth, manifold count, the manifolds stored for
    sleeping islands, sleeping bodies; and, since
    bodies near the ends of the ground can slide off and fall without limit, the kinetic energy of the bodies still
    at or above the ground's top ("ke_on": centre of mass above y = -1) and the number that have fallen off
    ("fallen": below y = -10)."""
    out = {k: [] for k in ("px", "py", "ke", "max_depth", "manifolds", "sleeping", "ke_on", "fallen", "stored")}
    for _ in range(steps):
        sim.update(1)
        sim.dump_state("t.")
        m = sim.blob("t.body.mass")
        vx, vy, w = sim.blob("t.body.velocityX"), sim.blob("t.body.velocityY"), sim.blob("t.body.angularVelocity")
        inertia = sim.blob("t.body.inertia")
        dyn = m > 0
        out["px"].append(float(np.sum((m * vx)[dyn], dtype=np.float64)))
        out["py"].append(float(np.sum((m * vy)[dyn], dtype=np.float64)))
        ke = 0.5 * (m * (vx * vx + vy * vy) + inertia * w * w)
        out["ke"].append(float(np.sum(ke[dyn], dtype=np.float64)))
        y = sim.blob("t.body.comY")
        out["ke_on"].append(float(np.sum(ke[dyn & (y > -1.0)], dtype=np.float64)))
        out["fallen"].append(int(np.sum(dyn & (y < -10.0))))
        depth = sim.blob("t.man.depth")
        out["max_depth"].append(float(depth.max()) if depth.size else 0.0)
        out["manifolds"].append(int(depth.size))
        out["stored"].append(int(sim.blob("t.isle.count").size))   # manifolds of sleeping islands
        gs = sim.blob("t.body.groupStarts")
        out["sleeping"].append(int(gs[2] - gs[1]))
    return {k: np.asarray(v) for k, v in out.items()}


def trajectory_fixture(path, n=256, steps=600):
    scene = scenes.make_c1(n, 0)
    r = refapi.RefSim(scene)
    stats = trajectory_stats(r, steps)
    np.savez_compressed(path, **stats)
    r.close()
    print(f"{os.path.basename(path)}: {steps} steps, final KE {stats['ke'][-1]:.3f}, "
          f"sleeping {stats['sleeping'][-1]}")


def ccd_fixture(path, max_steps=80):
    """First step with a continuous-collision hit in a serving-style request (c1 mix + 5% fast circles at 200 m/s,
    continuous collision on): the state entering the step, the spatial tap and the state after the move-back."""
    scene = scenes.make_c5_request(np.random.default_rng(3), 0, lo=200, hi=300)
    r = refapi.RefSim(scene, ccd=True)
    for step in range(max_steps):
        r.phase_step()
        if int(r.blob("ccd.hit").view(np.uint32)[0]):
            break
    else:
        raise RuntimeError("no continuous-collision hit")
    keep = {k: v for k, v in r.blobs().items() if k.startswith(("pre.", "sp.", "ccd."))
            and not k.endswith(tuple(x for x in DROP_SUFFIXES if x != ".minExtent"))}
    keep["meta.dt"] = np.array([scene.dt], np.float32)
    keep["meta.gravity"] = np.array(scene.gravity, np.float32)
    keep["meta.iters"] = np.array([scene.velocity_iterations, scene.position_iterations], np.uint32)
    keep["meta.materials"] = np.array([(1.0, 0.0, 0.0)] + list(scene.materials), np.float32)
    keep["meta.step"] = np.array([step], np.uint32)
    np.savez_compressed(path, **keep)
    r.close()
    print(f"{os.path.basename(path)}: step {step}, {scene.n} bodies")


def query_fixture(path, n=600, steps=700, queries=24):
    """Spatial queries through the reference's own trees (agref_query_shape: queryCollidersInShape with AABB and
    circle shapes, every tree selection) on a settled pile with sleeping bodies, with the colliders' AABBs and
    group ranges the queries ran on."""
    scene = scenes.make_c1(n, seed=5, width=60.0, height=40.0)
    r = refapi.RefSim(scene)
    r.update(steps)
    r.dump_state("q.")
    b = r.blobs("q.col.")
    rng = np.random.default_rng(9)
    params, shapes, trees, found, offsets = [], [], [], [], [0]
    for _ in range(queries):
        cx, cy = rng.uniform(-35, 35), rng.uniform(-5, 30)
        hw, hh, rad = rng.uniform(0.1, 15), rng.uniform(0.1, 15), rng.uniform(-1, 12)
        for t in (7, 1, 2, 4, 5):
            for shape, prm in ((0, (cx - hw, cy - hh, cx + hw, cy + hh, 0.0)), (1, (cx, cy, rad, 0.0, 0.0))):
                got = r.query_shape(shape, prm[:4] if shape == 0 else prm[:3], t)
                params.append(prm); shapes.append(shape); trees.append(t)
                found.append(np.sort(got)); offsets.append(offsets[-1] + got.size)
    keep = {k: b[k] for k in ("q.col.aabbMinX", "q.col.aabbMinY", "q.col.aabbMaxX", "q.col.aabbMaxY",
                              "q.col.groupStarts")}
    keep["params"] = np.asarray(params, np.float32)
    keep["shape"] = np.asarray(shapes, np.uint32)
    keep["trees"] = np.asarray(trees, np.uint32)
    keep["found"] = np.concatenate(found).astype(np.uint32)
    keep["offsets"] = np.asarray(offsets, np.uint32)
    np.savez_compressed(path, **keep)
    r.close()
    print(f"{os.path.basename(path)}: {len(shapes)} queries, groups {keep['q.col.groupStarts'].tolist()}")


def contacts_fixture(path, n=1500, steps=300, queries=60, capsules=False):
    """Circle contacts (agref_circle_contacts: the circle query's colliders through findCollisionsInCircle) and
    shape queries on a mixed-shape pile (circles, boxes, polygons in a U container; with 'capsules', capsules among
    them), with the full reference state they ran on, so that a world loaded from it answers the same queries."""
    scene = scenes.make_capsule_mix(n, 0) if capsules else scenes.make_c2(n, 2, columns=30)
    r = refapi.RefSim(scene)
    r.update(steps)
    r.dump_state("q.")
    keep = {k: v for k, v in r.blobs("q.").items() if not k.startswith("q.man.")}
    rng = np.random.default_rng(21)
    cparams, ctrees, cidx, csdf, coff = [], [], [], [], [0]
    sparams, sshape, strees, sidx, soff = [], [], [], [], [0]
    for _ in range(queries):
        c = int(rng.integers(0, keep["q.col.worldPosX"].size))   # near a random collider: contacts of every shape
        x = float(keep["q.col.worldPosX"][c]) + rng.uniform(-2.0, 2.0)
        y = float(keep["q.col.worldPosY"][c]) + rng.uniform(-2.0, 2.0)
        rad = rng.uniform(-0.5, 6.0)
        hw, hh = rng.uniform(0.1, 8.0), rng.uniform(0.1, 8.0)
        for t in (7, 1, 2, 4, 6):
            idx, sdf = r.circle_contacts(x, y, rad, t)
            order = np.argsort(idx, kind="stable")
            cparams.append((x, y, rad)); ctrees.append(t)
            cidx.append(idx[order]); csdf.append(sdf[order]); coff.append(coff[-1] + idx.size)
            for shape, prm in ((0, (x - hw, y - hh, x + hw, y + hh)), (1, (x, y, rad, 0.0))):
                got = np.sort(r.query_shape(shape, prm[:4] if shape == 0 else prm[:3], t))
                sparams.append(prm); sshape.append(shape); strees.append(t)
                sidx.append(got); soff.append(soff[-1] + got.size)
    keep["c.params"] = np.asarray(cparams, np.float32)
    keep["c.trees"] = np.asarray(ctrees, np.uint32)
    keep["c.idx"] = np.concatenate(cidx).astype(np.uint32)
    keep["c.sdf"] = np.concatenate(csdf).astype(np.float32)
    keep["c.offsets"] = np.asarray(coff, np.uint32)
    keep["s.params"] = np.asarray(sparams, np.float32)
    keep["s.shape"] = np.asarray(sshape, np.uint32)
    keep["s.trees"] = np.asarray(strees, np.uint32)
    keep["s.idx"] = np.concatenate(sidx).astype(np.uint32)
    keep["s.offsets"] = np.asarray(soff, np.uint32)
    keep["meta.materials"] = np.array([(1.0, 0.0, 0.0)] + list(scene.materials), np.float32)
    np.savez_compressed(path, **keep)
    r.close()
    print(f"{os.path.basename(path)}: {len(ctrees)} circle-contact queries ({keep['c.idx'].size} contacts), "
          f"{len(sshape)} shape queries, groups {keep['q.col.groupStarts'].tolist()}")


EVENT_STEPS = (40, 80, 130, 200)
EVENT_SLEEP_TIME = 1.0e6   # no body falls asleep: each step's state is the whole of what the next step reads
NEVER = float(np.finfo(np.float32).max)


def events_fixture(path, n=1200, steps=EVENT_STEPS):
    """Collision events (Simulation::setColliderCollisionCallback, events recorded in computeConstraintData and
    dispatched at the end of the step) on a mixed-shape drop: two recording callbacks, the colliders opted in by
    dense index (id 1 at threshold 0, id 2 at 0.5, id 1 at 3, none, id 2 never firing), and for each step in
    'steps' the reference's full state before it ("s<k>.", with each collider's callback id and threshold) and the
    events it dispatched ("e<k>.ev.*", by handle slot)."""
    scene = scenes.make_c2(n, 0, columns=30)
    r = refapi.RefSim(scene, sleep_time=EVENT_SLEEP_TIME)
    ids = [r.create_event_callback(), r.create_event_callback()]
    r.dump_state("c.")
    pattern = [(ids[0], 0.0), (ids[1], 0.5), (ids[0], 3.0), None, (ids[1], NEVER)]
    for i in range(r.blob("c.col.bodyIndex").size):
        p = pattern[i % len(pattern)]
        if p is not None:
            assert r.set_collider_callback(i, *p)
    keep, done, counts, r_manifolds = {}, 0, [], []
    for k in steps:
        r.update(k - done)
        done = k + 1
        r.events()   # the events of the steps before
        r.dump_state(f"s{k}.")
        keep.update({key: v for key, v in r.blobs(f"s{k}.").items()
                     if not key.startswith(f"s{k}.man.") and not key.startswith(f"s{k}.isle.")
                     and not key.endswith(DROP_SUFFIXES)})
        assert keep[f"s{k}.body.groupStarts"][1] == keep[f"s{k}.body.groupStarts"][2], "no body may sleep yet"
        r.update(1)
        r_manifolds.append(r.manifold_count)
        ev = r.events(f"e{k}.")
        keep.update({f"e{k}.ev.{name}": v for name, v in ev.items()})
        counts.append(ev["self"].size)
    keep["meta.steps"] = np.asarray(steps, np.uint32)
    keep["meta.sleep_time"] = np.array([EVENT_SLEEP_TIME], np.float32)
    keep["meta.dt"] = np.array([scene.dt], np.float32)
    keep["meta.gravity"] = np.array(scene.gravity, np.float32)
    keep["meta.iters"] = np.array([scene.velocity_iterations, scene.position_iterations], np.uint32)
    keep["meta.materials"] = np.array([(1.0, 0.0, 0.0)] + list(scene.materials), np.float32)
    np.savez_compressed(path, **dedupe(keep))
    r.close()
    print(f"{os.path.basename(path)}: events per step {dict(zip(steps, counts))}, manifolds {r_manifolds}")


FIXTURES = {
    "c1_n256_s0_step300.npz": lambda p: phase_fixture(scenes.make_c1(256, 0), 300, p),
    "c2_n2000_s1_step240.npz": lambda p: phase_fixture(scenes.make_c2(2000, 1, columns=50), 240, p),
    "c3_n1500_s0_step0.npz": lambda p: phase_fixture(scenes.make_c3(1500, 0, extent=70.0), 0, p),
    # The post-step taps are left out of the large fixture (no test reads them), to keep it small.
    "c2_n20000_s2_step420.npz": lambda p: phase_fixture(scenes.make_c2(20000, 2, columns=500), 420, p,
                                                        tuple(x for x in PHASE_PREFIXES if not x.startswith("post.")),
                                                        store_once=True),
    "capsules_n1500_s0_step300.npz": lambda p: phase_fixture(scenes.make_capsule_mix(1500, 0), 300, p,
                                                            store_once=True),
    # Sleeping islands' manifolds: 36 towers fall asleep in step 34 (108 records move to the store); four towers
    # wake in step 141 (12 stored records join the solver's list).
    "towers_s0_step33.npz": lambda p: phase_fixture(scenes.make_towers(seed=0), 33, p,
                                                    PHASE_PREFIXES + ("post.isle.",)),
    "towers_s0_step140.npz": lambda p: phase_fixture(scenes.make_towers(seed=0), 140, p,
                                                     PHASE_PREFIXES + ("post.isle.",)),
    "cossin_edge.npz": cossin_fixture,
    "wrap_edge.npz": wrap_fixture,
    "traj_c1_n256.npz": trajectory_fixture,
    "traj_c1_n2048.npz": lambda p: trajectory_fixture(p, n=2048),
    "c5_ccd_hit.npz": ccd_fixture,
    "query_c1_n600_step700.npz": query_fixture,
    "contacts_c2_n1500_step300.npz": contacts_fixture,
    "contacts_capsules_n1500_step300.npz": lambda p: contacts_fixture(p, capsules=True),
    "events_c2_n1200.npz": events_fixture,
}


def main():
    if not refapi.available():
        sys.exit("oracle/_ref/libagony_ref.so missing: run oracle/ref_build.sh first")
    names = sys.argv[1:] or list(FIXTURES)
    for name in names:
        FIXTURES[name](os.path.join(HERE, name))


if __name__ == "__main__":
    main()
