"""Bodies with several colliders (ObjectAPI::createBody + create*Collider, SimulationAPIs/ObjectAPI.h:28-32) through
the C ABI, against the reference engine making the same calls (oracle/ref_harness.cpp: agref_create_body,
agref_add_collider).

- Free flight: compound bodies (two circles on a bar, an L of two boxes, a capsule with a polygon, a rotated box
  ring) spinning and falling far apart, so each body's motion depends on its own state only. After 40 steps every
  body field and every collider's world pose and AABB equal the reference's bit for bit, colliders matched by owner
  body and creation order (dense orders differ by design).
- Landing: the same bodies dropped onto a static floor made by createBody with zero mass. The step on which the
  colliders first touch the floor gives the same manifolds (collider pair, normal, depth, points, feature ids) bit for
  bit; the impulses then differ by solving order only, so after the bodies settle their resting heights agree with the
  reference's to a millimetre.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from oracle import refapi  # noqa: E402

CIRCLE, BOX, POLYGON, CAPSULE = 0, 1, 2, 3
HEX = np.array([[np.cos(a), np.sin(a)] for a in np.arange(6) * np.pi / 3], np.float32) * 0.6
TRI = np.array([[0.0, 0.0], [1.2, 0.1], [0.3, 0.9]], np.float32)   # off-centre: recentred on its centroid

# (mass, inertia, centre of mass, [(shape, offset, rotation, params)]) per compound body.
BODIES = [
    (2.0, 1.3, (0.0, 0.0), [(CIRCLE, (-1.0, 0.0), 0.0, dict(radius=0.4)),
                            (CIRCLE, (1.0, 0.0), 0.0, dict(radius=0.4)),
                            (BOX, (0.0, 0.0), 0.0, dict(width=2.0, height=0.2))]),
    (3.0, 2.1, (0.25, 0.25), [(BOX, (0.0, 0.0), 0.0, dict(width=2.0, height=0.5)),
                              (BOX, (-0.75, 0.75), 0.0, dict(width=0.5, height=1.5))]),
    (1.5, 0.9, (0.1, -0.2), [(CAPSULE, (0.0, 0.0), 0.3, dict(length=1.6, radius=0.3)),
                             (POLYGON, (0.5, 0.4), 0.7, dict(vertices=TRI))]),
    (4.0, 3.5, (0.0, 0.0), [(BOX, (np.cos(a) * 1.2, np.sin(a) * 1.2), a + 1.5707964, dict(width=1.0, height=0.3))
                            for a in np.arange(5) * 2 * np.pi / 5 - np.pi / 10]),   # a plate at the bottom
    (2.5, 1.7, (0.0, 0.3), [(POLYGON, (0.0, 0.0), 0.0, dict(vertices=HEX)),
                            (CAPSULE, (0.0, 0.9), 1.5707964, dict(length=0.8, radius=0.2)),
                            (CIRCLE, (0.9, 0.0), 0.0, dict(radius=0.25))]),
]
BODY_FIELDS = [(ag2d.BODY_COM_X, "comX"), (ag2d.BODY_COM_Y, "comY"), (ag2d.BODY_VEL_X, "velocityX"),
               (ag2d.BODY_VEL_Y, "velocityY"), (ag2d.BODY_ROTATION, "rotation"),
               (ag2d.BODY_ANGULAR_VELOCITY, "angularVelocity"), (ag2d.BODY_ROT_COS, "rotationCos"),
               (ag2d.BODY_ROT_SIN, "rotationSin"), (ag2d.BODY_INV_MASS, "invMass"),
               (ag2d.BODY_INV_INERTIA, "invInertia")]
COL_FIELDS = [(ag2d.COL_WORLD_X, "worldPosX"), (ag2d.COL_WORLD_Y, "worldPosY"),
              (ag2d.COL_WORLD_COS, "worldRotationCos"), (ag2d.COL_WORLD_SIN, "worldRotationSin"),
              (ag2d.COL_WORLD_ROTATION, "worldRotation"), (ag2d.COL_AABB_MIN_X, "aabbMinX"),
              (ag2d.COL_AABB_MIN_Y, "aabbMinY"), (ag2d.COL_AABB_MAX_X, "aabbMaxX"),
              (ag2d.COL_AABB_MAX_Y, "aabbMaxY")]


MATERIAL = (0.0, 0.6, 0.4)   # elasticity, static friction, dynamic friction: the bodies come to rest


class _Scene:   # the settings RefSim reads; no bodies (they are made through create_body / add_collider)
    n = 0
    materials = []
    dt = 1.0 / 60.0
    velocity_iterations, position_iterations = 8, 3
    gravity = (0.0, -9.81)


def _build(layout):
    """Both engines with the floor (if any) and the compound bodies at layout[k] = (x, y, rotation, w).
    Returns (ref, world, ref body ids, our handles), the floor first when present."""
    ref = refapi.RefSim(_Scene())
    w = ag2d.World(dt=_Scene.dt, gravity=_Scene.gravity)
    rmat, gmat = ref.add_material(*MATERIAL), w.add_material(*MATERIAL)
    rids, hs = [], []
    if layout["floor"]:
        rids.append(ref.create_body(0.0, -1.0, mass=0.0, inertia=0.0))
        hs.append(w.create_body(0.0, -1.0, mass=0.0, inertia=0.0))
        ref.add_collider(rids[-1], BOX, material=rmat, width=200.0, height=2.0)
        w.add_collider(hs[-1], BOX, material=gmat, width=200.0, height=2.0)
    for (mass, inertia, com, cols), (x, y, rot, av) in zip(layout.get("bodies", BODIES), layout["poses"]):
        rids.append(ref.create_body(x, y, rotation=rot, w=av, mass=mass, inertia=inertia, com=com))
        hs.append(w.create_body(x, y, rotation=rot, w=av, mass=mass, inertia=inertia, com=com))
        for shape, off, lrot, params in cols:
            ref.add_collider(rids[-1], shape, offset=off, rotation=lrot, material=rmat, **params)
            w.add_collider(hs[-1], shape, offset=off, rotation=lrot, material=gmat, **params)
    return ref, w, rids, hs


def _collider_map(ref, w, rids, hs, prefix):
    """Our collider index -> the reference's, matching the colliders of each body in creation order."""
    ours_body = w.read(ag2d.COL_BODY)
    ref_body = ref.blob(prefix + "col.bodyIndex")
    mapping = {}
    for rid, h in zip(rids, hs):
        mine = np.nonzero(ours_body == w.body_index(h))[0]
        theirs = np.nonzero(ref_body == ref.body_index(rid))[0]
        assert mine.size == theirs.size
        # Creation order: ours keeps it in the dense order; the reference's dense order within one body's group
        # follows its handle slots, which it hands out in creation order on a fresh simulation.
        theirs = theirs[np.argsort(ref.blob(prefix + "col.handleSlot")[theirs], kind="stable")]
        mapping.update(zip(mine.tolist(), theirs.tolist()))
    return mapping


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_compound_bodies_in_free_flight_match_the_reference():
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    poses = [(12.0 * k, 20.0 + 3.0 * k, 0.3 * k, 1.5 - 0.7 * k) for k in range(len(BODIES))]
    ref, w, rids, hs = _build({"floor": False, "poses": poses})
    ref.update(40)
    w.step(40)
    ref.dump_state("f.")
    for f, name in BODY_FIELDS:
        mine, theirs = w.read(f), ref.blob("f.body." + name)
        for rid, h in zip(rids, hs):
            assert _bits(mine[w.body_index(h)]) == _bits(theirs[ref.body_index(rid)]), (name, rid)
    cmap = _collider_map(ref, w, rids, hs, "f.")
    assert len(cmap) == sum(len(b[3]) for b in BODIES)
    for f, name in COL_FIELDS:
        mine, theirs = w.read(f), ref.blob("f.col." + name)
        for c, rc in cmap.items():
            assert _bits(mine[c]) == _bits(theirs[rc]), (name, c)
    assert w.counters()["status"] == 0
    ref.close()


def test_compound_bodies_land_like_the_reference():
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    poses = [(12.0 * k - 24.0, 2.6, 0.0, 0.0) for k in range(len(BODIES))]
    ref, w, rids, hs = _build({"floor": True, "poses": poses})
    landed = set()
    compared = 0
    for step in range(1, 241):
        ref.update(1)
        w.step(1)
        if len(landed) == len(BODIES):
            continue
        # The step a body first touches the floor: its manifolds come from its free flight alone.
        ref.dump_state("l.")
        cmap = _collider_map(ref, w, rids, hs, "l.")
        body_of = {c: int(b) for c, b in enumerate(w.read(ag2d.COL_BODY))}
        which = {w.body_index(h): k for k, h in enumerate(hs[1:])}
        m = w.read(ag2d.PREV_MANIFOLDS)
        ra, rb = ref.blob("l.man.colA"), ref.blob("l.man.colB")
        rn, rd = ref.blob("l.man.normal").reshape(-1, 2), ref.blob("l.man.depth")
        rp, rc = ref.blob("l.man.points").reshape(-1, 4), ref.blob("l.man.count")
        rid_ = ref.blob("l.man.ids").reshape(-1, 2)
        index = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(ra, rb))}
        touching = {which[body_of[int(c)]] for c in np.concatenate([m["a"], m["b"]]) if body_of[int(c)] in which}
        new = touching - landed
        for rec in m:
            bodies = {which.get(body_of[int(rec["a"])]), which.get(body_of[int(rec["b"])])}
            if not bodies & new:
                continue
            k = index[(cmap[int(rec["a"])], cmap[int(rec["b"])])]
            n = int(rec["count"])
            assert n == int(rc[k])
            assert _bits([rec["nx"], rec["ny"], rec["depth"]]).tolist() == _bits([*rn[k], rd[k]]).tolist()
            pts = np.array([rec["px0"], rec["py0"], rec["px1"], rec["py1"]], np.float32)[:2 * n]
            assert _bits(pts).tolist() == _bits(rp[k][:2 * n]).tolist()
            assert [int(rec["id0"]), int(rec["id1"])][:n] == rid_[k][:n].tolist()
            compared += 1
        landed |= new
    assert landed == set(range(len(BODIES))) and compared >= len(BODIES)
    # After 240 steps every body rests on the floor at the reference's height.
    ref.dump_state("s.")
    cy, ry, vy = w.read(ag2d.BODY_COM_Y), ref.blob("s.body.comY"), w.read(ag2d.BODY_VEL_Y)
    for rid, h in zip(rids[1:], hs[1:]):
        assert abs(float(cy[w.body_index(h)]) - float(ry[ref.body_index(rid)])) < 1e-3, rid
        assert abs(float(vy[w.body_index(h)])) < 0.05
    assert w.counters()["status"] == 0
    ref.close()


def test_body_and_collider_setters_match_the_reference():
    """ObjectAPI's remaining setters in free flight (ObjectAPI.h:82-91): a body's local centre of mass moved, its
    inertia recomputed from its colliders, its mass set from a density; a collider's offset, rotation and material,
    a circle's radius, a box's size, a capsule's shape and two polygons' outlines changed (ObjectAPI.h:93; refused
    outlines refused on both sides). In each of the 30 steps after the edits every body field and every collider's
    pose and AABB equal the reference's bit for bit."""
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    poses = [(12.0 * k, 20.0 + 3.0 * k, 0.3 * k, 1.5 - 0.7 * k) for k in range(len(BODIES))]
    ref, w, rids, hs = _build({"floor": False, "poses": poses})
    ref.update(20)
    w.step(20)
    ref.dump_state("c.")
    cmap = _collider_map(ref, w, rids, hs, "c.")
    body_of = w.read(ag2d.COL_BODY)
    cols = {k: [c for c in range(body_of.size) if body_of[c] == w.body_index(h)] for k, h in enumerate(hs)}
    # Body commands (kinds 6-8 of agref_set_body).
    w.set_body_local_center_of_mass(hs[0], 0.3, -0.1)
    ref.set_body(rids[0], 6, 0.3, -0.1)
    w.recompute_body_inertia(hs[1])
    ref.set_body(rids[1], 7, 0.0)
    w.set_body_mass_from_density(hs[2], 1.7)
    ref.set_body(rids[2], 8, 1.7)
    w.recompute_body_inertia(hs[4])
    ref.set_body(rids[4], 7, 0.0)
    # Collider commands on the collider at the same place on both sides.
    edits = [(cols[0][0], ag2d.COMMAND_CIRCLE_RADIUS, 3, 0.6, 0.0),      # body 0: circle
             (cols[0][2], ag2d.COMMAND_BOX_SIZE, 4, 2.5, 0.3),           # body 0: bar
             (cols[2][0], ag2d.COMMAND_CAPSULE_SHAPE, 5, 2.0, 0.25),     # body 2: capsule
             (cols[3][1], ag2d.COMMAND_COLLIDER_OFFSET, 0, 0.2, 1.4),    # body 3: one plate
             (cols[3][2], ag2d.COMMAND_COLLIDER_ROTATION, 1, -7.0, 0.0),
             (cols[4][1], ag2d.COMMAND_COLLIDER_MATERIAL, 2, 0.0, 0.0),
             (cols[1][0], ag2d.COMMAND_CIRCLE_RADIUS, 3, 9.0, 0.0)]     # a box: no effect on either side
    for c, ours, theirs, a, b in edits:
        w.set_collider(c, ours, a, b)
        ref.set_collider(cmap[c], theirs, a, b)
    # Polygon outlines (setPolygonShape): off-centre ones, so the recentring shift goes into the offset (rotated by
    # the collider's local rotation on body 2); on a circle nothing happens; refused outlines queue nothing.
    quad = [(0.2, 0.1), (1.4, 0.3), (1.2, 1.2), (0.1, 0.9)]
    penta = [(0.5 + 0.8 * np.cos(t), -0.2 + 0.8 * np.sin(t)) for t in np.arange(5) * 2 * np.pi / 5]
    for c, xy in ((cols[2][1], quad), (cols[4][0], penta), (cols[0][1], quad)):
        assert w.set_polygon_shape(c, xy) and ref.set_polygon(cmap[c], xy)
    concave = [(0.0, 0.0), (2.0, 0.0), (1.0, 0.3), (2.0, 1.0), (0.0, 1.0)]
    many = [(np.cos(t), np.sin(t)) for t in np.arange(17) * 2 * np.pi / 17]
    for xy in (concave, many, [(0.0, 0.0), (1.0, 0.0)], [(0.0, 0.0), (1.0, 0.0), (2.0, 0.0)]):
        assert not w.set_polygon_shape(cols[4][0], xy) and not ref.set_polygon(cmap[cols[4][0]], xy)
    w.recompute_body_inertia(hs[3])    # after its collider moved
    ref.set_body(rids[3], 7, 0.0)
    for step in range(30):
        ref.update(1)
        w.step(1)
        ref.dump_state("f.")
        for f, name in BODY_FIELDS:
            mine, theirs = w.read(f), ref.blob("f.body." + name)
            for rid, h in zip(rids, hs):
                assert _bits(mine[w.body_index(h)]) == _bits(theirs[ref.body_index(rid)]), (step, name, rid)
        cmap = _collider_map(ref, w, rids, hs, "f.")
        for f, name in COL_FIELDS:
            mine, theirs = w.read(f), ref.blob("f.col." + name)
            for c, rc in cmap.items():
                assert _bits(mine[c]) == _bits(theirs[rc]), (step, name, c)
    assert w.counters()["status"] == 0
    ref.close()


COMB = [(0.0, 0.0), (2.4, 0.0), (2.4, 1.2), (2.0, 1.2), (2.0, 0.4), (1.4, 0.4), (1.4, 1.2), (1.0, 1.2), (1.0, 0.4),
        (0.4, 0.4), (0.4, 1.2), (0.0, 1.2)]
NOTCH = [(0.0, 0.0), (2.0, 0.0), (2.0, 1.5), (1.0, 0.6), (0.0, 1.5)]
RING = [(1.6 * np.cos(t), 1.6 * np.sin(t)) for t in np.arange(24) * 2 * np.pi / 24]   # convex, above 16 vertices
CONCAVE_BODIES = [
    (2.0, 1.5, (0.0, 0.0), [(POLYGON, (0.2, 0.1), 0.4, dict(vertices=COMB))]),
    (3.0, 2.0, (0.1, 0.0), [(POLYGON, (-0.5, 0.0), 0.0, dict(vertices=NOTCH)),
                            (CIRCLE, (1.5, 0.0), 0.0, dict(radius=0.3))]),
    (4.0, 5.0, (0.0, 0.0), [(POLYGON, (0.0, 0.0), 0.0, dict(vertices=RING))]),
]


def test_concave_and_large_polygon_colliders_match_the_reference():
    """Concave outlines and a 24-vertex convex outline as colliders (createPolygonCollider, ObjectManager.cpp:141-195):
    split into the reference's convex pieces, one collider each (Bayazit, fan split above 16 vertices); in each of
    30 free-flight steps every body field and every piece's pose and AABB equal the reference's bit for bit."""
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    poses = [(10.0 * k, 30.0, 0.5 * k, 1.0 - 0.9 * k) for k in range(len(CONCAVE_BODIES))]
    ref, w, rids, hs = _build({"floor": False, "poses": poses, "bodies": CONCAVE_BODIES})
    ref.dump_state("p.")
    cmap = _collider_map(ref, w, rids, hs, "p.")
    body_of = w.read(ag2d.COL_BODY)
    per_body = [int(np.sum(body_of == w.body_index(h))) for h in hs]
    assert per_body[0] >= 3 and per_body[1] >= 3 and per_body[2] == 2, per_body
    for step in range(30):
        ref.update(1)
        w.step(1)
        ref.dump_state("f.")
        for f, name in BODY_FIELDS:
            mine, theirs = w.read(f), ref.blob("f.body." + name)
            for rid, h in zip(rids, hs):
                assert _bits(mine[w.body_index(h)]) == _bits(theirs[ref.body_index(rid)]), (step, name, rid)
        for f, name in COL_FIELDS:
            mine, theirs = w.read(f), ref.blob("f.col." + name)
            for c, rc in cmap.items():
                assert _bits(mine[c]) == _bits(theirs[rc]), (step, name, c)
    assert w.counters()["status"] == 0
    ref.close()
