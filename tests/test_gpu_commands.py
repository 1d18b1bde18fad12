"""Deferred body commands (destroy, position, rotation, velocity, angular velocity, mass, inertia) through the
C ABI, against the reference engine making the same ObjectAPI calls (oracle/ref_harness.cpp: destroyBody and
setBody*, applied by its next update's flushCommands).

Scene: free-falling circles, boxes, polygons and capsules on a 10 m grid, plus static bodies, far enough apart that
nothing touches within the run, so each body's motion depends on its own state only (no solver order). After 10
steps the same commands are issued on both sides, including ones on a destroyed body's stale handle and a static
body made dynamic; after 20 more steps every live body's state is compared bit for bit, matched by handle (dense
indices differ by design: the reference pops destroyed bodies and moves bodies between groups, here they keep their
slot with a state flag).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402
from oracle import refapi  # noqa: E402

FIELDS = [(ag2d.BODY_COM_X, "comX"), (ag2d.BODY_COM_Y, "comY"), (ag2d.BODY_VEL_X, "velocityX"),
          (ag2d.BODY_VEL_Y, "velocityY"), (ag2d.BODY_ROTATION, "rotation"),
          (ag2d.BODY_ANGULAR_VELOCITY, "angularVelocity"), (ag2d.BODY_ROT_COS, "rotationCos"),
          (ag2d.BODY_ROT_SIN, "rotationSin"), (ag2d.BODY_INV_MASS, "invMass"), (ag2d.BODY_INV_INERTIA, "invInertia")]


def _scene(seed=5):
    rng = np.random.default_rng(seed)
    b = scenes._Builder([scenes.FRICTION_MATERIAL])
    for k in range(48):
        x, y = 10.0 * (k % 8), 10.0 * (k // 8)
        kind = k % 4
        if kind == 0:
            r = rng.uniform(0.3, 1.0)
            b.add(scenes.CIRCLE, x, y, radius=r, mass=np.pi * r * r, material=1)
        elif kind == 1:
            s = rng.uniform(0.5, 1.5)
            b.add(scenes.BOX, x, y, rot=rng.uniform(0, 1), width=s, height=s, mass=s * s, material=1)
        elif kind == 2:
            v = scenes.polygon_on_circle(rng, rng.uniform(0.5, 1.5))
            b.add(scenes.POLYGON, x, y, mass=scenes.polygon_area(v), verts=v, material=1)
        else:
            b.add(scenes.CAPSULE, x, y, rot=rng.uniform(0, 3), radius=0.4, width=1.2, mass=2.0, material=1)
    for k in range(4):   # static bodies, off to the side
        b.add(scenes.BOX, 200.0 + 10.0 * k, 0.0, width=2.0, height=2.0, mass=0.0, material=1)
    return b.build("commands")


# (scene body, command, a, b): the same calls on both sides, in this order.
COMMANDS = [(3, "destroy", 0, 0), (17, "destroy", 0, 0), (30, "destroy", 0, 0), (5, "position", 300.0, 300.0),
            (8, "velocity", 3.0, -2.0), (9, "angular_velocity", 0.5, 0), (12, "rotation", 1.3, 0),
            (40, "rotation", -0.7, 0), (20, "mass", 2.5, 0), (21, "mass", 0.0, 0), (49, "mass", 3.0, 0),
            (22, "inertia", 7.0, 0), (23, "position", -60.0, 40.0), (23, "velocity", 0.0, 4.0),
            (3, "velocity", 9.0, 9.0)]   # the last one names a destroyed body: dropped on both sides
REF_KIND = {"position": refapi.RefSim.SET_POSITION, "rotation": refapi.RefSim.SET_ROTATION,
            "velocity": refapi.RefSim.SET_VELOCITY, "angular_velocity": refapi.RefSim.SET_ANGULAR_VELOCITY,
            "mass": refapi.RefSim.SET_MASS, "inertia": refapi.RefSim.SET_INERTIA}


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_commands_match_the_reference():
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    sc = _scene()
    ref = refapi.RefSim(sc)
    w = ag2d.World(dt=sc.dt, gravity=sc.gravity)
    handles = w.add_scene(sc)
    ref.update(10)
    w.step(10)
    for i, kind, a, b in COMMANDS:
        h = int(handles[i])
        if kind == "destroy":
            ref.destroy_body(i)
            w.destroy_body(h)
        else:
            ref.set_body(i, REF_KIND[kind], a, b)
            if kind in ("position", "velocity"):
                getattr(w, f"set_body_{kind}")(h, a, b)
            else:
                getattr(w, f"set_body_{kind}")(h, a)
    ref.update(20)
    w.step(20)
    ref.dump_state("t.")
    ours = {f: w.read(f) for f, _ in FIELDS}
    state = w.read(ag2d.BODY_STATE)
    for i in range(sc.n):
        gi, ri = w.body_index(int(handles[i])), ref.body_index(i)
        if i in (3, 17, 30):
            assert gi == 0xFFFFFFFF and ri == 0xFFFFFFFF, i
            continue
        assert gi != 0xFFFFFFFF and ri != 0xFFFFFFFF, i
        for f, name in FIELDS:
            assert _bits(ours[f][gi]) == _bits(ref.blob("t.body." + name)[ri]), (i, name)
    assert int(np.sum(state == ag2d.STATE_DESTROYED)) == 3
    assert state[w.body_index(int(handles[21]))] == ag2d.STATE_STATIC     # mass 0: static
    assert state[w.body_index(int(handles[49]))] == ag2d.STATE_DYNAMIC    # static body given a mass
    assert w.counters()["status"] == 0
    ref.close()


def test_destroyed_bodies_leave_a_settling_pile():
    # A pile with contacts: bodies destroyed mid-run take no further part (neither integrated nor in any pair, so
    # they stay where they were), the others step on.
    sc = scenes.make_c1(256, 3, width=40.0, height=30.0)
    w = ag2d.World(dt=sc.dt, gravity=sc.gravity)
    hs = w.add_scene(sc)
    w.step(120)
    gone = [int(h) for h in hs[1:40:2]]
    for h in gone:
        w.destroy_body(h)
    w.flush_commands()
    state = w.read(ag2d.BODY_STATE)
    dead = np.nonzero(state == ag2d.STATE_DESTROYED)[0]
    assert dead.size == len(gone)
    assert all(w.body_index(h) == 0xFFFFFFFF for h in gone)
    y0 = w.read(ag2d.BODY_COM_Y)[dead].copy()
    w.step(60)
    assert w.counters()["status"] == 0
    assert np.array_equal(w.read(ag2d.BODY_COM_Y)[dead], y0)
    assert np.all(np.isfinite(w.read(ag2d.BODY_COM_Y)))
    assert int(np.sum(w.read(ag2d.BODY_STATE) == ag2d.STATE_DESTROYED)) == len(gone)
