"""Body constraints through the C ABI (ConstraintAPI, SimulationAPIs/ConstraintAPI.h:32-105: springs, revolute joints,
motors) against the reference engine making the same calls (oracle/ref_harness.cpp: agref_create_joint).

- Free bodies (no colliders, no sleep): a pendulum chain of revolute joints hanging from a static body, a spring
  ladder, a piston on a limited prismatic joint, a carriage on a limited slider joint, motors driving some links. Every body's position, rotation and velocities equal the reference's bit for bit
  after 240 steps, and so do the motors' accumulated impulses: the level schedule solves each kind in the
  reference's dense order.
- A random constraint graph (2,000 bodies, 6,000 springs and revolute, prismatic and slider joints with and without
  limits, 300 motors, some on static bodies):
  bit-exact after 60 steps; levels run in parallel with barriers between them.
- The API: a stale body handle is refused; destroys and edits wait for the next step; destroying a body takes its
  constraints; constraints between static bodies are inactive; a batch's engine takes no constraint calls.
- Jointed worlds in one batch step exactly as each world alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from oracle import refapi  # noqa: E402

REF_KIND = {ag2d.JOINT_SPRING: 0, ag2d.JOINT_REVOLUTE: 1, ag2d.JOINT_PRISMATIC: 2, ag2d.JOINT_SLIDER: 3,
            ag2d.JOINT_MOTOR: 4}
BODY_FIELDS = [(ag2d.BODY_COM_X, "comX"), (ag2d.BODY_COM_Y, "comY"), (ag2d.BODY_VEL_X, "velocityX"),
               (ag2d.BODY_VEL_Y, "velocityY"), (ag2d.BODY_ROTATION, "rotation"),
               (ag2d.BODY_ANGULAR_VELOCITY, "angularVelocity")]
NO_SLEEP = 1.0e6


class _Scene:   # the settings RefSim reads; bodies come through create_body
    n = 0
    materials = []
    dt = 1.0 / 60.0
    velocity_iterations, position_iterations = 8, 3
    gravity = (0.0, -9.81)


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


class _Pair:
    """The reference and this library driven through the same calls."""

    def __init__(self):
        self.ref = refapi.RefSim(_Scene(), sleep_time=NO_SLEEP)
        self.w = ag2d.World(dt=_Scene.dt, gravity=_Scene.gravity, sleep_time=NO_SLEEP)
        self.slots, self.handles = [], []
        # A static box far below, so that each world has a collider (the constrained bodies have none).
        self.ref.add_collider(self.ref.create_body(0.0, -1000.0, mass=0.0, inertia=0.0), 1, width=10.0, height=1.0)
        self.w.add_collider(self.w.create_body(0.0, -1000.0, mass=0.0, inertia=0.0), 1, width=10.0, height=1.0)

    def body(self, x, y, mass=1.0, inertia=0.2, rotation=0.0, vx=0.0, vy=0.0, w=0.0):
        self.slots.append(self.ref.create_body(x, y, rotation=rotation, vx=vx, vy=vy, w=w, mass=mass,
                                               inertia=inertia if mass > 0 else 0.0))
        self.handles.append(self.w.create_body(x, y, rotation=rotation, vx=vx, vy=vy, w=w, mass=mass,
                                               inertia=inertia if mass > 0 else 0.0))
        return len(self.slots) - 1

    def joint(self, kind, a, b=None, anchor_a=(0.0, 0.0), anchor_b=(0.0, 0.0), rest=0.0, k=0.0, c=0.0, speed=0.0,
              torque=0.0, axis=(1.0, 0.0), limits=(0.0, 0.0), enable_limit=False):
        if kind == ag2d.JOINT_SPRING:
            p = [*anchor_a, *anchor_b, rest, k, c]
        elif kind == ag2d.JOINT_REVOLUTE:
            p = [*anchor_a, *anchor_b, k, c]
        elif kind in (ag2d.JOINT_PRISMATIC, ag2d.JOINT_SLIDER):
            p = [*anchor_a, *anchor_b, *axis, k, c, *limits, 1.0 if enable_limit else 0.0]
        else:
            p = [speed, torque]
        slot = self.ref.body_slots   # create_body returns an index into it
        sb = slot[self.slots[b]] if b is not None else 0
        assert self.ref.create_joint(REF_KIND[kind], slot[self.slots[a]], sb, p) >= 0
        return self.w.create_joint(kind, self.handles[a], self.handles[b] if b is not None else 0, anchor_a,
                                   anchor_b, rest, k, c, speed, torque, axis, limits, enable_limit)

    def step(self, n):
        self.ref.update(n)
        self.w.step(n)

    def assert_bodies_equal(self):
        self.ref.dump_state("j.")
        ours = {f: self.w.read(f) for f, _ in BODY_FIELDS}
        for f, name in BODY_FIELDS:
            theirs = self.ref.blob("j.body." + name)
            mine = np.array([ours[f][self.w.body_index(h)] for h in self.handles], np.float32)
            want = np.array([theirs[self.ref.body_index(s)] for s in self.slots], np.float32)
            bad = np.nonzero(_bits(mine) != _bits(want))[0]
            assert bad.size == 0, (name, bad[:5], mine[bad[:5]], want[bad[:5]])

    def close(self):
        self.ref.close()
        self.w.close()


@pytest.fixture
def pair():
    if not refapi.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    p = _Pair()
    yield p
    p.close()


def test_chain_ladder_and_motors_match_the_reference_bit_for_bit(pair):
    anchor = pair.body(0.0, 20.0, mass=0.0)
    prev = anchor
    links = []
    for k in range(12):   # a pendulum chain starting horizontal
        b = pair.body(1.0 + k, 20.0, mass=1.0 + 0.1 * k, inertia=0.1)
        pair.joint(ag2d.JOINT_REVOLUTE, prev, b, (0.5, 0.0) if prev != anchor else (0.0, 0.0), (-0.5, 0.0),
                   k=5.0e4, c=50.0)
        links.append(b)
        prev = b
    rails = [pair.body(30.0 + 1.5 * k, 10.0, mass=2.0, inertia=0.4, vx=0.3 * k) for k in range(8)]
    rails2 = [pair.body(30.0 + 1.5 * k, 8.0, mass=1.0, inertia=0.3, w=0.2) for k in range(8)]
    top = pair.body(40.0, 14.0, mass=0.0)
    for a, b in zip(rails, rails[1:]):
        pair.joint(ag2d.JOINT_SPRING, a, b, (0.2, 0.1), (-0.2, 0.0), rest=1.4, k=300.0, c=4.0)
    for a, b in zip(rails, rails2):
        pair.joint(ag2d.JOINT_SPRING, a, b, (0.0, -0.1), (0.0, 0.1), rest=2.0, k=800.0, c=10.0)
    pair.joint(ag2d.JOINT_SPRING, top, rails[3], (0.0, 0.0), (0.0, 0.2), rest=3.0, k=2000.0, c=30.0)
    # A piston on a prismatic joint (limits hit while it falls) and a slider carriage on a tilted static rail.
    base = pair.body(60.0, 12.0, mass=0.0, rotation=0.2)
    piston = pair.body(60.5, 12.0, mass=1.5, inertia=0.3, rotation=0.5, w=1.0)
    pair.joint(ag2d.JOINT_PRISMATIC, base, piston, (0.2, 0.0), (0.0, 0.1), k=2.0e4, c=40.0, axis=(1.0, 2.0),
               limits=(-1.5, 0.5), enable_limit=True)
    rail = pair.body(80.0, 12.0, mass=0.0, rotation=-0.4)
    carriage = pair.body(81.0, 12.5, mass=2.0, inertia=0.5, vx=1.0)
    pair.joint(ag2d.JOINT_SLIDER, rail, carriage, (0.0, 0.0), (0.0, -0.2), k=1.0e4, c=20.0, axis=(3.0, 0.5),
               limits=(-4.0, 2.0), enable_limit=True)
    tail = pair.body(82.0, 11.0, mass=0.5, inertia=0.1)
    pair.joint(ag2d.JOINT_PRISMATIC, carriage, tail, (0.3, 0.0), (0.0, 0.0), k=5.0e3, c=5.0, axis=(0.0, 1.0))
    motors = [pair.joint(ag2d.JOINT_MOTOR, b, speed=2.0 - 0.5 * i, torque=5.0 + i) for i, b in
              enumerate(links[::3] + rails2[::2] + [piston])]
    for _ in range(4):
        pair.step(60)
        pair.assert_bodies_equal()
    imp, slot = pair.ref.motor_impulses()
    index_of_slot = {sl: i for i, sl in enumerate(pair.ref.body_slots)}
    ours = {pair.w.body_index(pair.handles[pair.slots.index(index_of_slot[s])]): v
            for s, v in zip(slot.tolist(), imp.tolist())}
    for h in motors:
        d = pair.w.joint(ag2d.JOINT_MOTOR, h)
        b = pair.w.body_index(d["body_a"])
        assert _bits([d["impulse"]])[0] == _bits([ours[b]])[0]
    assert pair.w.counters()["status"] == 0


def test_random_constraint_graph_matches_the_reference(pair):
    rng = np.random.default_rng(3)
    n = 2000
    for i in range(n):
        static = i % 50 == 0
        pair.body(float(rng.uniform(-50, 50)), float(rng.uniform(0, 100)), mass=0.0 if static else
                  float(rng.uniform(0.5, 3.0)), inertia=float(rng.uniform(0.05, 1.0)),
                  vx=float(rng.normal(0, 1)), vy=float(rng.normal(0, 1)), w=float(rng.normal(0, 0.5)))
    for j in range(6000):
        a, b = rng.choice(n, 2, replace=False).tolist()
        anchors = (tuple(rng.uniform(-0.5, 0.5, 2).tolist()), tuple(rng.uniform(-0.5, 0.5, 2).tolist()))
        if j % 4 == 0:
            pair.joint(ag2d.JOINT_SPRING, a, b, *anchors, rest=float(rng.uniform(0.5, 5.0)),
                       k=float(rng.uniform(10, 200)), c=float(rng.uniform(0.5, 5.0)))
        elif j % 4 == 1:
            pair.joint(ag2d.JOINT_REVOLUTE, a, b, *anchors, k=float(rng.uniform(50, 500)),
                       c=float(rng.uniform(1.0, 10.0)))
        else:
            lo = float(rng.uniform(-3, 0))
            pair.joint(ag2d.JOINT_PRISMATIC if j % 4 == 2 else ag2d.JOINT_SLIDER, a, b, *anchors,
                       k=float(rng.uniform(50, 500)), c=float(rng.uniform(1.0, 10.0)),
                       axis=tuple(rng.normal(0, 1, 2).tolist()), limits=(lo, lo + float(rng.uniform(0.5, 4))),
                       enable_limit=bool(j % 3))
    for b in rng.choice(n, 300, replace=False).tolist():
        pair.joint(ag2d.JOINT_MOTOR, b, speed=float(rng.uniform(-3, 3)), torque=float(rng.uniform(0.5, 20)))
    assert pair.w.joint_count(ag2d.JOINT_SLIDER) == 1500 and pair.w.joint_count(ag2d.JOINT_MOTOR) == 300
    for _ in range(3):
        pair.step(20)
        pair.assert_bodies_equal()


def test_constraint_api(pair):
    ground = pair.body(0.0, 0.0, mass=0.0)
    ground2 = pair.body(5.0, 0.0, mass=0.0)
    a = pair.body(0.0, 5.0)
    b = pair.body(2.0, 5.0)
    w = pair.w
    s = pair.joint(ag2d.JOINT_SPRING, ground, a, rest=5.0, k=100.0, c=2.0)
    r = pair.joint(ag2d.JOINT_REVOLUTE, a, b, (1.0, 0.0), (-1.0, 0.0), k=1e4, c=10.0)
    dead = pair.joint(ag2d.JOINT_SPRING, ground, ground2, rest=1.0, k=10.0, c=1.0)   # inactive: no body moves
    m = pair.joint(ag2d.JOINT_MOTOR, b, speed=1.0, torque=2.0)
    with pytest.raises(ag2d.Ag2dError):
        w.create_joint(ag2d.JOINT_SPRING, pair.handles[a], 12345 << 32)
    d = w.joint(ag2d.JOINT_SPRING, s)
    assert (d["rest_length"], d["stiffness"], d["damping"]) == (5.0, 100.0, 2.0)
    assert w.joint(ag2d.JOINT_SPRING, dead)["body_b"] == pair.handles[ground2]
    pz = pair.joint(ag2d.JOINT_PRISMATIC, ground, a, axis=(3.0, 4.0), k=100.0, c=1.0)   # axis normalised
    dp = w.joint(ag2d.JOINT_PRISMATIC, pz)
    assert (dp["axis_x"], dp["axis_y"]) == (float(np.float32(3.0) / np.float32(5.0)),
                                            float(np.float32(4.0) / np.float32(5.0)))
    pair.step(30)
    pair.assert_bodies_equal()
    # Deferred edits: nothing changes until the next step's flush; negative values are clamped at 0.
    w.set_joint(ag2d.JOINT_SPRING, s, ag2d.JOINT_REST_LENGTH, -3.0)
    w.set_joint(ag2d.JOINT_MOTOR, m, ag2d.JOINT_TARGET_SPEED, -2.0)
    w.set_joint(ag2d.JOINT_PRISMATIC, pz, ag2d.JOINT_LIMITS, 2.0, -1.0)    # either order
    w.set_joint(ag2d.JOINT_PRISMATIC, pz, ag2d.JOINT_AXIS_A, 0.0, 0.0)     # zero length: dropped
    assert w.joint(ag2d.JOINT_SPRING, s)["rest_length"] == 5.0
    w.step(1)
    dp = w.joint(ag2d.JOINT_PRISMATIC, pz)
    assert (dp["lower_limit"], dp["upper_limit"]) == (-1.0, 2.0) and dp["axis_y"] > 0.79
    assert w.joint(ag2d.JOINT_SPRING, s)["rest_length"] == 0.0
    assert w.joint(ag2d.JOINT_MOTOR, m)["target_speed"] == -2.0
    # Deferred destroy; a stale handle is dropped when the commands are applied.
    w.destroy_joint(ag2d.JOINT_REVOLUTE, r)
    w.destroy_joint(ag2d.JOINT_REVOLUTE, r)
    assert w.joint_count(ag2d.JOINT_REVOLUTE) == 1
    w.step(1)
    assert w.joint_count(ag2d.JOINT_REVOLUTE) == 0
    with pytest.raises(ag2d.Ag2dError):
        w.joint(ag2d.JOINT_REVOLUTE, r)
    # Destroying a body takes its constraints.
    w.destroy_body(pair.handles[b])
    w.step(1)
    assert w.joint_count(ag2d.JOINT_MOTOR) == 0 and w.joint_count(ag2d.JOINT_SPRING) == 2
    assert w.joint_count(ag2d.JOINT_PRISMATIC) == 1
    # The constraint API is per world: a batch's engine takes none.
    batch = ag2d.Batch([w])
    with pytest.raises(ag2d.Ag2dError):
        batch.engine.create_joint(ag2d.JOINT_MOTOR, pair.handles[a], target_speed=1.0, max_torque=1.0)
    assert w.counters()["status"] == 0


def test_constrained_bodies_sleep_and_wake_as_one_island(pair):
    """A chain on revolute joints lying on the ground (circle colliders too small to touch each other) settles; its
    links fall asleep in the same step, as one island with the joints as links, and a ball dropped on one end wakes
    all of them in the same step. Both engines settle the chain to the same heights within 5 mm."""
    w, ref = pair.w, pair.ref
    rm, wm = ref.add_material(0.0, 0.6, 0.5), w.add_material(0.0, 0.6, 0.5)   # no bounce, friction
    ground = pair.body(0.0, -1.0, mass=0.0)
    ref.add_collider(pair.slots[ground], 1, material=rm, width=60.0, height=2.0)
    w.add_collider(pair.handles[ground], 1, material=wm, width=60.0, height=2.0)
    links = []
    for k in range(6):
        b = pair.body(-3.0 + k, 0.3, mass=1.0, inertia=0.05)
        ref.add_collider(pair.slots[b], 0, material=rm, radius=0.3)
        w.add_collider(pair.handles[b], 0, material=wm, radius=0.3)
        if links:
            pair.joint(ag2d.JOINT_REVOLUTE, links[-1], b, (0.5, 0.0), (-0.5, 0.0), k=1.0e4, c=20.0)
        links.append(b)
    w_sleep = pair.w   # the pair's worlds never sleep; this test needs a world that does
    w2 = ag2d.World(dt=_Scene.dt, gravity=_Scene.gravity)
    m2 = w2.add_material(0.0, 0.6, 0.5)
    g2 = w2.create_body(0.0, -1.0, mass=0.0, inertia=0.0)
    w2.add_collider(g2, 1, material=m2, width=60.0, height=2.0)
    hs = []
    for k in range(6):
        h = w2.create_body(-3.0 + k, 0.3, mass=1.0, inertia=0.05)
        w2.add_collider(h, 0, material=m2, radius=0.3)
        if hs:
            w2.create_joint(ag2d.JOINT_REVOLUTE, hs[-1], h, (0.5, 0.0), (-0.5, 0.0), 0.0, 1.0e4, 20.0)
        hs.append(h)
    idx = [w2.body_index(h) for h in hs]
    slept_at = None
    for step in range(1, 601):
        w2.step(1)
        st = w2.read(ag2d.BODY_STATE)[idx]
        assert len(set(st.tolist())) == 1, (step, st)   # one island: all asleep or all awake
        if st[0] == 1:
            slept_at = step
            break
    assert slept_at is not None, "the chain never fell asleep"
    ball = w2.create_body(-3.0, 3.0, vy=-4.0, mass=2.0, inertia=0.1)
    w2.add_collider(ball, 0, material=m2, radius=0.3)
    woke = False
    for _ in range(120):
        w2.step(1)
        st = w2.read(ag2d.BODY_STATE)[idx]
        assert len(set(st.tolist())) == 1, st
        if st[0] == 2:
            woke = True
            break
    assert woke, "the ball did not wake the chain"
    assert w2.counters()["status"] == 0
    w2.close()
    # The never-sleeping pair settles to the reference's heights.
    del w_sleep
    pair.step(300)
    ref.dump_state("s.")
    cy = w.read(ag2d.BODY_COM_Y)
    ry = ref.blob("s.body.comY")
    for b in links:
        assert abs(float(cy[w.body_index(pair.handles[b])]) - float(ry[ref.body_index(pair.slots[b])])) < 5e-3


def test_constraint_dense_order_and_handles_match_the_reference(pair):
    """The host's constraint tables follow the reference's: the dense order after group moves (a constraint between
    static bodies goes to the inactive group in front, by boundary swaps), handles (slot and generation) and the
    reuse of a destroyed constraint's slot (last freed first, generation raised)."""
    w, ref = pair.w, pair.ref
    statics = [pair.body(float(i), 0.0, mass=0.0) for i in range(3)]
    movers = [pair.body(float(i), 5.0) for i in range(6)]

    def same_order():
        slots, gens, _ = ref.joint_order(0)
        ours = [w.joint_handle(ag2d.JOINT_SPRING, i) for i in range(w.joint_count(ag2d.JOINT_SPRING))]
        assert [h & 0xFFFFFFFF for h in ours] == slots.tolist()
        assert [h >> 32 for h in ours] == gens.tolist()

    plan = [(statics[0], movers[0]), (statics[0], statics[1]), (movers[1], movers[2]), (statics[1], statics[2]),
            (movers[3], statics[2]), (statics[2], statics[0]), (movers[4], movers[5])]
    hs = [pair.joint(ag2d.JOINT_SPRING, a, b, rest=1.0, k=10.0, c=1.0) for a, b in plan]
    same_order()
    for h in (hs[2], hs[1], hs[5]):   # active, inactive, inactive
        w.destroy_joint(ag2d.JOINT_SPRING, h)
        ref.destroy_joint(0, h & 0xFFFFFFFF, h >> 32)
    pair.step(1)
    same_order()
    more = [pair.joint(ag2d.JOINT_SPRING, a, b, rest=1.0, k=10.0, c=1.0)
            for a, b in ((statics[1], statics[0]), (movers[2], movers[0]), (movers[5], statics[1]))]
    assert [h & 0xFFFFFFFF for h in more] == [hs[5] & 0xFFFFFFFF, hs[1] & 0xFFFFFFFF, hs[2] & 0xFFFFFFFF]
    same_order()
    pair.step(30)
    pair.assert_bodies_equal()


def _jointed_world(seed):
    """A ground box, a pile of boxes and a few jointed contraptions (chain, ladder, piston, motorised wheel)."""
    rng = np.random.default_rng(seed)
    w = ag2d.World(dt=_Scene.dt, gravity=_Scene.gravity)
    mat = w.add_material(0.1, 0.6, 0.5)
    g = w.create_body(0.0, -1.0, mass=0.0, inertia=0.0)
    w.add_collider(g, 1, material=mat, width=80.0, height=2.0)
    for i in range(int(rng.integers(10, 40))):
        b = w.create_body(float(rng.uniform(-20, 20)), float(rng.uniform(1, 15)), mass=1.0, inertia=0.2)
        w.add_collider(b, 1, material=mat, width=0.8, height=0.8)
    hook = w.create_body(float(rng.uniform(-10, 10)), 20.0, mass=0.0, inertia=0.0)
    prev = hook
    for k in range(int(rng.integers(3, 9))):
        b = w.create_body(w.read(ag2d.BODY_COM_X)[w.body_index(hook)] + 1.0 + k, 20.0, mass=1.0, inertia=0.1)
        w.create_joint(ag2d.JOINT_REVOLUTE, prev, b, (0.5, 0.0) if prev != hook else (0.0, 0.0), (-0.5, 0.0), 0.0,
                       2.0e4, 30.0)
        prev = b
    w.create_joint(ag2d.JOINT_MOTOR, prev, 0, target_speed=float(rng.uniform(-3, 3)), max_torque=8.0)
    a = w.create_body(-25.0, 6.0, mass=2.0, inertia=0.5)
    b = w.create_body(-23.0, 6.0, mass=1.0, inertia=0.3)
    w.add_collider(a, 0, material=mat, radius=0.5)
    w.add_collider(b, 0, material=mat, radius=0.5)
    w.create_joint(ag2d.JOINT_SPRING, a, b, (0.2, 0.0), (-0.2, 0.0), 1.8, 400.0, 5.0)
    w.create_joint(ag2d.JOINT_SLIDER, g, a, (-25.0, 1.0), (0.0, 0.0), 0.0, 5.0e3, 20.0, axis=(0.0, 1.0),
                   limits=(2.0, 8.0), enable_limit=True)
    w.create_joint(ag2d.JOINT_PRISMATIC, a, b, (0.0, 0.0), (0.0, 0.0), 0.0, 3.0e3, 10.0, axis=(1.0, 0.2))
    return w


def test_batched_jointed_worlds_match_each_world_alone():
    """Worlds with body constraints in one batch step exactly as each world alone: the constraints of every world
    keep their order in the batch's tables and the level schedule never mixes worlds' bodies."""
    alone = [_jointed_world(s) for s in range(5)]
    batch = ag2d.Batch([_jointed_world(s) for s in range(5)])
    for w in alone:
        w.step(150)
    batch.step(150)
    for k, w in enumerate(alone):
        for f, _ in BODY_FIELDS:
            assert np.array_equal(_bits(batch.read(k, f)), _bits(w.read(f))), (k, f)
    assert batch.counters()["status"] == 0
    with pytest.raises(ag2d.Ag2dError):
        batch.save()   # checkpoints hold no body constraints
