"""Seeded synthetic scenes for the five workloads of the collision/contact pipeline.

The reference publishes no scenes or datasets; these generators stand in for its demo scenes
(App/Scenes.cpp: load_LargeWorld, load_StackedPyramid, makeConvexPolygon) with the shapes, sizes and value
distributions each workload names. A scene is a flat, numpy-backed body list that both this library and the
reference engine can be loaded from, so every comparison starts from bit-identical inputs.

Shape codes follow the reference's ColliderShapeType (PS_AGONY2D/Types/Types.h:35-42): 0 circle, 1 box, 2 polygon,
3 capsule.
Mass 0 means a static body (ObjectManager::appendBody, PS_AGONY2D/SimulationImpl/ObjectManager.cpp:1285).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

CIRCLE, BOX, POLYGON, CAPSULE = 0, 1, 2, 3


@dataclasses.dataclass
class Scene:
    """Bodies with one collider each, in creation order.

    Arrays are float32 unless noted. Polygon vertices are body-local, CCW, in a CSR layout
    (poly_offset[i] .. poly_offset[i] + poly_count[i] into poly_xy), indexed by body for polygon bodies.
    """
    kind: np.ndarray          # uint8 shape code per body
    px: np.ndarray
    py: np.ndarray
    rot: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    w: np.ndarray
    mass: np.ndarray          # 0 = static
    radius: np.ndarray        # circles and capsules
    width: np.ndarray         # boxes (full size); capsules: core length (end cap centre to end cap centre)
    height: np.ndarray
    poly_offset: np.ndarray   # int64, polygons
    poly_count: np.ndarray    # int32, polygons
    poly_xy: np.ndarray       # float32 [V, 2]
    material: np.ndarray      # uint32 index into materials
    materials: list           # [(elasticity, static friction, dynamic friction)]
    dt: float = 1.0 / 60.0
    velocity_iterations: int = 8
    position_iterations: int = 3
    gravity: tuple = (0.0, -9.81)
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.kind.shape[0])

    def polygon_vertices(self, i: int) -> np.ndarray:
        o, c = int(self.poly_offset[i]), int(self.poly_count[i])
        return self.poly_xy[o:o + c]


class _Builder:
    def __init__(self, materials):
        self.materials = list(materials)
        self.rows = []
        self.poly = []

    def add(self, kind, px, py, rot=0.0, vx=0.0, vy=0.0, w=0.0, mass=0.0, radius=0.0, width=0.0, height=0.0,
            verts=None, material=1):
        self.rows.append((kind, px, py, rot, vx, vy, w, mass, radius, width, height, material))
        self.poly.append(None if verts is None else np.asarray(verts, dtype=np.float32).reshape(-1, 2))

    def build(self, name, **kw) -> Scene:
        n = len(self.rows)
        cols = list(zip(*self.rows)) if n else [[] for _ in range(12)]
        f32 = lambda c: np.asarray(c, dtype=np.float32)
        counts = np.array([0 if p is None else p.shape[0] for p in self.poly], dtype=np.int32)
        offsets = np.zeros(n, dtype=np.int64)
        if n:
            offsets[1:] = np.cumsum(counts[:-1])
        xy = np.concatenate([p for p in self.poly if p is not None], axis=0) if any(
            p is not None for p in self.poly) else np.zeros((0, 2), np.float32)
        return Scene(kind=np.asarray(cols[0], dtype=np.uint8), px=f32(cols[1]), py=f32(cols[2]), rot=f32(cols[3]),
                     vx=f32(cols[4]), vy=f32(cols[5]), w=f32(cols[6]), mass=f32(cols[7]), radius=f32(cols[8]),
                     width=f32(cols[9]), height=f32(cols[10]), poly_offset=offsets, poly_count=counts,
                     poly_xy=xy.astype(np.float32), material=np.asarray(cols[11], dtype=np.uint32),
                     materials=self.materials, name=name, **kw)


def polygon_on_circle(rng: np.random.Generator, radius: float, n_min: int = 3, n_max: int = 8,
                      jitter: float = 0.15) -> np.ndarray:
    """Convex-ish polygon: n vertices evenly spaced on a circle, each radius jittered by +-jitter (CCW).

    Same construction as the reference demo's convex polygon maker (App/Scenes.cpp:29-77): evenly spaced
    angles with a random phase and a per-vertex radial jitter.
    """
    nv = int(rng.integers(n_min, n_max + 1))
    phase = rng.uniform(0.0, 2.0 * math.pi / nv)
    ang = phase + 2.0 * math.pi * np.arange(nv) / nv
    r = radius * rng.uniform(1.0 - jitter, 1.0 + jitter, nv)
    return np.stack([r * np.cos(ang), r * np.sin(ang)], axis=1).astype(np.float32)


def polygon_area(xy: np.ndarray) -> float:
    x, y = xy[:, 0].astype(np.float64), xy[:, 1].astype(np.float64)
    return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


FRICTION_MATERIAL = (0.0, 0.4, 0.4)   # restitution 0, static = dynamic friction 0.4


def make_c1(n: int = 2048, seed: int = 0, width: float = 200.0, height: float = 100.0) -> Scene:
    """Plain single world: n convex 3-8-gons (radius U[0.5,2], +-15% radial jitter, density 1) uniform in a
    width x height region above a static 220 m x 2 m ground box whose top is y = 0. Zero initial velocity."""
    rng = np.random.default_rng(seed)
    b = _Builder([FRICTION_MATERIAL])
    b.add(BOX, 0.0, -1.0, width=220.0, height=2.0, mass=0.0, material=1)
    for _ in range(n):
        R = rng.uniform(0.5, 2.0)
        verts = polygon_on_circle(rng, R)
        x = rng.uniform(-0.5 * width, 0.5 * width)
        y = rng.uniform(2.5, 2.5 + height)
        b.add(POLYGON, x, y, mass=polygon_area(verts), verts=verts, material=1)
    return b.build(f"c1_n{n}_s{seed}")


def make_c2(n: int = 100_000, seed: int = 0, columns: int = 500, cell: float = 4.8) -> Scene:
    """Single large world: n mixed bodies (60% boxes side U[0.3,1.5], 25% circles r U[0.2,1], 15% 3-8-gons from
    the c1 generator) placed one per cell of a columns-wide grid (rows = n / columns) above the floor of a static
    U-shaped container (three boxes). Density 1, zero initial velocity."""
    rng = np.random.default_rng(seed)
    b = _Builder([FRICTION_MATERIAL])
    rows = (n + columns - 1) // columns
    inner = columns * cell
    wall_h = rows * cell + 20.0
    b.add(BOX, 0.0, -1.0, width=inner + 4.0, height=2.0, mass=0.0, material=1)
    b.add(BOX, -0.5 * inner - 1.0, 0.5 * wall_h, width=2.0, height=wall_h, mass=0.0, material=1)
    b.add(BOX, 0.5 * inner + 1.0, 0.5 * wall_h, width=2.0, height=wall_h, mass=0.0, material=1)
    kinds = rng.random(n)
    for i in range(n):
        col, row = i % columns, i // columns
        x = -0.5 * inner + (col + 0.5) * cell
        y = 0.5 * cell + row * cell
        u = kinds[i]
        if u < 0.60:
            s = rng.uniform(0.3, 1.5)
            b.add(BOX, x, y, width=s, height=s, mass=s * s, material=1)
        elif u < 0.85:
            r = rng.uniform(0.2, 1.0)
            b.add(CIRCLE, x, y, radius=r, mass=math.pi * r * r, material=1)
        else:
            verts = polygon_on_circle(rng, rng.uniform(0.5, 2.0))
            b.add(POLYGON, x, y, mass=polygon_area(verts), verts=verts, material=1)
    return b.build(f"c2_n{n}_s{seed}")


def make_capsule_mix(n: int = 1500, seed: int = 0, columns: int = 40, cell: float = 4.8) -> Scene:
    """Every shape pair, capsules included: n bodies (30% capsules of core length U[0.4,2.4] m and radius
    U[0.15,0.6] m at random rotations, 25% boxes side U[0.3,1.5], 20% circles r U[0.2,1], 25% 3-8-gons from the c1
    generator), one per cell of a columns-wide grid above the floor of a static U container, density 1."""
    rng = np.random.default_rng(seed)
    b = _Builder([FRICTION_MATERIAL])
    rows = (n + columns - 1) // columns
    inner = columns * cell
    wall_h = rows * cell + 20.0
    b.add(BOX, 0.0, -1.0, width=inner + 4.0, height=2.0, mass=0.0, material=1)
    b.add(BOX, -0.5 * inner - 1.0, 0.5 * wall_h, width=2.0, height=wall_h, mass=0.0, material=1)
    b.add(BOX, 0.5 * inner + 1.0, 0.5 * wall_h, width=2.0, height=wall_h, mass=0.0, material=1)
    kinds = rng.random(n)
    for i in range(n):
        col, row = i % columns, i // columns
        x = -0.5 * inner + (col + 0.5) * cell
        y = 0.5 * cell + row * cell
        u = kinds[i]
        if u < 0.30:
            length, r = rng.uniform(0.4, 2.4), rng.uniform(0.15, 0.6)
            b.add(CAPSULE, x, y, rot=rng.uniform(0.0, math.pi), radius=r, width=length,
                  mass=length * 2.0 * r + math.pi * r * r, material=1)
        elif u < 0.55:
            s = rng.uniform(0.3, 1.5)
            b.add(BOX, x, y, width=s, height=s, mass=s * s, material=1)
        elif u < 0.75:
            r = rng.uniform(0.2, 1.0)
            b.add(CIRCLE, x, y, radius=r, mass=math.pi * r * r, material=1)
        else:
            verts = polygon_on_circle(rng, rng.uniform(0.5, 2.0))
            b.add(POLYGON, x, y, mass=polygon_area(verts), verts=verts, material=1)
    return b.build(f"capmix_n{n}_s{seed}")


def make_towers(towers: int = 40, levels: int = 3, drops: int = 12, seed: int = 0, spacing: float = 3.0,
                drop_height: float = 30.0, group: int = 4) -> Scene:
    """Sleep and wake: `towers` stacks of `levels` boxes (side U[0.8,1.0]) on a static ground, 3 m apart, each its
    own island that falls asleep after settling; `drops` circles (r U[0.3,0.5]) fall onto every third tower from
    drop_height + 8 m x (k // group), so `group` islands wake in the same step, with their stored manifolds."""
    rng = np.random.default_rng(seed)
    b = _Builder([FRICTION_MATERIAL])
    width = towers * spacing + 10.0
    b.add(BOX, 0.0, -1.0, width=width, height=2.0, mass=0.0, material=1)
    x0 = -0.5 * (towers - 1) * spacing
    for t in range(towers):
        y = 0.0
        for _ in range(levels):
            s = rng.uniform(0.8, 1.0)
            b.add(BOX, x0 + t * spacing + rng.uniform(-0.05, 0.05), y + 0.5 * s + 0.005, width=s, height=s,
                  mass=s * s, material=1)
            y += s + 0.01
    for k in range(drops):
        t = (3 * k) % towers
        r = rng.uniform(0.3, 0.5)
        b.add(CIRCLE, x0 + t * spacing + rng.uniform(-0.2, 0.2), drop_height + 8.0 * (k // group), radius=r,
              mass=math.pi * r * r, material=1)
    return b.build(f"towers_{towers}x{levels}_s{seed}")


def make_c3(n: int = 1_000_000, seed: int = 0, extent: float = 4000.0) -> Scene:
    """Broad+narrow stress: n bodies, 50% circles / 50% 4-6-gons, size (radius) log-uniform in [0.1, 2] m,
    uniform in an extent x extent box, velocities N(0, 5 m/s), no gravity, no static bodies.
    """
    rng = np.random.default_rng(seed)
    b = _Builder([FRICTION_MATERIAL])
    size = np.exp(rng.uniform(math.log(0.1), math.log(2.0), n))
    xs = rng.uniform(-0.5 * extent, 0.5 * extent, n)
    ys = rng.uniform(-0.5 * extent, 0.5 * extent, n)
    vel = rng.normal(0.0, 5.0, (n, 2))
    kinds = rng.random(n)
    for i in range(n):
        if kinds[i] < 0.5:
            r = float(size[i])
            b.add(CIRCLE, xs[i], ys[i], vx=vel[i, 0], vy=vel[i, 1], radius=r, mass=math.pi * r * r, material=1)
        else:
            verts = polygon_on_circle(rng, float(size[i]), 4, 6)
            b.add(POLYGON, xs[i], ys[i], vx=vel[i, 0], vy=vel[i, 1], mass=polygon_area(verts), verts=verts,
                  material=1)
    return b.build(f"c3_n{n}_s{seed}", gravity=(0.0, 0.0))


def log_uniform_counts(rng: np.random.Generator, count: int, lo: int, hi: int) -> np.ndarray:
    return np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), count))).astype(np.int64).clip(lo, hi)


def _c4_world(args):
    count, world_seed = args
    scale = math.sqrt(count / 2048.0)
    return make_c1(int(count), world_seed, width=max(20.0, 200.0 * scale), height=max(10.0, 100.0 * scale))


def c4_counts(worlds: int = 4096, seed: int = 0, lo: int = 16, hi: int = 2048) -> np.ndarray:
    """Body counts of the batched-worlds workload: log-uniform in [lo, hi], one draw per world."""
    return log_uniform_counts(np.random.default_rng(seed), worlds, lo, hi)


def shard_by_bodies(counts, ranks: int) -> list:
    """Greedy body-count balancing of independent worlds over ranks: worlds largest first (ties: lower index), each
    to the rank with the fewest bodies so far (ties: lower rank). Returns each rank's world indices, ascending. The
    loads differ by at most the largest world's count."""
    counts = np.asarray(counts, dtype=np.int64)
    order = sorted(range(counts.size), key=lambda k: (-int(counts[k]), k))
    load = [0] * ranks
    out = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda j: (load[j], j))
        out[r].append(k)
        load[r] += int(counts[k])
    return [sorted(x) for x in out]


def make_c4_worlds(worlds: int = 4096, seed: int = 0, lo: int = 16, hi: int = 2048, processes: int = 1,
                   subset=None) -> list:
    """Batched worlds: body counts log-uniform in [lo, hi]; world k is make_c1(count_k, seed + k) (c1 shape mix,
    own ground box), with the region scaled so the body density matches c1 (2048 bodies in 200 x 100 m).
    subset: only these world indices (in that order), e.g. one rank's shard_by_bodies share of the job.
    processes > 1 generates the worlds in a spawned process pool (same worlds: each has its own seed)."""
    counts = c4_counts(worlds, seed, lo, hi)
    ks = range(worlds) if subset is None else list(subset)
    jobs = [(int(counts[k]), seed + k) for k in ks]
    worlds = len(jobs)
    if processes > 1 and worlds > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(processes) as pool:
            return pool.map(_c4_world, jobs, chunksize=max(1, worlds // (4 * processes)))
    return [_c4_world(j) for j in jobs]


def _c5_world(args):
    request_id, count, seed = args
    scale = math.sqrt(count / 2048.0)
    base = make_c1(count, seed, width=max(20.0, 200.0 * scale), height=max(10.0, 100.0 * scale))
    r2 = np.random.default_rng(seed ^ 0x5EED)
    fast = r2.random(base.n) < 0.05
    fast[0] = False   # ground stays a box
    for i in np.nonzero(fast)[0]:
        base.kind[i] = CIRCLE
        base.radius[i] = 0.05
        base.mass[i] = math.pi * 0.05 * 0.05
        ang = r2.uniform(-math.pi * 0.75, -math.pi * 0.25)
        base.vx[i] = 200.0 * math.cos(ang)
        base.vy[i] = 200.0 * math.sin(ang)
        base.poly_count[i] = 0
    base.name = f"c5_req{request_id}_n{count}"
    return base


def make_c5_request(rng: np.random.Generator, request_id: int, lo: int = 32, hi: int = 8192) -> Scene:
    """Serving request: a world of log-uniform [lo, hi] bodies in the c1 mix, of which 5% are small fast
    circles (r = 0.05 m) moving at 200 m/s towards the ground (continuous collision detection exercise)."""
    count = int(log_uniform_counts(rng, 1, lo, hi)[0])
    seed = int(rng.integers(0, 2**31 - 1))
    return _c5_world((request_id, count, seed))


def make_c5_requests(requests: int, seed: int = 0, lo: int = 32, hi: int = 8192, processes: int = 1) -> list:
    """The first `requests` worlds of the serving stream with this seed (make_c5_request in order); processes > 1
    builds them in a spawned process pool (the same worlds)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(requests):
        count = int(log_uniform_counts(rng, 1, lo, hi)[0])
        jobs.append((k, count, int(rng.integers(0, 2**31 - 1))))
    if processes > 1 and requests > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(processes) as pool:
            return pool.map(_c5_world, jobs, chunksize=max(1, requests // (4 * processes)))
    return [_c5_world(j) for j in jobs]
