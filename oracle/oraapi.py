"""ctypes wrapper over oracle/liboracle.so, the CPU restatement of the collision/contact pipeline.

TEST INFRASTRUCTURE ONLY (the oracle). Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, and only as the checker; the product path never imports it.

World state is exchanged as a dict of numpy arrays named like the reference engine's SoA fields
("body.comX", "col.aabbMinX", "poly.vertices", ...), the format tests/golden/ fixtures use.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_F = ctypes.POINTER(ctypes.c_float)
_U = ctypes.POINTER(ctypes.c_uint32)


class OraWorldC(ctypes.Structure):
    _fields_ = [("n_bodies", ctypes.c_uint32), ("n_colliders", ctypes.c_uint32), ("n_materials", ctypes.c_uint32),
                ("body_starts", ctypes.c_uint32 * 4), ("col_starts", ctypes.c_uint32 * 4)] + \
               [(n, _F) for n in ("comX", "comY", "velX", "velY", "rot", "angVel", "invMass", "invInertia",
                                  "rotCos", "rotSin", "wrapCount", "boundRadius", "sleepTimer")] + \
               [("islandId", _U)] + [(n, _U) for n in ("bodyIndex", "shapeType", "shapeIndex", "material")] + \
               [(n, _F) for n in ("comOffX", "comOffY", "localRot", "worldX", "worldY", "worldRot", "worldCos",
                                  "worldSin", "minX", "minY", "maxX", "maxY", "circleRadius", "boxHalfW",
                                  "boxHalfH")] + \
               [("polyOffset", _U), ("polyCount", _U)] + \
               [(n, _F) for n in ("polyVerts", "polyNormals", "matElasticity", "matStaticFriction",
                                  "matDynamicFriction")]


class Manifold(ctypes.Structure):
    _fields_ = [("a", ctypes.c_uint32), ("b", ctypes.c_uint32), ("nx", ctypes.c_float), ("ny", ctypes.c_float),
                ("depth", ctypes.c_float), ("count", ctypes.c_uint32), ("px", ctypes.c_float * 2),
                ("py", ctypes.c_float * 2), ("id", ctypes.c_uint32 * 2), ("jn", ctypes.c_float * 2),
                ("jt", ctypes.c_float * 2)]


MANIFOLD_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("nx", "<f4"), ("ny", "<f4"), ("depth", "<f4"),
                           ("count", "<u4"), ("px", "<f4", 2), ("py", "<f4", 2), ("id", "<u4", 2),
                           ("jn", "<f4", 2), ("jt", "<f4", 2)])
assert MANIFOLD_DTYPE.itemsize == ctypes.sizeof(Manifold)

EVENT_DTYPE = np.dtype([("self", "<u4"), ("other", "<u4"), ("selfBody", "<u4"), ("otherBody", "<u4"),
                        ("callback", "<u4"), ("px", "<f4"), ("py", "<f4"), ("nx", "<f4"), ("ny", "<f4"),
                        ("impulse", "<f4")])

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        W = ctypes.POINTER(OraWorldC)
        vp, u32, i64, f = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int64, ctypes.c_float
        L.ora_integrate_velocity_verlet.argtypes = [W, u32, u32, f, f, f, f]
        L.ora_wrap_body_rotations.argtypes = [W, u32, u32]
        L.ora_fastcossin_array.argtypes = [vp, vp, vp, u32]
        L.ora_body_cossin.argtypes = [W, u32, u32]
        L.ora_collider_world_positions.argtypes = [W, u32, u32]
        L.ora_collider_world_rotations.argtypes = [W, u32, u32]
        L.ora_collider_aabbs.argtypes = [W, u32, u32]
        L.ora_morton_codes.argtypes = [W, u32, u32, vp, vp]
        L.ora_sort_by_morton.argtypes = [vp, u32, u32, vp, vp]
        L.ora_broad_pairs.restype = i64
        L.ora_broad_pairs.argtypes = [W, vp, i64]
        L.ora_narrow.restype = i64
        L.ora_narrow.argtypes = [W, vp, i64, vp]
        L.ora_warm_start.argtypes = [vp, vp, vp, i64, vp, vp, vp, i64]
        L.ora_solve.argtypes = [W, vp, i64, vp, u32, u32]
        L.ora_solve_f64.argtypes = [W, vp, i64, vp, u32, u32, vp, vp, vp]
        L.ora_islands.restype = u32
        L.ora_islands.argtypes = [W, vp, i64, vp]
        L.ora_update_sleeping.argtypes = [W, vp, u32, f, f, f, vp]
        L.ora_collision_events.argtypes = [W, vp, i64, vp, vp, vp, i64]
        L.ora_collision_events.restype = i64
        _lib = L
    return _lib


DEFAULT_MATERIALS = [(1.0, 0.0, 0.0)]   # MaterialManager: index 0 is the default material (elasticity 1)


class OraWorld:
    """Owns numpy copies of one world's state and a C view of them."""

    BODY_F = {"comX": "comX", "comY": "comY", "velX": "velocityX", "velY": "velocityY", "rot": "rotation",
              "angVel": "angularVelocity", "invMass": "invMass", "invInertia": "invInertia", "rotCos": "rotationCos",
              "rotSin": "rotationSin", "wrapCount": "renderRotationWrapCount", "boundRadius": "boundRadius",
              "sleepTimer": "sleepingTimer"}
    COL_F = {"comOffX": "comOffsetX", "comOffY": "comOffsetY", "localRot": "localRotation", "worldX": "worldPosX",
             "worldY": "worldPosY", "worldRot": "worldRotation", "worldCos": "worldRotationCos",
             "worldSin": "worldRotationSin", "minX": "aabbMinX", "minY": "aabbMinY", "maxX": "aabbMaxX",
             "maxY": "aabbMaxY"}
    COL_U = {"bodyIndex": "bodyIndex", "shapeType": "shapeType", "shapeIndex": "shapeIndex",
             "material": "materialIndex"}

    def __init__(self, state: dict, prefix: str = "", materials=None, body_prefix=None):
        bp = prefix if body_prefix is None else body_prefix

        def g(k):
            # Bodies come from body_prefix; shapes never change within a step, so they may come from "pre.".
            for p in ((bp,) if k.startswith("body.") else (prefix, "pre.")):
                if p + k in state:
                    return np.array(state[p + k])
            raise KeyError(prefix + k)
        self.a = {}
        for cname, rname in self.BODY_F.items():
            self.a[cname] = np.ascontiguousarray(g("body." + rname), dtype=np.float32)
        self.a["islandId"] = np.ascontiguousarray(g("body.islandId"), dtype=np.uint32)
        for cname, rname in self.COL_F.items():
            self.a[cname] = np.ascontiguousarray(g("col." + rname), dtype=np.float32)
        for cname, rname in self.COL_U.items():
            self.a[cname] = np.ascontiguousarray(g("col." + rname), dtype=np.uint32)
        self.a["circleRadius"] = np.ascontiguousarray(g("circle.radius"), dtype=np.float32)
        self.a["boxHalfW"] = np.ascontiguousarray(g("box.halfWidth"), dtype=np.float32)
        self.a["boxHalfH"] = np.ascontiguousarray(g("box.halfHeight"), dtype=np.float32)
        counts = np.ascontiguousarray(g("poly.counts"), dtype=np.uint32)
        offs = np.zeros_like(counts)
        if counts.size:
            offs[1:] = np.cumsum(counts[:-1])
        self.a["polyCount"] = counts
        self.a["polyOffset"] = offs
        self.a["polyVerts"] = np.ascontiguousarray(g("poly.vertices"), dtype=np.float32)
        self.a["polyNormals"] = np.ascontiguousarray(g("poly.normals"), dtype=np.float32)
        mats = list(materials) if materials is not None else list(DEFAULT_MATERIALS)
        m = np.asarray(mats, dtype=np.float32).reshape(-1, 3)
        self.a["matElasticity"] = np.ascontiguousarray(m[:, 0])
        self.a["matStaticFriction"] = np.ascontiguousarray(m[:, 1])
        self.a["matDynamicFriction"] = np.ascontiguousarray(m[:, 2])
        self.body_starts = np.array(g("body.groupStarts"), dtype=np.uint32)
        self.col_starts = np.array(g("col.groupStarts"), dtype=np.uint32)
        self.c = OraWorldC()
        self.c.n_bodies = self.a["comX"].size
        self.c.n_colliders = self.a["bodyIndex"].size
        self.c.n_materials = m.shape[0]
        for k in range(4):
            self.c.body_starts[k] = int(self.body_starts[k])
            self.c.col_starts[k] = int(self.col_starts[k])
        for name, arr in self.a.items():
            ptr_t = _U if arr.dtype == np.uint32 else _F
            setattr(self.c, name, arr.ctypes.data_as(ptr_t))

    @property
    def ref(self):
        return ctypes.byref(self.c)

    def group(self, starts, g):
        return int(starts[g]), int(starts[g + 1])

    # --- phases ---
    def integrate(self, dt, gx, gy, damping=1.0):
        b, e = self.group(self.body_starts, 2)
        lib().ora_integrate_velocity_verlet(self.ref, b, e, dt, gx, gy, damping)
        lib().ora_wrap_body_rotations(self.ref, b, e)
        lib().ora_body_cossin(self.ref, b, e)

    def spatial(self, full: bool):
        """Collider poses and AABBs: the whole live range (rebuild after structural changes) or the dynamic range."""
        if full:
            b, e = 0, int(self.col_starts[3])
        else:
            b, e = self.group(self.col_starts, 2)
        lib().ora_collider_world_positions(self.ref, b, e)
        lib().ora_collider_world_rotations(self.ref, b, e)
        lib().ora_collider_aabbs(self.ref, b, e)

    def morton(self, group=2):
        b, e = self.group(self.col_starts, group)
        n = e - b
        codes = np.zeros(max(n, 1), np.uint32)
        bounds = np.zeros(4, np.float32)
        lib().ora_morton_codes(self.ref, b, e, codes.ctypes.data, bounds.ctypes.data)
        sorted_c = np.zeros(max(n, 1), np.uint32)
        sorted_k = np.zeros(max(n, 1), np.uint32)
        lib().ora_sort_by_morton(codes.ctypes.data, b, n, sorted_c.ctypes.data, sorted_k.ctypes.data)
        return codes[:n], sorted_c[:n], sorted_k[:n], bounds

    def broad_pairs(self):
        cap = max(16, 8 * int(self.c.n_colliders))
        while True:
            out = np.zeros((cap, 2), np.uint32)
            n = lib().ora_broad_pairs(self.ref, out.ctypes.data, cap)
            if n >= 0:
                return out[:n].copy()
            cap = -n

    def narrow(self, pairs: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros(max(1, p.shape[0]), MANIFOLD_DTYPE)
        n = lib().ora_narrow(self.ref, p.ctypes.data, p.shape[0], out.ctypes.data)
        return out[:n].copy()

    def solve(self, manifolds: np.ndarray, order=None, vel_iters=8, pos_iters=3) -> np.ndarray:
        m = np.ascontiguousarray(manifolds.copy())
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int64)
        lib().ora_solve(self.ref, m.ctypes.data, m.shape[0], None if o is None else o.ctypes.data,
                        vel_iters, pos_iters)
        return m

    def solve_f64(self, manifolds: np.ndarray, order=None, vel_iters=8, pos_iters=3):
        m = np.ascontiguousarray(manifolds.copy())
        nb = int(self.c.n_bodies)
        vel = np.stack([self.a["velX"], self.a["velY"], self.a["angVel"]], 1).astype(np.float64).copy()
        pos = np.stack([self.a["comX"], self.a["comY"]], 1).astype(np.float64).copy()
        imp = np.zeros((max(1, m.shape[0]), 4), np.float64)
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int64)
        lib().ora_solve_f64(self.ref, m.ctypes.data, m.shape[0], None if o is None else o.ctypes.data,
                            vel_iters, pos_iters, vel.ctypes.data, pos.ctypes.data, imp.ctypes.data)
        assert vel.shape[0] == nb
        return vel, pos, imp[:m.shape[0]]

    def collision_events(self, manifolds: np.ndarray, callback: np.ndarray, threshold: np.ndarray) -> np.ndarray:
        """Events (EVENT_DTYPE, dense indices) of the manifolds from the world's current velocities, in manifold
        order with side a first, for colliders opted in by callback id and threshold."""
        m = np.ascontiguousarray(manifolds)
        cb = np.ascontiguousarray(callback, dtype=np.uint32)
        th = np.ascontiguousarray(threshold, dtype=np.float32)
        out = np.zeros(max(1, 2 * m.shape[0]), EVENT_DTYPE)
        k = lib().ora_collision_events(self.ref, m.ctypes.data, m.shape[0], cb.ctypes.data, th.ctypes.data,
                                       out.ctypes.data, out.size)
        assert k >= 0
        return out[:k].copy()

    def islands(self, body_edges: np.ndarray):
        e = np.ascontiguousarray(body_edges, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros(max(1, int(self.c.n_bodies)), np.uint32)
        k = lib().ora_islands(self.ref, e.ctypes.data, e.shape[0], out.ctypes.data)
        return out[:int(self.c.n_bodies)], int(k)

    def update_sleeping(self, island_id, island_count, dt, speed=0.1, time=0.5):
        ii = np.ascontiguousarray(island_id, dtype=np.uint32)
        out = np.zeros(max(1, int(self.c.n_bodies)), np.uint8)
        lib().ora_update_sleeping(self.ref, ii.ctypes.data, island_count, dt, speed, time, out.ctypes.data)
        return out[:int(self.c.n_bodies)]


def warm_start(prev: np.ndarray, prev_slots: np.ndarray, cur: np.ndarray, cur_slots: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(prev)
    c = np.ascontiguousarray(cur.copy())
    pa = np.ascontiguousarray(prev_slots[:, 0], dtype=np.uint32)
    pb = np.ascontiguousarray(prev_slots[:, 1], dtype=np.uint32)
    ca = np.ascontiguousarray(cur_slots[:, 0], dtype=np.uint32)
    cb = np.ascontiguousarray(cur_slots[:, 1], dtype=np.uint32)
    lib().ora_warm_start(p.ctypes.data, pa.ctypes.data, pb.ctypes.data, p.shape[0], c.ctypes.data, ca.ctypes.data,
                         cb.ctypes.data, c.shape[0])
    return c


def broad_pairs_from_aabbs(minx, miny, maxx, maxy, body) -> np.ndarray:
    """Candidate pairs of a world whose colliders are all dynamic, from their AABBs and owner bodies (the oracle's
    x-sweep, ora_broad_pairs): (min, max) collider pairs that overlap strictly and belong to different bodies."""
    n = int(np.asarray(minx).size)
    c = OraWorldC()
    c.n_bodies = int(np.max(body)) + 1 if n else 0
    c.n_colliders = n
    for k, v in enumerate((0, 0, 0, n)):
        c.col_starts[k] = v
    keep = []
    for name, arr in (("minX", minx), ("minY", miny), ("maxX", maxx), ("maxY", maxy), ("bodyIndex", body)):
        a = np.ascontiguousarray(arr, dtype=np.uint32 if name == "bodyIndex" else np.float32)
        keep.append(a)
        setattr(c, name, a.ctypes.data_as(_U if a.dtype == np.uint32 else _F))
    cap = max(16 * n, 1024)
    while True:
        out = np.zeros((cap, 2), np.uint32)
        got = lib().ora_broad_pairs(ctypes.byref(c), out.ctypes.data, cap)
        if got >= 0:
            return out[:got]
        cap = int(-got)   # the buffer was too small: the count comes back negated


def fastcossin(angles: np.ndarray):
    a = np.ascontiguousarray(angles, dtype=np.float32)
    c = np.empty_like(a)
    s = np.empty_like(a)
    lib().ora_fastcossin_array(a.ctypes.data, c.ctypes.data, s.ctypes.data, a.size)
    return c, s


def manifolds_from_dump(d: dict, prefix: str) -> np.ndarray:
    """Manifold records from a reference dump (names <prefix>colA, colB, normal, depth, count, points, ids,
    impulses) with dense collider indices."""
    n = np.asarray(d[prefix + "count"]).size
    m = np.zeros(n, MANIFOLD_DTYPE)
    m["a"] = d[prefix + "colA"]
    m["b"] = d[prefix + "colB"]
    nrm = np.asarray(d[prefix + "normal"]).reshape(-1, 2)
    m["nx"], m["ny"] = nrm[:, 0], nrm[:, 1]
    m["depth"] = d[prefix + "depth"]
    m["count"] = d[prefix + "count"]
    pts = np.asarray(d[prefix + "points"]).reshape(-1, 4)
    m["px"] = pts[:, [0, 2]]
    m["py"] = pts[:, [1, 3]]
    m["id"] = np.asarray(d[prefix + "ids"]).reshape(-1, 2)
    imp = np.asarray(d[prefix + "impulses"]).reshape(-1, 4)
    m["jn"] = imp[:, [0, 2]]
    m["jt"] = imp[:, [1, 3]]
    return m
