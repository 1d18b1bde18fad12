"""ctypes wrapper over oracle/_ref/libagony_ref.so, the reference engine (PS_AGONY2D) built on the CPU.

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py, by the oracle self-checks in tests/ and by the
reference (CPU baseline) arm of bench.py. The product path never imports it.

Scenes come from ag2d.scenes (the same generator feeds this library), so both sides start from identical inputs.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libagony_ref.so")


class _Settings(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("velocity_iterations", ctypes.c_uint32),
                ("position_iterations", ctypes.c_uint32), ("gravity_x", ctypes.c_float),
                ("gravity_y", ctypes.c_float), ("ccd", ctypes.c_int32), ("sleep_speed", ctypes.c_float),
                ("sleep_time", ctypes.c_float), ("threads", ctypes.c_int32)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} is missing: run oracle/ref_build.sh")
        L = ctypes.CDLL(LIB_PATH)
        vp, f, u32, i32, i64 = ctypes.c_void_p, ctypes.c_float, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int64
        L.agref_create.restype = vp
        L.agref_create.argtypes = [ctypes.POINTER(_Settings)]
        L.agref_destroy.argtypes = [vp]
        L.agref_material.restype = u32
        L.agref_material.argtypes = [vp, f, f, f]
        L.agref_add_polygon.restype = i64
        L.agref_add_polygon.argtypes = [vp, vp, u32, f, f, f, f, f, f, f, u32]
        L.agref_add_box.restype = i64
        L.agref_add_box.argtypes = [vp, f, f, f, f, f, f, f, f, f, u32]
        L.agref_add_circle.restype = i64
        L.agref_add_circle.argtypes = [vp, f, f, f, f, f, f, f, f, u32]
        L.agref_add_capsule.restype = i64
        L.agref_add_capsule.argtypes = [vp, f, f, f, f, f, f, f, f, f, u32]
        L.agref_create_body.restype = i64
        L.agref_create_body.argtypes = [vp, f, f, f, f, f, f, f, f, f, f]
        L.agref_add_collider.restype = i64
        L.agref_add_collider.argtypes = [vp, u32, i32, f, f, f, u32, f, f, vp, u32]
        L.agref_flush_commands.argtypes = [vp]
        L.agref_update.argtypes = [vp, i32]
        L.agref_destroy_body.argtypes = [vp, u32]
        L.agref_set_body.argtypes = [vp, u32, i32, f, f]
        L.agref_set_collider.argtypes = [vp, u32, i32, f, f]
        L.agref_set_polygon.argtypes = [vp, u32, ctypes.POINTER(ctypes.c_float), u32]
        L.agref_set_polygon.restype = i32
        L.agref_decompose.argtypes = [ctypes.POINTER(ctypes.c_float), u32, ctypes.POINTER(ctypes.c_float), u32,
                                      ctypes.POINTER(ctypes.c_uint32), u32]
        L.agref_decompose.restype = i32
        L.agref_body_index.restype = u32
        L.agref_body_index.argtypes = [vp, u32]
        L.agref_timed_update.restype = ctypes.c_double
        L.agref_timed_update.argtypes = [vp, i32]
        L.agref_timed_collide.restype = ctypes.c_double
        L.agref_timed_collide.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.agref_body_count.restype = u32
        L.agref_body_count.argtypes = [vp]
        L.agref_collider_count.restype = u32
        L.agref_collider_count.argtypes = [vp]
        L.agref_manifold_count.restype = u32
        L.agref_manifold_count.argtypes = [vp]
        L.agref_dump_state.argtypes = [vp, ctypes.c_char_p]
        L.agref_set_body_field.restype = i32
        L.agref_set_body_field.argtypes = [vp, ctypes.c_char_p, vp]
        L.agref_phase_step.argtypes = [vp]
        L.agref_blob_size.restype = ctypes.c_uint64
        L.agref_blob_size.argtypes = [vp, ctypes.c_char_p]
        L.agref_blob_copy.restype = i32
        L.agref_blob_copy.argtypes = [vp, ctypes.c_char_p, vp]
        L.agref_blob_names.restype = ctypes.c_uint64
        L.agref_blob_names.argtypes = [vp, ctypes.c_char_p, ctypes.c_uint64]
        L.agref_clear_blobs.argtypes = [vp]
        L.agref_query_shape.argtypes = [vp, i32, vp, u32, vp, ctypes.c_uint64]
        L.agref_query_shape.restype = ctypes.c_int64
        L.agref_circle_contacts.argtypes = [vp, f, f, f, u32, vp, vp, ctypes.c_uint64]
        L.agref_circle_contacts.restype = ctypes.c_int64
        L.agref_fastcossin.argtypes = [vp, vp, vp, ctypes.c_uint64]
        L.agref_create_joint.restype = i64
        L.agref_create_joint.argtypes = [vp, i32, u32, u32, vp]
        L.agref_joint_order.restype = u32
        L.agref_joint_order.argtypes = [vp, i32, vp, vp, vp, u32]
        L.agref_destroy_joint.argtypes = [vp, i32, u32, u32]
        L.agref_motor_impulses.restype = u32
        L.agref_motor_impulses.argtypes = [vp, vp, vp, u32]
        L.agref_create_event_callback.restype = i32
        L.agref_create_event_callback.argtypes = [vp]
        L.agref_destroy_event_callback.restype = i32
        L.agref_destroy_event_callback.argtypes = [vp, u32]
        L.agref_set_collider_callback.restype = i32
        L.agref_set_collider_callback.argtypes = [vp, u32, u32, f]
        L.agref_set_events_enabled.argtypes = [vp, i32]
        L.agref_dump_events.argtypes = [vp, ctypes.c_char_p]
        _lib = L
    return _lib


_U32_SUFFIXES = ("bodyIndex", "materialIndex", "shapeType", "shapeIndex", "groupStarts", "handleSlot", "handleGen",
                 "islandId", "sleepIslandId", "colliderIndices", "counts", "colA", "colB", "slotA", "slotB", "count",
                 "ids", "sorted", "morton", "pairs", "spatialDirty", "callbackId", "self", "other", "selfBody",
                 "otherBody", "callback")


def _dtype_for(name: str):
    last = name.rsplit(".", 1)[-1]
    return np.uint32 if last in _U32_SUFFIXES else np.float32


class RefSim:
    """One reference Simulation (Simulation.h:36-255) configured like a Scene and loaded with its bodies."""

    def __init__(self, scene, threads: int = 0, ccd: bool = False, sleep_speed: float = 0.1,
                 sleep_time: float = 0.5):
        L = lib()
        s = _Settings(scene.dt, scene.velocity_iterations, scene.position_iterations, scene.gravity[0],
                      scene.gravity[1], 1 if ccd else 0, sleep_speed, sleep_time, threads)
        self.h = L.agref_create(ctypes.byref(s))
        self.scene = scene
        mats = [L.agref_material(self.h, *m) for m in scene.materials]
        self.body_slots = []
        for i in range(scene.n):
            mat = mats[int(scene.material[i]) - 1] if int(scene.material[i]) >= 1 else 0
            args = (float(scene.px[i]), float(scene.py[i]), float(scene.rot[i]), float(scene.vx[i]),
                    float(scene.vy[i]), float(scene.w[i]), float(scene.mass[i]), mat)
            k = int(scene.kind[i])
            if k == 2:
                v = np.ascontiguousarray(scene.polygon_vertices(i), dtype=np.float32)
                slot = L.agref_add_polygon(self.h, v.ctypes.data, v.shape[0], *args)
            elif k == 1:
                slot = L.agref_add_box(self.h, float(scene.width[i]), float(scene.height[i]), *args)
            elif k == 3:
                slot = L.agref_add_capsule(self.h, float(scene.width[i]), float(scene.radius[i]), *args)
            else:
                slot = L.agref_add_circle(self.h, float(scene.radius[i]), *args)
            if slot < 0:
                raise ValueError(f"reference rejected body {i}")
            self.body_slots.append(slot)

    def close(self):
        if self.h:
            lib().agref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ObjectAPI deferred body commands, by the handle slot the constructor recorded for scene body i.
    SET_POSITION, SET_ROTATION, SET_VELOCITY, SET_ANGULAR_VELOCITY, SET_MASS, SET_INERTIA = range(6)

    def destroy_body(self, i: int):
        lib().agref_destroy_body(self.h, self.body_slots[i])

    def set_body(self, i: int, kind: int, a: float, b: float = 0.0):
        lib().agref_set_body(self.h, self.body_slots[i], kind, a, b)

    def add_material(self, elasticity: float, static_friction: float, dynamic_friction: float) -> int:
        """Simulation::addMaterial; the new material's index."""
        return int(lib().agref_material(self.h, elasticity, static_friction, dynamic_friction))

    def create_body(self, x, y, rotation=0.0, vx=0.0, vy=0.0, w=0.0, mass=1.0, inertia=1.0, com=(0.0, 0.0)) -> int:
        """ObjectAPI::createBody: a body without colliders. Returns its index in body_slots (like a scene body's)."""
        slot = lib().agref_create_body(self.h, x, y, rotation, vx, vy, w, mass, inertia, com[0], com[1])
        if slot < 0:
            raise ValueError("reference rejected the body")
        self.body_slots.append(slot)
        return len(self.body_slots) - 1

    def add_collider(self, i: int, shape: int, offset=(0.0, 0.0), rotation=0.0, material=0, radius=0.0, width=0.0,
                     height=0.0, length=0.0, vertices=None) -> int:
        """ObjectAPI::create*Collider on body i (0 circle, 1 box, 2 polygon, 3 capsule); the collider's dense index.
        material is a material index as returned by the reference (0 = its default material)."""
        p0, p1 = {0: (radius, 0.0), 1: (width, height), 2: (0.0, 0.0), 3: (length, radius)}[shape]
        xy, n = None, 0
        if vertices is not None:
            v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 2)
            xy, n = v.ctypes.data, v.shape[0]
        c = lib().agref_add_collider(self.h, self.body_slots[i], shape, offset[0], offset[1], rotation, material, p0,
                                     p1, xy, n)
        if c < 0:
            raise ValueError("reference rejected the collider")
        return int(c)

    def set_collider(self, index: int, kind: int, a: float, b: float = 0.0):
        """A collider setter on the collider at dense index 'index' (applied at the next flush)."""
        lib().agref_set_collider(self.h, index, kind, a, b)

    def set_polygon(self, index: int, xy) -> bool:
        """ObjectAPI::setPolygonShape on the collider at dense index 'index' (applied at the next flush)."""
        v = np.ascontiguousarray(np.asarray(xy, np.float32).reshape(-1))
        return bool(lib().agref_set_polygon(self.h, index, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                            v.size // 2))

    def body_index(self, i: int) -> int:
        """Dense index of scene body i now (2**32 - 1 once destroyed)."""
        return int(lib().agref_body_index(self.h, self.body_slots[i]))

    def flush_commands(self):
        """Applies the queued commands now (the first part of the next update)."""
        lib().agref_flush_commands(self.h)

    def update(self, steps: int = 1):
        lib().agref_update(self.h, steps)

    def timed_collide(self):
        """(seconds, pairs, manifolds) of one collision detection pass (spatial data, broad, narrow)."""
        p, m = ctypes.c_uint64(), ctypes.c_uint64()
        t = lib().agref_timed_collide(self.h, ctypes.byref(p), ctypes.byref(m))
        return float(t), int(p.value), int(m.value)

    def timed_update(self, steps: int) -> float:
        return float(lib().agref_timed_update(self.h, steps))

    def phase_step(self):
        lib().agref_clear_blobs(self.h)
        lib().agref_phase_step(self.h)

    def dump_state(self, prefix: str = "state."):
        lib().agref_dump_state(self.h, prefix.encode())

    def set_body_field(self, field: str, values: np.ndarray):
        v = np.ascontiguousarray(values, dtype=np.float32)
        if lib().agref_set_body_field(self.h, field.encode(), v.ctypes.data) != 0:
            raise KeyError(field)

    def blob_names(self):
        L = lib()
        n = L.agref_blob_names(self.h, None, 0)
        buf = ctypes.create_string_buffer(int(n))
        L.agref_blob_names(self.h, buf, n)
        return [s for s in buf.value.decode().split("\n") if s]

    def blob(self, name: str) -> np.ndarray:
        L = lib()
        size = L.agref_blob_size(self.h, name.encode())
        if size == 2**64 - 1:
            raise KeyError(name)
        dt = _dtype_for(name)
        out = np.empty(int(size) // np.dtype(dt).itemsize, dtype=dt)
        if size:
            L.agref_blob_copy(self.h, name.encode(), out.ctypes.data)
        return out

    def blobs(self, prefix: str = "") -> dict:
        return {k: self.blob(k) for k in self.blob_names() if k.startswith(prefix)}

    def query_shape(self, shape: int, params, trees: int = 7) -> np.ndarray:
        """Dense collider indices a shape query finds in the reference's trees (0 = AABB, 1 = circle)."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        n = lib().agref_query_shape(self.h, shape, p.ctypes.data, trees, None, 0)
        out = np.empty(max(int(n), 1), np.uint32)
        lib().agref_query_shape(self.h, shape, p.ctypes.data, trees, out.ctypes.data, out.size)
        return out[:int(n)]

    def circle_contacts(self, x: float, y: float, r: float, trees: int = 7):
        """(colliders, signed distances) the reference's findCollisionsInCircle reports for its circle query."""
        L = lib()
        n = L.agref_circle_contacts(self.h, x, y, r, trees, None, None, 0)
        idx = np.empty(max(int(n), 1), np.uint32)
        sdf = np.empty(max(int(n), 1), np.float32)
        L.agref_circle_contacts(self.h, x, y, r, trees, idx.ctypes.data, sdf.ctypes.data, idx.size)
        return idx[:int(n)], sdf[:int(n)]

    def create_joint(self, kind: int, a: int, b: int, params) -> int:
        """A spring (0), revolute joint (1) or motor (4, body a) between bodies given by handle slot."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        return int(lib().agref_create_joint(self.h, kind, a, b, p.ctypes.data))

    def joint_order(self, kind: int):
        """(handle slots, generations, group starts) of a constraint system in dense order."""
        slot = np.zeros(65536, np.uint32)
        gen = np.zeros(65536, np.uint32)
        starts = np.zeros(4, np.uint32)
        n = int(lib().agref_joint_order(self.h, kind, slot.ctypes.data, gen.ctypes.data, starts.ctypes.data,
                                        slot.size))
        return slot[:n].copy(), gen[:n].copy(), starts

    def destroy_joint(self, kind: int, slot: int, gen: int):
        lib().agref_destroy_joint(self.h, kind, slot, gen)

    def motor_impulses(self):
        """(accumulated impulses, body handle slots) of the motors in dense order."""
        imp = np.zeros(4096, np.float32)
        slot = np.zeros(4096, np.uint32)
        n = int(lib().agref_motor_impulses(self.h, imp.ctypes.data, slot.ctypes.data, imp.size))
        return imp[:n].copy(), slot[:n].copy()

    def create_event_callback(self) -> int:
        """A collision callback that records every event it receives (Simulation::createCollisionCallback)."""
        return int(lib().agref_create_event_callback(self.h))

    def destroy_event_callback(self, cb: int) -> bool:
        return bool(lib().agref_destroy_event_callback(self.h, cb))

    def set_collider_callback(self, collider: int, cb: int, threshold: float) -> bool:
        """Simulation::setColliderCollisionCallback on a dense collider index."""
        return bool(lib().agref_set_collider_callback(self.h, collider, cb, threshold))

    def set_events_enabled(self, enable: bool):
        lib().agref_set_events_enabled(self.h, 1 if enable else 0)

    def events(self, prefix: str = "e.") -> dict:
        """The events recorded since the last call (handle slots, points, normals, impulses), in dispatch order."""
        lib().agref_dump_events(self.h, prefix.encode())
        return {k[len(prefix) + 3:]: self.blob(k) for k in (prefix + "ev." + n for n in
                ("self", "other", "selfBody", "otherBody", "callback", "px", "py", "nx", "ny", "impulse"))}

    @property
    def manifold_count(self) -> int:
        return int(lib().agref_manifold_count(self.h))


def fastcossin(angles: np.ndarray):
    a = np.ascontiguousarray(angles, dtype=np.float32)
    c = np.empty_like(a)
    s = np.empty_like(a)
    lib().agref_fastcossin(a.ctypes.data, c.ctypes.data, s.ctypes.data, a.size)
    return c, s


def decompose(xy):
    """The reference's convex pieces for an outline (preparePolygonOutline, decomposeConcave, the 16-vertex limit):
    a list of (k, 2) float32 arrays, or None when the outline is refused."""
    v = np.ascontiguousarray(np.asarray(xy, np.float32).reshape(-1))
    out = np.zeros(4096, np.float32)
    counts = np.zeros(512, np.uint32)
    f = ctypes.POINTER(ctypes.c_float)
    k = lib().agref_decompose(v.ctypes.data_as(f), v.size // 2, out.ctypes.data_as(f), out.size // 2,
                              counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), counts.size)
    if k < 0:
        return None
    pieces, at = [], 0
    for c in counts[:k].tolist():
        pieces.append(out[2 * at:2 * (at + c)].reshape(-1, 2).copy())
        at += c
    return pieces
