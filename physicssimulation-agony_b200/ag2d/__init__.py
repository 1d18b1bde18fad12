"""ag2d: B200-native collision and contact pipeline behind the PS_AGONY2D world/body/shape/step API.

Python binding over the C ABI of libag2d.so (include/ag2d.h). The library is the CUDA implementation; there is no
CPU fallback: the first call into the library raises ImportError when the built library is missing (the scene
generators import without it), and creating a world without a CUDA device returns AG2D_ERR_NO_DEVICE.

    from ag2d import World, scenes
    w = World.from_scene(scenes.make_c1(2048))
    w.step(600)
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import scenes  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libag2d.so")

OK = 0
ERR_INVALID_ARG, ERR_OOM, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_NO_DEVICE, ERR_UNSUPPORTED = -1, -2, -3, -4, -5, -6, -7

# enum ag2d_field
BODY_COM_X, BODY_COM_Y, BODY_VEL_X, BODY_VEL_Y, BODY_ROTATION, BODY_ANGULAR_VELOCITY, BODY_ROT_COS, BODY_ROT_SIN, \
    BODY_WRAP_COUNT, BODY_SLEEP_TIMER, BODY_STATE, BODY_SLEEP_ISLAND, BODY_POSE, BODY_INV_MASS, \
    BODY_INV_INERTIA = range(1, 16)
COL_WORLD_X, COL_WORLD_Y, COL_WORLD_ROTATION, COL_WORLD_COS, COL_WORLD_SIN, COL_AABB_MIN_X, COL_AABB_MIN_Y, \
    COL_AABB_MAX_X, COL_AABB_MAX_Y, COL_BODY = range(32, 42)
DYN_SORTED, DYN_MORTON, PAIRS, MANIFOLDS, PREV_MANIFOLDS, SOLVE_ORDER, COLOR_STARTS, ISLAND_MANIFOLDS, \
    ISLAND_IDS = range(64, 73)
# enum ag2d_phase
# enum ag2d_command: collider setters (by dense collider index)
COMMAND_COLLIDER_OFFSET, COMMAND_COLLIDER_ROTATION, COMMAND_COLLIDER_MATERIAL, COMMAND_CIRCLE_RADIUS, \
    COMMAND_BOX_SIZE, COMMAND_CAPSULE_SHAPE, COMMAND_POLYGON_SHAPE = range(16, 23)
PHASE_INTEGRATE, PHASE_SPATIAL_FULL, PHASE_SPATIAL_DYNAMIC, PHASE_BROAD, PHASE_NARROW, PHASE_SOLVE, \
    PHASE_ISLANDS, PHASE_COLLIDE, PHASE_CCD, PHASE_WAKE, PHASE_EVENTS = range(1, 12)

MANIFOLD_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("nx", "<f4"), ("ny", "<f4"), ("depth", "<f4"),
                           ("count", "<u4"), ("id0", "<u4"), ("id1", "<u4"), ("px0", "<f4"), ("py0", "<f4"),
                           ("px1", "<f4"), ("py1", "<f4"), ("jn0", "<f4"), ("jt0", "<f4"), ("jn1", "<f4"),
                           ("jt1", "<f4")])
assert MANIFOLD_DTYPE.itemsize == 64

_U32_FIELDS = {BODY_STATE, BODY_SLEEP_ISLAND, COL_BODY, DYN_SORTED, DYN_MORTON, SOLVE_ORDER, COLOR_STARTS,
               ISLAND_IDS}


class Ag2dError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"ag2d error {code}: {message}")
        self.code = code


class WorldSettings(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("velocity_iterations", ctypes.c_uint32),
                ("position_iterations", ctypes.c_uint32), ("gravity_x", ctypes.c_float),
                ("gravity_y", ctypes.c_float), ("angular_damping", ctypes.c_float), ("sleep_speed", ctypes.c_float),
                ("sleep_time", ctypes.c_float), ("ccd", ctypes.c_int32), ("device", ctypes.c_int32)]


class BodyDesc(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("rotation", ctypes.c_float), ("vx", ctypes.c_float),
                ("vy", ctypes.c_float), ("angular_velocity", ctypes.c_float), ("mass", ctypes.c_float),
                ("material", ctypes.c_uint32)]


_BODY_DESC_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("rotation", "<f4"), ("vx", "<f4"), ("vy", "<f4"),
                             ("w", "<f4"), ("mass", "<f4"), ("material", "<u4")])
assert _BODY_DESC_DTYPE.itemsize == ctypes.sizeof(BodyDesc)


class Counters(ctypes.Structure):
    _fields_ = [("status", ctypes.c_uint32), ("pairs", ctypes.c_uint32), ("manifolds", ctypes.c_uint32),
                ("colors", ctypes.c_uint32), ("woke", ctypes.c_uint32), ("slept", ctypes.c_uint32),
                ("warm_hits", ctypes.c_uint32), ("sleeping", ctypes.c_uint32), ("ccd_hits", ctypes.c_uint32),
                ("restored", ctypes.c_uint32), ("events", ctypes.c_uint32), ("stored", ctypes.c_uint32),
                ("steps", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("list_rebuilds", ctypes.c_uint64), ("retries", ctypes.c_uint64),
                ("regrows", ctypes.c_uint64), ("host_ms", ctypes.c_double), ("sync_ms", ctypes.c_double),
                ("device_allocs", ctypes.c_uint64)]


class CollisionEvent(ctypes.Structure):
    """ag2d_collision_event: one collision event from one collider's side (Types/CollisionEvent.h:18-26)."""
    _fields_ = [("self", ctypes.c_uint32), ("other", ctypes.c_uint32), ("self_body", ctypes.c_uint32),
                ("other_body", ctypes.c_uint32), ("self_body_handle", ctypes.c_uint64),
                ("other_body_handle", ctypes.c_uint64), ("point_x", ctypes.c_float), ("point_y", ctypes.c_float),
                ("normal_x", ctypes.c_float), ("normal_y", ctypes.c_float), ("impulse", ctypes.c_float),
                ("callback_id", ctypes.c_uint16), ("pad", ctypes.c_uint16)]


EVENT_DTYPE = np.dtype([(n, {ctypes.c_uint32: "<u4", ctypes.c_uint64: "<u8", ctypes.c_float: "<f4",
                             ctypes.c_uint16: "<u2"}[t]) for n, t in CollisionEvent._fields_])
assert EVENT_DTYPE.itemsize == ctypes.sizeof(CollisionEvent) == 56
COLLISION_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.POINTER(CollisionEvent), ctypes.c_void_p, ctypes.c_void_p)
NO_COLLISION_EVENT_THRESHOLD = float(np.finfo(np.float32).max)


# enum ag2d_joint_kind / ag2d_joint_field
JOINT_SPRING, JOINT_REVOLUTE, JOINT_PRISMATIC, JOINT_SLIDER, JOINT_MOTOR = range(5)
JOINT_ANCHOR_A, JOINT_ANCHOR_B, JOINT_REST_LENGTH, JOINT_STIFFNESS, JOINT_DAMPING, JOINT_TARGET_SPEED, \
    JOINT_MAX_TORQUE, JOINT_AXIS_A, JOINT_LIMITS, JOINT_ENABLE_LIMIT, JOINT_RESET_REFERENCE_ANGLE = range(11)


class JointDesc(ctypes.Structure):
    """ag2d_joint_desc: a spring, revolute joint or motor."""
    _fields_ = [("kind", ctypes.c_int32), ("enable_limit", ctypes.c_int32), ("body_a", ctypes.c_uint64),
                ("body_b", ctypes.c_uint64)] + \
               [(n, ctypes.c_float) for n in ("anchor_a_x", "anchor_a_y", "anchor_b_x", "anchor_b_y", "rest_length",
                                              "stiffness", "damping", "target_speed", "max_torque", "axis_x",
                                              "axis_y", "lower_limit", "upper_limit", "reference_angle", "impulse")]


class Tuning(ctypes.Structure):
    _fields_ = [("team_colliders", ctypes.c_uint32), ("team_threads", ctypes.c_uint32), ("query_threads", ctypes.c_uint32),
                ("narrow_threads", ctypes.c_uint32), ("solve_ms", ctypes.c_float), ("query_ms", ctypes.c_float),
                ("narrow_ms", ctypes.c_float), ("team_cons_on_chip", ctypes.c_uint32),
                ("big_team_mode", ctypes.c_uint32)]


TIMED_PHASES = ("integrate", "pose", "tree_dynamic", "tree_other", "query", "narrow", "compact", "warm", "wake",
                "color", "solve", "islands", "sort", "lbvh", "ccd")


class ServerSettings(ctypes.Structure):
    _fields_ = [("world", WorldSettings), ("memory_budget_bytes", ctypes.c_uint64),
                ("steps_per_round", ctypes.c_uint32), ("max_worlds", ctypes.c_uint32),
                ("reserve_bodies", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "completed", "waiting", "resident",
                                               "peak_resident", "rounds", "body_steps")] + \
               [(n, ctypes.c_double) for n in ("busy_ms", "step_ms", "repack_ms", "p50_ms", "p99_ms", "max_ms")]


REQUEST_WAITING, REQUEST_RUNNING, REQUEST_DONE = 0, 1, 2
# enum ag2d_body_state (AG2D_BODY_STATE values)
STATE_STATIC, STATE_SLEEPING, STATE_DYNAMIC, STATE_DESTROYED = 0, 1, 2, 3
# enum ag2d_tree_flag / ag2d_query_shape
TREE_DYNAMIC, TREE_STATIC, TREE_SLEEPING, TREE_ALL = 1, 2, 4, 7
QUERY_AABB, QUERY_CIRCLE = 0, 1

_P = ctypes.c_void_p


class StateDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("n_bodies", "n_colliders", "n_circles", "n_boxes", "n_polygons",
                                               "n_materials")] + \
               [(n, _P) for n in ("body_group_starts", "com_x", "com_y", "vel_x", "vel_y", "rotation",
                                  "angular_velocity", "inv_mass", "inv_inertia", "rot_cos", "rot_sin", "wrap_count",
                                  "bound_radius", "sleep_timer", "sleep_island", "col_body", "col_shape_type",
                                  "col_shape_index", "col_material", "col_com_offset_x", "col_com_offset_y",
                                  "col_local_rotation", "circle_radius", "box_half_width", "box_half_height",
                                  "poly_count", "poly_vertices", "poly_normals", "materials", "col_world_x",
                                  "col_world_y", "col_world_cos", "col_world_sin", "col_aabb_min_x",
                                  "col_aabb_min_y", "col_aabb_max_x", "col_aabb_max_y")] + \
               [("n_capsules", ctypes.c_uint32), ("capsule_half_length", _P), ("capsule_radius", _P)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with physicssimulation-agony_b200/build.py "
                          "(the CUDA library is required; there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    i32, u32, u64, vp = ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
    L.ag2d_last_error_string.restype = ctypes.c_char_p
    L.ag2d_version.restype = i32
    L.ag2d_device_count.argtypes = [ctypes.POINTER(i32)]
    L.ag2d_world_create.argtypes = [ctypes.POINTER(WorldSettings), ctypes.POINTER(vp)]
    L.ag2d_world_destroy.argtypes = [vp]
    L.ag2d_world_add_material.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.POINTER(u32)]
    L.ag2d_world_add_circle.argtypes = [vp, ctypes.POINTER(BodyDesc), ctypes.c_float, ctypes.POINTER(u64)]
    L.ag2d_world_add_box.argtypes = [vp, ctypes.POINTER(BodyDesc), ctypes.c_float, ctypes.c_float,
                                     ctypes.POINTER(u64)]
    L.ag2d_world_add_polygon.argtypes = [vp, ctypes.POINTER(BodyDesc), vp, u32, ctypes.POINTER(u64)]
    L.ag2d_world_add_capsule.argtypes = [vp, ctypes.POINTER(BodyDesc), ctypes.c_float, ctypes.c_float,
                                         ctypes.POINTER(u64)]
    L.ag2d_world_body_index.restype = u32
    L.ag2d_world_create_body.argtypes = [vp, ctypes.POINTER(BodyDesc), ctypes.c_float, ctypes.c_float,
                                         ctypes.c_float, ctypes.POINTER(u64)]
    L.ag2d_world_add_collider.argtypes = [vp, u64, i32, ctypes.c_float, ctypes.c_float, ctypes.c_float, u32, vp, vp,
                                          u32, ctypes.POINTER(u32)]
    L.ag2d_world_add_bodies.argtypes = [vp, u32, ctypes.POINTER(BodyDesc), vp, vp, vp, vp, vp, vp]
    L.ag2d_world_body_index.argtypes = [vp, u64]
    L.ag2d_world_destroy_body.argtypes = [vp, u64]
    for name in ("position", "velocity"):
        getattr(L, f"ag2d_world_set_body_{name}").argtypes = [vp, u64, ctypes.c_float, ctypes.c_float]
    for name in ("rotation", "angular_velocity", "mass", "inertia"):
        getattr(L, f"ag2d_world_set_body_{name}").argtypes = [vp, u64, ctypes.c_float]
    L.ag2d_world_flush_commands.argtypes = [vp]
    L.ag2d_world_set_body_local_center_of_mass.argtypes = [vp, u64, ctypes.c_float, ctypes.c_float]
    L.ag2d_world_recompute_body_inertia.argtypes = [vp, u64]
    L.ag2d_world_set_body_mass_from_density.argtypes = [vp, u64, ctypes.c_float]
    L.ag2d_world_set_collider.argtypes = [vp, u32, i32, ctypes.c_float, ctypes.c_float]
    L.ag2d_world_set_polygon_shape.argtypes = [vp, u32, ctypes.POINTER(ctypes.c_float), u32]
    L.ag2d_decompose_polygon.argtypes = [ctypes.POINTER(ctypes.c_float), u32, ctypes.POINTER(ctypes.c_float), u32,
                                         ctypes.POINTER(u32), u32, ctypes.POINTER(u32)]
    L.ag2d_world_create_joint.argtypes = [vp, ctypes.POINTER(JointDesc), ctypes.POINTER(u64)]
    L.ag2d_world_destroy_joint.argtypes = [vp, i32, u64]
    L.ag2d_world_set_joint.argtypes = [vp, i32, u64, i32, ctypes.c_float, ctypes.c_float]
    L.ag2d_world_joint.argtypes = [vp, i32, u64, ctypes.POINTER(JointDesc)]
    L.ag2d_world_joint_count.argtypes = [vp, i32, ctypes.POINTER(u32)]
    L.ag2d_world_joint_handle.argtypes = [vp, i32, u32, ctypes.POINTER(u64)]
    L.ag2d_world_set_joint_iterations.argtypes = [vp, i32, u32]
    L.ag2d_world_create_collision_callback.argtypes = [vp, COLLISION_CALLBACK, vp, ctypes.POINTER(ctypes.c_uint16)]
    L.ag2d_world_destroy_collision_callback.argtypes = [vp, ctypes.c_uint16]
    L.ag2d_world_set_collider_collision_callback.argtypes = [vp, u32, ctypes.c_uint16, ctypes.c_float]
    L.ag2d_world_set_collision_events.argtypes = [vp, i32]
    L.ag2d_world_collision_events.argtypes = [vp, vp, u32, ctypes.POINTER(u32)]
    L.ag2d_world_load_state.argtypes = [vp, ctypes.POINTER(StateDesc)]
    L.ag2d_world_step.argtypes = [vp, i32]
    L.ag2d_world_counters.argtypes = [vp, ctypes.POINTER(Counters)]
    L.ag2d_device_allocs.argtypes = [ctypes.POINTER(u64)]
    L.ag2d_world_body_count.argtypes = [vp, ctypes.POINTER(u32), ctypes.POINTER(u32)]
    L.ag2d_world_read.argtypes = [vp, i32, vp, u64, ctypes.POINTER(u64)]
    L.ag2d_world_write.argtypes = [vp, i32, vp, u64]
    L.ag2d_world_read_async.argtypes = [vp, i32, vp, u64, ctypes.POINTER(u64)]
    L.ag2d_world_read_wait.argtypes = [vp]
    L.ag2d_host_alloc.argtypes = [u64, ctypes.POINTER(vp)]
    L.ag2d_host_free.argtypes = [vp]
    L.ag2d_batch_save.argtypes = [vp, vp, u64, ctypes.POINTER(u64)]
    L.ag2d_batch_restore.argtypes = [vp, u64, i32, ctypes.POINTER(vp)]
    L.ag2d_batch_load.argtypes = [vp, vp, u64]
    L.ag2d_world_run_phase.argtypes = [vp, i32]
    L.ag2d_world_set_profiling.argtypes = [vp, i32]
    L.ag2d_world_autotune.argtypes = [vp, i32, ctypes.POINTER(Tuning)]
    L.ag2d_world_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.ag2d_world_query_shape.argtypes = [vp, i32, vp, u32, vp, u32, ctypes.POINTER(u32)]
    L.ag2d_world_query_circle_contacts.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, u32, vp, vp,
                                                   u32, ctypes.POINTER(u32)]
    L.ag2d_world_phase_times.argtypes = [vp, vp, vp, i32]
    L.ag2d_world_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.ag2d_batch_create.argtypes = [ctypes.POINTER(vp), u32, ctypes.POINTER(vp)]
    L.ag2d_batch_step.argtypes = [vp, i32]
    L.ag2d_batch_engine.argtypes = [vp, ctypes.POINTER(vp)]
    L.ag2d_batch_world_count.argtypes = [vp, ctypes.POINTER(u32)]
    L.ag2d_batch_read.argtypes = [vp, u32, i32, vp, u64, ctypes.POINTER(u64)]
    L.ag2d_batch_destroy.argtypes = [vp]
    L.ag2d_server_create.argtypes = [ctypes.POINTER(ServerSettings), ctypes.POINTER(vp)]
    L.ag2d_server_submit.argtypes = [vp, vp, u32, ctypes.POINTER(u64)]
    L.ag2d_server_poll.argtypes = [vp, u64, ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_double)]
    L.ag2d_server_wait_all.argtypes = [vp, ctypes.c_double]
    L.ag2d_server_read.argtypes = [vp, u64, i32, vp, u64, ctypes.POINTER(u64)]
    L.ag2d_server_release.argtypes = [vp, u64]
    L.ag2d_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.ag2d_server_destroy.argtypes = [vp]
    return L


class _Lib:
    """Loads libag2d.so on first use (so that ag2d.scenes imports without it) and raises if it is missing."""

    _handle = None

    def __getattr__(self, name):
        if _Lib._handle is None:
            _Lib._handle = _load()
        return getattr(_Lib._handle, name)


lib = _Lib()


def device_allocs() -> int:
    """Device buffer allocations the library has made in this process (ag2d_counters.device_allocs)."""
    n = ctypes.c_uint64()
    _check(lib.ag2d_device_allocs(ctypes.byref(n)))
    return int(n.value)


def _check(code: int):
    if code != OK:
        raise Ag2dError(code, lib.ag2d_last_error_string().decode(errors="replace"))


class _HostBlock:
    """Page-locked host memory from ag2d_host_alloc, freed with the last array that views it."""

    def __init__(self, nbytes: int):
        p = ctypes.c_void_p()
        _check(lib.ag2d_host_alloc(max(int(nbytes), 1), ctypes.byref(p)))
        self.p = p.value
        self.nbytes = int(nbytes)

    def __del__(self):
        try:
            if self.p:
                lib.ag2d_host_free(self.p)
                self.p = None
        except Exception:
            pass


def host_empty(nbytes: int) -> np.ndarray:
    """A uint8 array of `nbytes` in page-locked host memory: the destination asynchronous reads require, and the
    fastest one for reads and checkpoints (one DMA, no staging). View it with .view(dtype) as needed."""
    block = _HostBlock(nbytes)
    raw = (ctypes.c_uint8 * max(block.nbytes, 1)).from_address(block.p)
    raw._ag2d_block = block   # the ctypes array keeps the allocation alive; numpy keeps the ctypes array
    return np.frombuffer(raw, dtype=np.uint8)[:block.nbytes]


def _field_view(buf: np.ndarray, field: int) -> np.ndarray:
    if field in (MANIFOLDS, PREV_MANIFOLDS, ISLAND_MANIFOLDS):
        return buf.view(MANIFOLD_DTYPE)
    if field == PAIRS:
        return buf.view(np.uint32).reshape(-1, 2)
    return buf.view(np.uint32 if field in _U32_FIELDS else np.float32)


def _out_bytes(out: np.ndarray):
    if not out.flags["C_CONTIGUOUS"]:
        raise ValueError("destination must be C-contiguous")
    return out.ctypes.data, out.nbytes


def device_count() -> int:
    n = ctypes.c_int32(0)
    _check(lib.ag2d_device_count(ctypes.byref(n)))
    return int(n.value)


class World:
    """One simulated world (the reference's Simulation, Simulation.h:36-255) resident on a GPU."""

    def __init__(self, dt=1.0 / 60.0, velocity_iterations=8, position_iterations=3, gravity=(0.0, -9.81),
                 angular_damping=1.0, sleep_speed=0.1, sleep_time=0.5, ccd=False, device=0):
        s = WorldSettings(dt, velocity_iterations, position_iterations, gravity[0], gravity[1], angular_damping,
                          sleep_speed, sleep_time, 1 if ccd else 0, device)
        h = ctypes.c_void_p()
        _check(lib.ag2d_world_create(ctypes.byref(s), ctypes.byref(h)))
        self.h = h
        self.settings = s
        self._keep = []

    @classmethod
    def _borrowed(cls, handle, owner):
        """A non-owning view of an engine instance owned by 'owner' (a Batch)."""
        w = cls.__new__(cls)
        w.h = handle
        w.settings = None
        w._keep = []
        w._owner = owner
        return w

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owner", None) is None:
                lib.ag2d_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- creation (ObjectAPI) ---
    def add_material(self, elasticity, static_friction, dynamic_friction) -> int:
        idx = ctypes.c_uint32()
        _check(lib.ag2d_world_add_material(self.h, elasticity, static_friction, dynamic_friction, ctypes.byref(idx)))
        return int(idx.value)

    @staticmethod
    def _desc(x, y, rotation, vx, vy, w, mass, material):
        return BodyDesc(x, y, rotation, vx, vy, w, mass, material)

    def add_circle(self, radius, x, y, rotation=0.0, vx=0.0, vy=0.0, w=0.0, mass=1.0, material=0) -> int:
        h = ctypes.c_uint64()
        d = self._desc(x, y, rotation, vx, vy, w, mass, material)
        _check(lib.ag2d_world_add_circle(self.h, ctypes.byref(d), radius, ctypes.byref(h)))
        return int(h.value)

    def add_box(self, width, height, x, y, rotation=0.0, vx=0.0, vy=0.0, w=0.0, mass=1.0, material=0) -> int:
        h = ctypes.c_uint64()
        d = self._desc(x, y, rotation, vx, vy, w, mass, material)
        _check(lib.ag2d_world_add_box(self.h, ctypes.byref(d), width, height, ctypes.byref(h)))
        return int(h.value)

    def add_polygon(self, vertices, x, y, rotation=0.0, vx=0.0, vy=0.0, w=0.0, mass=1.0, material=0) -> int:
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 2)
        h = ctypes.c_uint64()
        d = self._desc(x, y, rotation, vx, vy, w, mass, material)
        _check(lib.ag2d_world_add_polygon(self.h, ctypes.byref(d), v.ctypes.data, v.shape[0], ctypes.byref(h)))
        return int(h.value)

    def add_capsule(self, length, radius, x, y, rotation=0.0, vx=0.0, vy=0.0, w=0.0, mass=1.0, material=0) -> int:
        """A capsule body: a core of `length` along the body's x axis swept by `radius`."""
        h = ctypes.c_uint64()
        d = self._desc(x, y, rotation, vx, vy, w, mass, material)
        _check(lib.ag2d_world_add_capsule(self.h, ctypes.byref(d), length, radius, ctypes.byref(h)))
        return int(h.value)

    def create_body(self, x, y, rotation=0.0, vx=0.0, vy=0.0, w=0.0, mass=1.0, inertia=1.0, com=(0.0, 0.0)) -> int:
        """A body with explicit mass, inertia and local centre of mass and no collider yet (ObjectAPI::createBody)."""
        h = ctypes.c_uint64()
        d = self._desc(x, y, rotation, vx, vy, w, mass, 0)
        _check(lib.ag2d_world_create_body(self.h, ctypes.byref(d), inertia, com[0], com[1], ctypes.byref(h)))
        return int(h.value)

    def add_collider(self, body: int, shape: int, offset=(0.0, 0.0), rotation=0.0, material=0, radius=0.0,
                     width=0.0, height=0.0, length=0.0, vertices=None) -> int:
        """Attaches a collider to `body` at a local offset and rotation (ObjectAPI::create*Collider); returns its
        dense collider index. shape: CIRCLE (radius), BOX (width, height), POLYGON (convex `vertices`, recentred
        on their centroid), CAPSULE (length, radius)."""
        params = (ctypes.c_float * 2)()
        if shape == 0:
            params[0] = radius
        elif shape == 1:
            params[0], params[1] = width, height
        elif shape == 3:
            params[0], params[1] = length, radius
        xy, n = None, 0
        if vertices is not None:
            v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 2)
            xy, n = v.ctypes.data, v.shape[0]
        out = ctypes.c_uint32()
        _check(lib.ag2d_world_add_collider(self.h, body, shape, offset[0], offset[1], rotation, material, params,
                                          xy, n, ctypes.byref(out)))
        return int(out.value)

    def body_index(self, handle: int) -> int:
        return int(lib.ag2d_world_body_index(self.h, handle))

    # --- deferred body commands (ObjectAPI::destroyBody / setBody*): applied at the start of the next step ---
    def destroy_body(self, handle: int):
        _check(lib.ag2d_world_destroy_body(self.h, handle))

    def set_body_position(self, handle: int, x: float, y: float):
        _check(lib.ag2d_world_set_body_position(self.h, handle, x, y))

    def set_body_rotation(self, handle: int, rotation: float):
        _check(lib.ag2d_world_set_body_rotation(self.h, handle, rotation))

    def set_body_velocity(self, handle: int, vx: float, vy: float):
        _check(lib.ag2d_world_set_body_velocity(self.h, handle, vx, vy))

    def set_body_angular_velocity(self, handle: int, w: float):
        _check(lib.ag2d_world_set_body_angular_velocity(self.h, handle, w))

    def set_body_mass(self, handle: int, mass: float):
        _check(lib.ag2d_world_set_body_mass(self.h, handle, mass))

    def set_body_inertia(self, handle: int, inertia: float):
        _check(lib.ag2d_world_set_body_inertia(self.h, handle, inertia))

    def set_body_local_center_of_mass(self, handle: int, x: float, y: float):
        _check(lib.ag2d_world_set_body_local_center_of_mass(self.h, handle, x, y))

    def recompute_body_inertia(self, handle: int):
        _check(lib.ag2d_world_recompute_body_inertia(self.h, handle))

    def set_body_mass_from_density(self, handle: int, density: float):
        _check(lib.ag2d_world_set_body_mass_from_density(self.h, handle, density))

    def set_collider(self, collider: int, command: int, a: float, b: float = 0.0):
        """A deferred collider setter (COMMAND_COLLIDER_OFFSET ... COMMAND_CAPSULE_SHAPE) by dense index."""
        _check(lib.ag2d_world_set_collider(self.h, collider, command, a, b))

    def set_polygon_shape(self, collider: int, xy) -> bool:
        """ObjectAPI::setPolygonShape: new collider-local vertices for a polygon collider, applied at the next
        step. False, with nothing queued, for an outline the reference refuses (degenerate, concave, > 16)."""
        v = np.ascontiguousarray(np.asarray(xy, np.float32).reshape(-1, 2))
        code = lib.ag2d_world_set_polygon_shape(self.h, collider, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                v.shape[0])
        if code == ERR_INVALID_ARG:
            return False
        _check(code)
        return True

    def flush_commands(self):
        _check(lib.ag2d_world_flush_commands(self.h))

    # --- body constraints (ConstraintAPI, SimulationAPIs/ConstraintAPI.h:32-105) ---
    def create_joint(self, kind, body_a, body_b=0, anchor_a=(0.0, 0.0), anchor_b=(0.0, 0.0), rest_length=0.0,
                     stiffness=0.0, damping=0.0, target_speed=0.0, max_torque=0.0, axis=(1.0, 0.0),
                     limits=(0.0, 0.0), enable_limit=False) -> int:
        d = JointDesc(kind, 1 if enable_limit else 0, body_a, body_b, anchor_a[0], anchor_a[1], anchor_b[0],
                      anchor_b[1], rest_length, stiffness, damping, target_speed, max_torque, axis[0], axis[1],
                      limits[0], limits[1], 0.0, 0.0)
        out = ctypes.c_uint64()
        _check(lib.ag2d_world_create_joint(self.h, ctypes.byref(d), ctypes.byref(out)))
        return int(out.value)

    def create_spring(self, body_a, body_b, anchor_a, anchor_b, rest_length, stiffness, damping) -> int:
        return self.create_joint(JOINT_SPRING, body_a, body_b, anchor_a, anchor_b, rest_length, stiffness, damping)

    def create_revolute_joint(self, body_a, body_b, anchor_a, anchor_b, stiffness, damping) -> int:
        return self.create_joint(JOINT_REVOLUTE, body_a, body_b, anchor_a, anchor_b, 0.0, stiffness, damping)

    def create_motor(self, body, target_speed, max_torque) -> int:
        return self.create_joint(JOINT_MOTOR, body, 0, target_speed=target_speed, max_torque=max_torque)

    def destroy_joint(self, kind, handle):
        _check(lib.ag2d_world_destroy_joint(self.h, kind, handle))

    def set_joint(self, kind, handle, field, a, b=0.0):
        _check(lib.ag2d_world_set_joint(self.h, kind, handle, field, a, b))

    def joint(self, kind, handle) -> dict:
        d = JointDesc()
        _check(lib.ag2d_world_joint(self.h, kind, handle, ctypes.byref(d)))
        return {n: getattr(d, n) for n, _ in JointDesc._fields_}

    def joint_count(self, kind) -> int:
        n = ctypes.c_uint32()
        _check(lib.ag2d_world_joint_count(self.h, kind, ctypes.byref(n)))
        return int(n.value)

    def joint_handle(self, kind, index) -> int:
        out = ctypes.c_uint64()
        _check(lib.ag2d_world_joint_handle(self.h, kind, index, ctypes.byref(out)))
        return int(out.value)

    def set_joint_iterations(self, kind, iterations):
        _check(lib.ag2d_world_set_joint_iterations(self.h, kind, iterations))

    # --- collision events (Simulation::createCollisionCallback / destroyCollisionCallback /
    # setColliderCollisionCallback, Simulation.h:169-179) ---
    def create_collision_callback(self, fn) -> int:
        """Registers fn(event) (a CollisionEvent) to be called after each step for the events of the colliders that
        use the returned id; returns the id."""
        def trampoline(ev, _world, _user):
            fn(ev.contents)
        c = COLLISION_CALLBACK(trampoline)
        out = ctypes.c_uint16()
        _check(lib.ag2d_world_create_collision_callback(self.h, c, None, ctypes.byref(out)))
        self._callbacks = getattr(self, "_callbacks", {})
        self._callbacks[int(out.value)] = c   # the C function pointer lives as long as the id
        return int(out.value)

    def destroy_collision_callback(self, cb: int):
        _check(lib.ag2d_world_destroy_collision_callback(self.h, cb))
        getattr(self, "_callbacks", {}).pop(int(cb), None)

    def set_collider_collision_callback(self, collider: int, cb: int, threshold: float = 0.0):
        _check(lib.ag2d_world_set_collider_collision_callback(self.h, collider, cb, threshold))

    def set_collision_events(self, enable: bool):
        _check(lib.ag2d_world_set_collision_events(self.h, 1 if enable else 0))

    def collision_events(self) -> np.ndarray:
        """The last step's events (EVENT_DTYPE records), in the order they were dispatched."""
        n = ctypes.c_uint32()
        _check(lib.ag2d_world_collision_events(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(int(n.value), EVENT_DTYPE)
        if out.size:
            _check(lib.ag2d_world_collision_events(self.h, out.ctypes.data, out.size, ctypes.byref(n)))
        return out

    @classmethod
    def from_scene(cls, scene, device=0, **kw):
        w = cls(dt=scene.dt, velocity_iterations=scene.velocity_iterations,
                position_iterations=scene.position_iterations, gravity=scene.gravity, device=device, **kw)
        w.add_scene(scene)
        return w

    def add_scene(self, scene) -> np.ndarray:
        """Adds every body of a scene (ag2d.scenes.Scene) with one ag2d_world_add_bodies call; returns handles."""
        mats = np.asarray([self.add_material(*m) for m in scene.materials] or [0], dtype=np.uint32)
        n = scene.n
        descs = (BodyDesc * max(n, 1))()
        d = np.ctypeslib.as_array(ctypes.cast(descs, ctypes.POINTER(ctypes.c_uint8)),
                                  shape=(max(n, 1) * ctypes.sizeof(BodyDesc),)).view(_BODY_DESC_DTYPE)[:n]
        d["x"], d["y"], d["rotation"] = scene.px, scene.py, scene.rot
        d["vx"], d["vy"], d["w"], d["mass"] = scene.vx, scene.vy, scene.w, scene.mass
        m = scene.material.astype(np.int64)
        d["material"] = np.where(m >= 1, mats[np.clip(m - 1, 0, len(mats) - 1)], 0)
        kinds = np.ascontiguousarray(scene.kind, dtype=np.uint32)
        params = np.zeros((max(n, 1), 2), np.float32)
        circ, box, cap = kinds == scenes.CIRCLE, kinds == scenes.BOX, kinds == scenes.CAPSULE
        params[:n, 0] = np.where(circ, scene.radius, np.where(box | cap, scene.width, 0.0))
        params[:n, 1] = np.where(box, scene.height, np.where(cap, scene.radius, 0.0))
        offs = np.ascontiguousarray(scene.poly_offset, dtype=np.uint32)
        cnts = np.ascontiguousarray(scene.poly_count, dtype=np.uint32)
        xy = np.ascontiguousarray(scene.poly_xy, dtype=np.float32).reshape(-1)
        handles = np.zeros(max(n, 1), np.uint64)
        _check(lib.ag2d_world_add_bodies(self.h, n, descs, kinds.ctypes.data, params.ctypes.data, offs.ctypes.data,
                                         cnts.ctypes.data, xy.ctypes.data if xy.size else None,
                                         handles.ctypes.data))
        return handles[:n]

    def load_state(self, state: dict, prefix: str = "", materials=None, body_prefix=None, with_poses=False):
        """Replaces the world by a reference-layout state dict ("body.comX", "col.bodyIndex", ...)."""
        bp = prefix if body_prefix is None else body_prefix

        def g(k, dt):
            for p in ((bp,) if k.startswith("body.") else (prefix, "pre.")):
                if p + k in state:
                    return np.ascontiguousarray(np.asarray(state[p + k]), dtype=dt)
            raise KeyError(prefix + k)

        f, u = np.float32, np.uint32
        arrays = {
            "body_group_starts": g("body.groupStarts", u), "com_x": g("body.comX", f), "com_y": g("body.comY", f),
            "vel_x": g("body.velocityX", f), "vel_y": g("body.velocityY", f), "rotation": g("body.rotation", f),
            "angular_velocity": g("body.angularVelocity", f), "inv_mass": g("body.invMass", f),
            "inv_inertia": g("body.invInertia", f), "rot_cos": g("body.rotationCos", f),
            "rot_sin": g("body.rotationSin", f), "wrap_count": g("body.renderRotationWrapCount", f),
            "bound_radius": g("body.boundRadius", f), "sleep_timer": g("body.sleepingTimer", f),
            "sleep_island": g("body.sleepIslandId", u), "col_body": g("col.bodyIndex", u),
            "col_shape_type": g("col.shapeType", u), "col_shape_index": g("col.shapeIndex", u),
            "col_material": g("col.materialIndex", u), "col_com_offset_x": g("col.comOffsetX", f),
            "col_com_offset_y": g("col.comOffsetY", f), "col_local_rotation": g("col.localRotation", f),
            "circle_radius": g("circle.radius", f), "box_half_width": g("box.halfWidth", f),
            "box_half_height": g("box.halfHeight", f), "poly_count": g("poly.counts", u),
            "poly_vertices": g("poly.vertices", f), "poly_normals": g("poly.normals", f),
        }
        for k, name in (("capsule.halfLength", "capsule_half_length"), ("capsule.radius", "capsule_radius")):
            try:
                arrays[name] = g(k, f)
            except KeyError:
                arrays[name] = np.zeros(0, f)
        mats = np.ascontiguousarray(np.asarray(materials if materials is not None else [(1.0, 0.0, 0.0)],
                                               dtype=np.float32).reshape(-1, 3))
        arrays["materials"] = mats
        # Collider poses and AABBs as the state holds them, when it does (all four of a kind or none).
        for keys, names in ((("col.worldPosX", "col.worldPosY", "col.worldRotationCos", "col.worldRotationSin"),
                             ("col_world_x", "col_world_y", "col_world_cos", "col_world_sin")),
                            (("col.aabbMinX", "col.aabbMinY", "col.aabbMaxX", "col.aabbMaxY"),
                             ("col_aabb_min_x", "col_aabb_min_y", "col_aabb_max_x", "col_aabb_max_y"))):
            if with_poses and all(prefix + k in state for k in keys):
                for k, name in zip(keys, names):
                    arrays[name] = np.ascontiguousarray(np.asarray(state[prefix + k]), dtype=f)
        d = StateDesc()
        d.n_bodies = arrays["com_x"].size
        d.n_colliders = arrays["col_body"].size
        d.n_circles = arrays["circle_radius"].size
        d.n_boxes = arrays["box_half_width"].size
        d.n_polygons = arrays["poly_count"].size
        d.n_materials = mats.shape[0]
        d.n_capsules = arrays["capsule_half_length"].size
        for k, v in arrays.items():
            setattr(d, k, v.ctypes.data if v.size else None)
        self._keep = list(arrays.values())
        _check(lib.ag2d_world_load_state(self.h, ctypes.byref(d)))

    # --- stepping ---
    def step(self, steps: int = 1):
        _check(lib.ag2d_world_step(self.h, steps))

    def run_phase(self, phase: int):
        _check(lib.ag2d_world_run_phase(self.h, phase))

    def counters(self) -> dict:
        c = Counters()
        _check(lib.ag2d_world_counters(self.h, ctypes.byref(c)))
        return {n: (float(getattr(c, n)) if t is ctypes.c_double else int(getattr(c, n))) for n, t in Counters._fields_}

    def autotune(self, steps_per_candidate: int = 3) -> dict:
        """Launch-shape autotuner (solver team size, query and narrow block sizes); advances the world."""
        t = Tuning()
        _check(lib.ag2d_world_autotune(self.h, steps_per_candidate, ctypes.byref(t)))
        return {n: (float(getattr(t, n)) if k is ctypes.c_float else int(getattr(t, n))) for n, k in Tuning._fields_}

    def _query(self, shape, params, trees):
        p = np.ascontiguousarray(params, dtype=np.float32)
        n = ctypes.c_uint32()
        _check(lib.ag2d_world_query_shape(self.h, shape, p.ctypes.data, trees, None, 0, ctypes.byref(n)))
        out = np.empty(max(int(n.value), 1), np.uint32)
        _check(lib.ag2d_world_query_shape(self.h, shape, p.ctypes.data, trees, out.ctypes.data, out.size,
                                          ctypes.byref(n)))
        return out[:int(n.value)]

    def query_aabb(self, lo, hi, trees: int = TREE_ALL) -> np.ndarray:
        """Colliders whose AABB strictly overlaps [lo, hi] (BroadPhaseCollisionDetector::queryCollidersInShape
        with an AABBQuery), ascending indices."""
        return self._query(QUERY_AABB, [lo[0], lo[1], hi[0], hi[1]], trees)

    def query_circle(self, centre, radius: float, trees: int = TREE_ALL) -> np.ndarray:
        """Colliders whose AABB is within 'radius' of 'centre' (a CircleQuery), ascending indices."""
        return self._query(QUERY_CIRCLE, [centre[0], centre[1], radius], trees)

    def query_circle_contacts(self, centre, radius: float, trees: int = TREE_ALL):
        """(indices, signed distances) of the colliders the circle touches (findCollisionsInCircle over the circle
        query's colliders), ascending indices."""
        n = ctypes.c_uint32()
        args = (self.h, float(centre[0]), float(centre[1]), float(radius), trees)
        _check(lib.ag2d_world_query_circle_contacts(*args, None, None, 0, ctypes.byref(n)))
        idx = np.empty(max(int(n.value), 1), np.uint32)
        dist = np.empty(max(int(n.value), 1), np.float32)
        _check(lib.ag2d_world_query_circle_contacts(*args, idx.ctypes.data, dist.ctypes.data, idx.size,
                                                    ctypes.byref(n)))
        return idx[:int(n.value)], dist[:int(n.value)]

    def set_tuning(self, tuning: dict):
        """Applies launch shapes (a dict as autotune returns); results do not depend on them."""
        t = Tuning()
        for n, k in Tuning._fields_:
            if n in tuning:
                setattr(t, n, tuning[n])
        _check(lib.ag2d_world_set_tuning(self.h, ctypes.byref(t)))

    def set_profiling(self, enable: bool = True):
        _check(lib.ag2d_world_set_profiling(self.h, 1 if enable else 0))

    def phase_times(self) -> dict:
        """Cumulative device milliseconds and call counts per timed phase (profiling must be on)."""
        ms = np.zeros(len(TIMED_PHASES), np.float64)
        calls = np.zeros(len(TIMED_PHASES), np.uint64)
        _check(lib.ag2d_world_phase_times(self.h, ms.ctypes.data, calls.ctypes.data, len(TIMED_PHASES)))
        return {name: (float(ms[i]), int(calls[i])) for i, name in enumerate(TIMED_PHASES)}

    def stream(self) -> int:
        """cudaStream_t of the world's kernels (an integer handle)."""
        s = ctypes.c_void_p()
        _check(lib.ag2d_world_stream(self.h, ctypes.byref(s)))
        return int(s.value or 0)

    def counts(self):
        b, c = ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib.ag2d_world_body_count(self.h, ctypes.byref(b), ctypes.byref(c)))
        return int(b.value), int(c.value)

    # --- field access ---
    def field_bytes(self, field: int) -> int:
        """Bytes a read of `field` returns (body and collider fields: no device access)."""
        n = ctypes.c_uint64()
        _check(lib.ag2d_world_read(self.h, field, None, 0, ctypes.byref(n)))
        return int(n.value)

    def read(self, field: int, out: np.ndarray = None) -> np.ndarray:
        """A field as a host array; with `out` (any contiguous array large enough, page-locked for the fastest
        copy) the values land there and a view of its first bytes is returned."""
        if out is None:
            out = np.empty(self.field_bytes(field), dtype=np.uint8)
        ptr, cap = _out_bytes(out)
        n = ctypes.c_uint64()
        _check(lib.ag2d_world_read(self.h, field, ptr if cap else None, cap, ctypes.byref(n)))
        return _field_view(out.reshape(-1).view(np.uint8)[:int(n.value)], field)

    def read_async(self, field: int, out: np.ndarray) -> np.ndarray:
        """Queues a read of a body or collider field into page-locked `out` (ag2d.host_empty); the copy overlaps the
        steps that follow. The values are valid after read_wait()."""
        ptr, cap = _out_bytes(out)
        n = ctypes.c_uint64()
        _check(lib.ag2d_world_read_async(self.h, field, ptr, cap, ctypes.byref(n)))
        return _field_view(out.reshape(-1).view(np.uint8)[:int(n.value)], field)

    def read_wait(self):
        """Waits until every read_async of this world has landed."""
        _check(lib.ag2d_world_read_wait(self.h))

    def write(self, field: int, data: np.ndarray):
        if field in (MANIFOLDS, PREV_MANIFOLDS, ISLAND_MANIFOLDS):
            a = np.ascontiguousarray(data, dtype=MANIFOLD_DTYPE)
        elif field == PAIRS:
            a = np.ascontiguousarray(data, dtype=np.uint32).reshape(-1, 2)
        elif field in _U32_FIELDS:
            a = np.ascontiguousarray(data, dtype=np.uint32)
        else:
            a = np.ascontiguousarray(data, dtype=np.float32)
        _check(lib.ag2d_world_write(self.h, field, a.ctypes.data if a.size else None, a.nbytes))


class Batch:
    """Many independent worlds advanced together: their current states are packed into one world-segmented
    engine instance stepped by one launch sequence per step. The source worlds are copied, not advanced."""

    def __init__(self, worlds):
        worlds = list(worlds)
        arr = (ctypes.c_void_p * len(worlds))(*[w.h for w in worlds])
        h = ctypes.c_void_p()
        _check(lib.ag2d_batch_create(arr, len(worlds), ctypes.byref(h)))
        self._adopt(h)

    def _adopt(self, h):
        self.h = h
        n = ctypes.c_uint32()
        _check(lib.ag2d_batch_world_count(self.h, ctypes.byref(n)))
        self.n_worlds = int(n.value)
        e = ctypes.c_void_p()
        _check(lib.ag2d_batch_engine(self.h, ctypes.byref(e)))
        self.engine = World._borrowed(e, self)

    @classmethod
    def restore(cls, blob: np.ndarray, device: int = -1) -> "Batch":
        """A batch from a checkpoint (Batch.save); it steps on exactly as the saved batch does. A page-locked blob
        (ag2d.host_empty) goes over in one DMA per array."""
        ptr, nbytes = _out_bytes(blob)
        h = ctypes.c_void_p()
        _check(lib.ag2d_batch_restore(ptr, nbytes, device, ctypes.byref(h)))
        b = cls.__new__(cls)
        b._adopt(h)
        return b

    def load(self, blob: np.ndarray):
        """Replaces this batch's state by a checkpoint (same settings), reusing its device buffers."""
        ptr, nbytes = _out_bytes(blob)
        _check(lib.ag2d_batch_load(self.h, ptr, nbytes))

    def save(self, out: np.ndarray = None) -> np.ndarray:
        """Checkpoint of the whole batch as a uint8 array (page-locked unless `out` is given)."""
        n = ctypes.c_uint64()
        _check(lib.ag2d_batch_save(self.h, None, 0, ctypes.byref(n)))
        if out is None:
            out = host_empty(int(n.value))
        ptr, cap = _out_bytes(out)
        _check(lib.ag2d_batch_save(self.h, ptr, cap, ctypes.byref(n)))
        return out.reshape(-1).view(np.uint8)[:int(n.value)]

    def step(self, steps: int = 1):
        _check(lib.ag2d_batch_step(self.h, steps))

    def read(self, world: int, field: int, out: np.ndarray = None) -> np.ndarray:
        """A body field, collider field or the manifolds of one world, in that world's own indices."""
        n = ctypes.c_uint64()
        if out is None:
            _check(lib.ag2d_batch_read(self.h, world, field, None, 0, ctypes.byref(n)))
            out = np.empty(int(n.value), dtype=np.uint8)
        ptr, cap = _out_bytes(out)
        _check(lib.ag2d_batch_read(self.h, world, field, ptr if cap else None, cap, ctypes.byref(n)))
        buf = out.reshape(-1).view(np.uint8)[:int(n.value)]
        if field in (MANIFOLDS, PREV_MANIFOLDS, ISLAND_MANIFOLDS):
            return buf.view(MANIFOLD_DTYPE)
        return buf.view(np.uint32 if field in _U32_FIELDS else np.float32)

    def counters(self) -> dict:
        return self.engine.counters()

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "engine", None) is not None:
                self.engine.h = None
            lib.ag2d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request server: submitted worlds wait in arrival order, join the resident batch while
    their estimated device memory fits the budget, advance together in rounds of up to `steps_per_round` steps and
    leave with their final body state once their requested steps are done. Every request's result equals the same
    world stepped alone."""

    def __init__(self, memory_budget_bytes=8 << 30, steps_per_round=8, max_worlds=0, reserve_bodies=0, dt=1.0 / 60.0,
                 velocity_iterations=8, position_iterations=3, gravity=(0.0, -9.81), angular_damping=1.0,
                 sleep_speed=0.1, sleep_time=0.5, ccd=False, device=0):
        w = WorldSettings(dt, velocity_iterations, position_iterations, gravity[0], gravity[1], angular_damping,
                          sleep_speed, sleep_time, 1 if ccd else 0, device)
        s = ServerSettings(w, memory_budget_bytes, steps_per_round, max_worlds, reserve_bodies, 0)
        h = ctypes.c_void_p()
        _check(lib.ag2d_server_create(ctypes.byref(s), ctypes.byref(h)))
        self.h = h

    def submit(self, world: World, steps: int) -> int:
        """Queues a copy of the world's current state for `steps` steps; returns the request id."""
        r = ctypes.c_uint64()
        _check(lib.ag2d_server_submit(self.h, world.h, steps, ctypes.byref(r)))
        return int(r.value)

    def poll(self, request: int):
        """(state, latency_ms): REQUEST_WAITING / RUNNING / DONE; the latency once done, else -1."""
        st, lat = ctypes.c_int32(), ctypes.c_double()
        _check(lib.ag2d_server_poll(self.h, request, ctypes.byref(st), ctypes.byref(lat)))
        return int(st.value), float(lat.value)

    def wait_all(self, timeout_ms: float = -1.0):
        _check(lib.ag2d_server_wait_all(self.h, timeout_ms))

    def read(self, request: int, field: int) -> np.ndarray:
        """A body field of a finished request (positions, rotation, velocities, pose or state)."""
        n = ctypes.c_uint64()
        _check(lib.ag2d_server_read(self.h, request, field, None, 0, ctypes.byref(n)))
        buf = np.empty(int(n.value), dtype=np.uint8)
        _check(lib.ag2d_server_read(self.h, request, field, buf.ctypes.data if buf.size else None, buf.size,
                                    ctypes.byref(n)))
        return buf.view(np.uint32 if field in _U32_FIELDS else np.float32)

    def release(self, request: int):
        _check(lib.ag2d_server_release(self.h, request))

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib.ag2d_server_stats_get(self.h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            lib.ag2d_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
