"""Algorithmic bytes per phase of the collision/contact step (the HBM roofline's numerator).

A phase's algorithmic bytes are the bytes its kernel must move between HBM and the SMs for the work it does, with
each input read once per pass and each output written once (no scratch): achieved GB/s = these bytes / the kernel's
measured time, and frac = achieved / the measured HBM copy bandwidth. Only the solver makes several dependent passes
over the same records (see SOLVE_VELOCITY_PER_ITERATION). Per-unit figures follow the device
layout (csrc/ag2d_world.cuh): body state float4 (16 B) + float4 (16 B) + cos/sin float2 (8 B); collider pose and
AABB float4 each; manifold 64 B; solver constraint 128 B.
"""
from __future__ import annotations

SHAPE_BYTES = {0: 4, 1: 8}          # circle radius; box half extents (polygons: see shape_bytes)


def polygon_bytes(nv: float) -> float:
    return 8.0 + 16.0 * nv             # offset + count, vertices + normals (float2 each)


def integrate_bytes(dynamic_bodies: float) -> float:
    # list index 4; read bvel, bpos 32, wrap count 4; write bvel, bpos 32, cos/sin 8, wrap count 4.
    return dynamic_bodies * 84.0


def pose_bytes(colliders: float, mean_shape_bytes: float) -> float:
    # list 4, owner 4, shape word 4, offsets 16, body pose 16 + cos/sin 8, shape data; write pose 16, rot 4, AABB 16.
    return colliders * (88.0 + mean_shape_bytes)


def narrow_bytes(pairs: float, mean_shape_bytes: float, manifolds: float) -> float:
    # pair 8; per side shape word 4, pose 16, shape data; hit flag 4; manifold slot 64 per hit.
    return pairs * (8.0 + 2.0 * (20.0 + mean_shape_bytes) + 4.0) + manifolds * 64.0


# Solver bytes per manifold. The velocity and position passes are Gauss-Seidel sweeps: each pass depends on the one
# before, so each reads its constraint again (the unit of the measurement specification: per manifold per velocity
# iteration 112 B of constraint, 48 B of two bodies' velocity and angular velocity read and written, 32 B of the two
# contacts' normal and tangent impulses read and written). Preparation, warm start, position passes and the
# impulse write-back are listed separately, each input read once within its pass.
SOLVE_VELOCITY_PER_ITERATION = 112 + 48 + 32
SOLVE_PREP = 64 + 16 + 2 * 32 + 112          # manifold, owners + materials, two bodies' state, constraint written
SOLVE_WARM = 32 + 48                         # impulses read, two bodies' velocities read and written
SOLVE_POSITION_PER_ITERATION = 48 + 48       # anchors, normal and penetration; two bodies' x, y, angle read+written
SOLVE_SCATTER = 16                           # accumulated impulses written back to the manifold


def solve_bytes_breakdown(manifolds: float, velocity_iterations: int, position_iterations: int) -> dict:
    """Algorithmic bytes of one solve, by pass: prep, warm, velocity (the measurement unit's 192 B per manifold per
    velocity iteration), position, scatter."""
    m = float(manifolds)
    return {"prep": m * SOLVE_PREP, "warm": m * SOLVE_WARM,
            "velocity": m * velocity_iterations * SOLVE_VELOCITY_PER_ITERATION,
            "position": m * position_iterations * SOLVE_POSITION_PER_ITERATION, "scatter": m * SOLVE_SCATTER}


def solve_bytes(manifolds: float, velocity_iterations: int, position_iterations: int) -> float:
    return float(sum(solve_bytes_breakdown(manifolds, velocity_iterations, position_iterations).values()))


def sort_bytes(keys: float) -> float:
    # histogram pass reads keys (4); four onesweep passes read and write key + value (16 each).
    return keys * (4.0 + 4 * 16.0)


def query_bytes(dynamic_colliders: float, pairs: float) -> float:
    # per query: leaf AABB 16, own index 4 + owner 4, count 4 (count pass) + offset 4; per pair written 8.
    return dynamic_colliders * 32.0 + pairs * 8.0


def broad_narrow_bytes_per_step(n: float, mean_shape_bytes: float, pairs: float, manifolds: float) -> float:
    """Bytes(C3) of the broad + narrow phase per step: per collider pose + AABB, Morton key, sort, LBVH build and
    query; per pair the narrow-phase inputs; per manifold the 64-byte record."""
    per_collider = (88.0 + mean_shape_bytes) + (16.0 + 8.0) + (4.0 + 4 * 16.0) + 52.0 + 32.0
    return n * per_collider + pairs * (8.0 + 2.0 * (20.0 + mean_shape_bytes) + 4.0) + manifolds * 64.0
