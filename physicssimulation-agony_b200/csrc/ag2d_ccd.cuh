// Continuous collision detection (CollisionDetection/CCD/ContinuousCollisionDetector.cpp): a fast dynamic collider's
// "core" circle (radius coreFraction x its min extent, centred at the collider origin) is swept from the collider's
// pose before integration to its pose after it, against the static colliders inflated by the core radius. The
// earliest time of impact moves the body back along its own displacement. Translation only; velocities are kept.
//
// The ray casts restate castCircle / castBox / castPolygon (ContinuousCollisionDetector.cpp:41-203) with the same
// operation order; std::fmin / std::fmax are the glibc forms (rfminf / rfmaxf), std::sqrt is IEEE (-prec-sqrt).
#pragma once

#include "ag2d_math.cuh"

namespace ag2d {

constexpr float CCD_NO_HIT = 2.0f;
constexpr float CCD_FAST_FACTOR = 1.0f;        // ContinuousCollisionDetector::Settings::fastFactor
constexpr float CCD_CORE_FRACTION = 0.5f;      // ContinuousCollisionDetector::Settings::coreFraction
constexpr float CCD_MIN_DISPLACEMENT_SQ = 1e-8f;

// Ray from (mx, my) along (dx, dy) (|d|^2 = dd) against a circle of 'radius' at the origin: hit time < best.
__device__ __forceinline__ float ccd_cast_circle(float mx, float my, float dx, float dy, float dd, float radius,
                                                 float best)
{
    const float c = mx * mx + my * my - radius * radius;
    const float b = mx * dx + my * dy;
    if (c <= 0.0f || b >= 0.0f) return CCD_NO_HIT;   // inside or moving away
    if (c >= -2.0f * b * best) return CCD_NO_HIT;
    const float disc = b * b - dd * c;
    if (disc < 0.0f) return CCD_NO_HIT;
    return c / (sqrtf(disc) - b);
}

// Box of half extents (hw, hh) inflated by 'radius' (rounded corners), ray in the box frame.
__device__ __forceinline__ float ccd_cast_box(V2 q0, V2 dl, float dd, float hw, float hh, float radius, float best)
{
    const float sx = copysignf(1.0f, q0.x);
    const float sy = copysignf(1.0f, q0.y);
    const float qx = q0.x * sx;
    const float qy = q0.y * sy;
    const float vx = dl.x * sx;
    const float vy = dl.y * sy;
    const float w = hw + radius;
    const float h = hh + radius;
    const float gapX = qx - w;
    const float gapY = qy - h;
    if (gapX <= 0.0f && gapY <= 0.0f) return CCD_NO_HIT;   // starts inside
    float tx = 0.0f;
    if (gapX > 0.0f) {
        if (vx >= 0.0f || gapX >= best * -vx) return CCD_NO_HIT;
        tx = gapX / -vx;
    }
    float ty = 0.0f;
    if (gapY > 0.0f) {
        if (vy >= 0.0f || gapY >= best * -vy) return CCD_NO_HIT;
        ty = gapY / -vy;
    }
    const float t = rfmaxf(tx, ty);
    const float px = qx + vx * t;
    const float py = qy + vy * t;
    if (tx >= ty ? fabsf(py) > h : fabsf(px) > w) return CCD_NO_HIT;
    if (fabsf(px) > hw && fabsf(py) > hh)   // entry in a corner square: the rounded corner decides
        return ccd_cast_circle(qx - copysignf(hw, px), qy - copysignf(hh, py), vx, vy, dd, radius, best);
    return t;
}

// Convex polygon (local vertices / outward normals) inflated by 'radius': offset half-planes give the entry and
// exit times; an entry beyond its edge's span is decided by the rounded corner.
// castCapsule (ContinuousCollisionDetector.cpp:222-240): the slab on q0's side, then the two end circles.
__device__ __forceinline__ float ccd_cast_capsule(V2 q0, V2 dl, float dd, float halfLength, float capsuleRadius,
                                                  float radius, float best)
{
    const float inflated = capsuleRadius + radius;
    const float nvy = -copysignf(1.0f, q0.y) * dl.y;
    const float gap = fabsf(q0.y) - inflated;
    if (nvy > 0.0f && gap >= 0.0f && gap < best * nvy) {
        const float time = gap / nvy;
        if (fabsf(q0.x + dl.x * time) <= halfLength) return time;
    }
    const float t = rfminf(ccd_cast_circle(q0.x + halfLength, q0.y, dl.x, dl.y, dd, inflated, best), best);
    return rfminf(ccd_cast_circle(q0.x - halfLength, q0.y, dl.x, dl.y, dd, inflated, t), t);
}

__device__ __forceinline__ float ccd_cast_polygon(V2 q0, V2 dl, float dd, const float2* verts, const float2* normals,
                                                  uint32_t count, float radius, float best)
{
    float tEnter = 0.0f, tExit = best;
    uint32_t enterEdge = 0;
    float gaps[MAX_POLYGON_VERTICES];
    for (uint32_t i = 0; i < count; i++) {
        const V2 n = ld2(normals, i);
        const float speed = dot(n, dl);
        const float gap = dot(n, q0 - ld2(verts, i)) - radius;
        gaps[i] = gap;
        if (speed < 0.0f) {
            if (gap > 0.0f) {
                const float approach = -speed;
                if (gap >= tExit * approach) return CCD_NO_HIT;
                const float t = gap / approach;
                if (t > tEnter) { tEnter = t; enterEdge = i; }
            }
        } else if (gap > 0.0f) {
            return CCD_NO_HIT;   // outside and not approaching
        } else if (speed > 0.0f) {
            tExit = rfminf(tExit, -gap / speed);
        }
    }
    if (tEnter >= tExit) return CCD_NO_HIT;
    uint32_t edge = enterEdge;
    const bool startedInside = tEnter == 0.0f;
    if (startedInside) {
        float maxGap = -FLT_MAX;
        for (uint32_t i = 0; i < count; i++)
            if (gaps[i] > maxGap) { maxGap = gaps[i]; edge = i; }
    }
    const V2 p = q0 + dl * tEnter;
    const uint32_t next = edge + 1 == count ? 0u : edge + 1;
    const V2 a = ld2(verts, edge), b = ld2(verts, next);
    const V2 ab = b - a;
    const float u = dot(p - a, ab);
    if (u >= 0.0f && u <= dot(ab, ab)) return startedInside ? CCD_NO_HIT : tEnter;
    const V2 corner = u < 0.0f ? a : b;
    return ccd_cast_circle(q0.x - corner.x, q0.y - corner.y, dl.x, dl.y, dd, radius, tExit);
}

}  // namespace ag2d
