// Device-side fp32 arithmetic of the collision/contact pipeline, shared by every kernel.
//
// Each function reproduces one reference routine operation for operation (PS_AGONY2D, paths relative to
// PhysicsSimulation-Agony/PS_AGONY2D/). The library is compiled with --fmad=false, so a*b+c stays two roundings as
// in the reference's parity build; __fmaf_rn appears only where the reference's AVX2 path issues an FMA
// instruction (Simd::negMulAdd in the rotation wrap). sqrtf and '/' are IEEE-rounded (-prec-sqrt/-prec-div on).
//
// Where the reference's SIMD body and scalar tail compute differently, a 'simd' flag selects the variant: the
// reference processes a range [begin, end) in 8-lane AVX2 chunks, so element begin + k takes the SIMD path iff
// k < ((end - begin) & ~7).
#pragma once

#include <cfloat>
#include <cstdint>

namespace ag2d {

// Constants.h:7-14 — double constants rounded to float.
constexpr double FULL_PI = 3.14159265358979323846;
constexpr float HALF_PI_F = float(FULL_PI * 0.5);
constexpr float INV_HALF_PI_F = float(1.0 / (FULL_PI * 0.5));
constexpr float TWO_PI_F = float(FULL_PI * 2.0);
constexpr float INV_TWO_PI_F = float(1.0 / (FULL_PI * 2.0));

// FastCosSin.cpp:10-14.
constexpr float COEF0 = float(9.9999999999953215e-01);
constexpr float COEF1 = float(-1.6666666534403832e-01);
constexpr float COEF2 = float(8.3332302391869520e-03);
constexpr float COEF3 = float(-1.9818200679665358e-04);
constexpr float COEF4 = float(2.6182346015248291e-06);

// Narrow/Constants.h:7-37.
constexpr float ZERO_DIVISION_BOUNDARY = 1e-4f;
constexpr float ZERO_DIVISION_BOUNDARY_SQUARED = 1e-8f;
constexpr float SAT_EPSILON = 1e-4f;
constexpr uint32_t REFERENCE_BODY_TAG = 0x80000000u;

enum ShapeType : uint32_t { SHAPE_CIRCLE = 0, SHAPE_BOX = 1, SHAPE_POLYGON = 2, SHAPE_CAPSULE = 3 };
constexpr uint32_t CAPSULE_VERTEX_CONTACT_TAG = 0x40000000u;   // Narrow/Constants.h:40
constexpr float CAPSULE_PARALLEL_SIN_SQUARED = 1e-3f;          // Narrow/Constants.h:41
constexpr uint32_t MAX_POLYGON_VERTICES = 16;   // Limits.h:6

// std::fmax / std::fmin as glibc implements them on x86-64 (the reference's build): the first argument if it
// compares greater (resp. smaller) or the second is NaN, else the second. fmax(+0, -0) is -0.
__host__ __device__ __forceinline__ float rfmaxf(float a, float b) { return (a > b || b != b) ? a : b; }
__host__ __device__ __forceinline__ float rfminf(float a, float b) { return (a < b || b != b) ? a : b; }

// glm::clamp for scalars: min(max(x, lo), hi) with max(x, y) = (x < y) ? y : x and min(x, y) = (y < x) ? y : x.
__host__ __device__ __forceinline__ float glm_clamp(float x, float lo, float hi)
{
    const float t = (x < lo) ? lo : x;
    return (hi < t) ? hi : t;
}

__device__ __forceinline__ float xor_sign(float v, uint32_t bit) { return __uint_as_float(__float_as_uint(v) ^ bit); }

// FastCosSin::order5Array, one element (FastCosSin.cpp:26-109).
__device__ __forceinline__ void fast_cos_sin(float x, bool simd, float& out_cos, float& out_sin)
{
    const int q = int(x * INV_HALF_PI_F);                       // truncation (cvttps / int cast)
    const float u = x - float(q) * HALF_PI_F;
    const float mirror = float(q & 1);
    const float a = mirror * (HALF_PI_F - 2.0f * u) + u;
    const float a2 = a * a;
    float s = COEF4;
    s = s * a2 + COEF3;
    s = s * a2 + COEF2;
    s = s * a2 + COEF1;
    s = s * a2 + COEF0;
    s = s * a;
    s = (s < 1.0f) ? s : 1.0f;                                  // min(sinMag, 1)
    const float c = sqrtf(1.0f - s * s);
    if (simd) {
        out_sin = xor_sign(s, uint32_t(q & 2) << 30);
        out_cos = xor_sign(c, uint32_t((q + 1) & 2) << 30);
    } else {
        const float sinSign = 1.0f - 2.0f * float(q >> 1);
        const float cosSign = 1.0f - 2.0f * float(((q + 1) >> 1) & 1);
        out_sin = sinSign * s;
        out_cos = cosSign * c;
    }
}

// wrapBodyRotations / wrapColliderRotations, one element (SimulationImpl/LeftOutFunctions.cpp:13-102).
// Returns the wrapped angle in [0, 2 pi]; 'wraps' receives the whole-turn count removed.
__device__ __forceinline__ float wrap_angle(float rot, bool simd, float& wraps)
{
    float wc;
    if (simd) {
        wc = truncf(rot * (1.0f / TWO_PI_F));
        rot = __fmaf_rn(-wc, TWO_PI_F, rot);                    // _mm256_fnmadd_ps
        if (rot < 0.0f) { rot += TWO_PI_F; wc -= 1.0f; } else { rot += 0.0f; wc -= 0.0f; }
    } else {
        wc = truncf(rot * INV_TWO_PI_F);
        rot -= wc * TWO_PI_F;
        const float neg = float(rot < 0.0f);
        rot += neg * TWO_PI_F;
        wc -= neg;
    }
    wraps = wc;
    return rot;
}

__device__ __forceinline__ uint32_t part1by1(uint32_t x)
{
    x &= 0x0000ffffu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

// ---------------------------------------------------------------------------------------------------------------
// Narrow phase (CollisionDetection/Narrow/*). Vectors are (x, y) pairs of floats; glm::dot(a, b) = a.x*b.x + a.y*b.y.
// ---------------------------------------------------------------------------------------------------------------

struct V2 { float x, y; };
__device__ __forceinline__ V2 v2(float x, float y) { return V2{x, y}; }
__device__ __forceinline__ float dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ V2 operator-(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ V2 operator+(V2 a, V2 b) { return V2{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ V2 operator*(V2 a, float s) { return V2{a.x * s, a.y * s}; }
__device__ __forceinline__ V2 operator-(V2 a) { return V2{-a.x, -a.y}; }
__device__ __forceinline__ uint32_t next_index(uint32_t i, uint32_t n) { return i + 1 == n ? 0u : i + 1; }

// One collider as the narrow phase sees it: world pose and shape parameters.
struct ColliderView {
    V2 pos;
    float c, s;            // world rotation cos/sin
    uint32_t type;
    float r;               // circle radius; capsule radius
    float hw, hh;          // box half extents; capsule: hw = half length of the core
    const float2* verts;   // polygon, body-local (centred on the piece centroid)
    const float2* normals;
    uint32_t nv;
};

// Manifold as produced by a method (before warm start).
struct Contact {
    V2 n;
    float depth;
    uint32_t count;
    V2 p[2];
    uint32_t id[2];
};

// clipSegment (HelperMethods.h:36-52). True if both points are outside the plane.
__device__ __forceinline__ bool clip_segment(V2& p1, V2& p2, V2 planePoint, V2 planeNormal)
{
    const float d1 = dot(p1 - planePoint, planeNormal);
    const float d2 = dot(p2 - planePoint, planeNormal);
    if (d1 >= 0.0f && d2 >= 0.0f) return false;
    if (d1 < 0.0f && d2 < 0.0f) return true;
    const float t = d1 / (d1 - d2);
    const V2 dir = p2 - p1;
    const V2 inter = p1 + dir * t;
    if (d1 >= 0.0f) p2 = inter; else p1 = inter;
    return false;
}

// flipSignIfNegative (HelperMethods.h:26-34).
__device__ __forceinline__ V2 flip_if_negative(V2 v, float sign)
{
    const uint32_t bit = __float_as_uint(sign) & 0x80000000u;
    return V2{xor_sign(v.x, bit), xor_sign(v.y, bit)};
}

__device__ __forceinline__ V2 ld2(const float2* p, uint32_t k)
{
    const float2 f = __ldg(p + k);
    return V2{f.x, f.y};
}

// collisionCircleCircle (CircleCircle.cpp:14-179).
__device__ __forceinline__ bool collide_circle_circle(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const V2 d = B.pos - A.pos;
    const float rs = A.r + B.r;
    const float sq = dot(d, d);
    if (!(sq < rs * rs)) return false;
    const float dist = sqrtf(sq);
    V2 n;
    if (dist < ZERO_DIVISION_BOUNDARY) n = v2(1.0f, 0.0f);
    else { const float inv = 1.0f / dist; n = d * inv; }
    out.n = n; out.depth = rs - dist; out.count = 1;
    out.p[0] = A.pos + n * A.r; out.id[0] = 0;
    return true;
}

// collisionCircleBox (CircleBox.cpp:9-120). A circle, B box.
__device__ __forceinline__ bool collide_circle_box(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const float cB = B.c, sB = B.s, hw = B.hw, hh = B.hh, rA = A.r;
    const V2 dg = A.pos - B.pos;
    const V2 loc = v2(dg.x * cB + dg.y * sB, dg.x * -sB + dg.y * cB);
    const V2 cl = v2(rfminf(rfmaxf(loc.x, -hw), hw), rfminf(rfmaxf(loc.y, -hh), hh));
    const V2 dl = cl - loc;
    const float sq = dot(dl, dl);
    if (sq >= rA * rA) return false;
    out.count = 1;
    if (sq >= ZERO_DIVISION_BOUNDARY_SQUARED) {
        const float dist = sqrtf(sq);
        const float inv = 1.0f / dist;
        const V2 wd = v2(cB * dl.x - sB * dl.y, sB * dl.x + cB * dl.y);
        const V2 n = wd * inv;
        uint32_t id = 0;
        id |= uint32_t(loc.x > hw);
        id |= uint32_t(loc.x < -hw) << 1;
        id |= uint32_t(loc.y > hh) << 2;
        id |= uint32_t(loc.y < -hh) << 3;
        out.n = n; out.depth = rA - dist; out.p[0] = A.pos + n * rA; out.id[0] = id;
        return true;
    }
    const float dx = hw - fabsf(loc.x);
    const float dy = hh - fabsf(loc.y);
    const bool useY = dy <= dx;
    const float minPen = useY ? dy : dx;
    const float sign = copysignf(1.0f, useY ? loc.y : loc.x);
    const V2 nl = v2(useY ? 0.0f : sign, useY ? sign : 0.0f);
    const uint32_t id = 1u << (uint32_t(sign <= 0.0f) + (uint32_t(useY) << 1));
    const V2 n = -v2(cB * nl.x - sB * nl.y, sB * nl.x + cB * nl.y);
    out.n = n; out.depth = rA + minPen; out.p[0] = A.pos + n * rA; out.id[0] = id;
    return true;
}

// collisionCirclePolygon (CirclePolygon.cpp:10-103), findSupportEdge / closestPointOnSegment
// (HelperMethods.h:73-109). A circle, B polygon.
__device__ __forceinline__ bool collide_circle_polygon(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const float cB = B.c, sB = B.s, rA = A.r;
    const V2 dg = A.pos - B.pos;
    const V2 loc = v2(dg.x * cB + dg.y * sB, dg.x * -sB + dg.y * cB);
    float maxSep = -FLT_MAX;
    uint32_t edge = 0;
    for (uint32_t i = 0; i < B.nv; i++) {
        const float sep = dot(ld2(B.normals, i), loc - ld2(B.verts, i));
        if (sep > rA) return false;
        if (sep > maxSep) { maxSep = sep; edge = i; }
    }
    V2 nl;
    float separation;
    if (maxSep >= ZERO_DIVISION_BOUNDARY) {
        const V2 va = ld2(B.verts, edge), vb = ld2(B.verts, next_index(edge, B.nv));
        const V2 ab = vb - va;
        const float denom = dot(ab, ab);
        V2 cp;
        if (denom < ZERO_DIVISION_BOUNDARY_SQUARED) cp = va;
        else {
            const float t = dot(loc - va, ab) / denom;
            cp = va + ab * rfminf(rfmaxf(t, 0.0f), 1.0f);
        }
        const V2 cpd = loc - cp;
        const float d2 = dot(cpd, cpd);
        if (d2 > rA * rA) return false;
        if (d2 < ZERO_DIVISION_BOUNDARY_SQUARED) { separation = 0.0f; nl = ld2(B.normals, edge); }
        else { separation = sqrtf(d2); nl = cpd * (1.0f / separation); }
    } else {
        nl = ld2(B.normals, edge);
        separation = maxSep;
    }
    const V2 n = -v2(cB * nl.x - sB * nl.y, sB * nl.x + cB * nl.y);
    out.n = n; out.depth = rA - separation; out.count = 1; out.p[0] = A.pos + n * rA; out.id[0] = edge;
    return true;
}

// collisionBoxBox (BoxBox.cpp:13-227).
__device__ __forceinline__ bool collide_box_box(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const float cA = A.c, sA = A.s, cB = B.c, sB = B.s;
    const float hwA = A.hw, hhA = A.hh, hwB = B.hw, hhB = B.hh;
    const V2 rightA = v2(cA, sA), upA = v2(-sA, cA), rightB = v2(cB, sB), upB = v2(-sB, cB);
    const float relCos = cA * cB + sA * sB;
    const float relSin = cA * sB - sA * cB;
    const float arc = fabsf(relCos), ars = fabsf(relSin);
    const V2 cd = B.pos - A.pos;
    const float hwL[4] = {hwB, hwB, hwA, hwA}, hhL[4] = {hhB, hhB, hhA, hhA}, hwhL[4] = {hwA, hhA, hwB, hhB};
    const float cs1[4] = {arc, ars, arc, ars}, cs2[4] = {ars, arc, ars, arc};
    const float axX[4] = {cA, -sA, cB, -sB}, axY[4] = {sA, cA, sB, cB};
    float ov[4], cdoa[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float rsum = hwL[k] * cs1[k] + hhL[k] * cs2[k] + hwhL[k];
        cdoa[k] = cd.x * axX[k] + cd.y * axY[k];
        ov[k] = rsum - fabsf(cdoa[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) if (ov[k] < 0.0f) return false;
    const float depth = rfminf(rfminf(ov[0], ov[1]), rfminf(ov[2], ov[3]));
    const uint32_t n0 = ov[0] != depth;
    const uint32_t n01 = n0 & uint32_t(ov[1] != depth);
    const uint32_t n012 = n01 & uint32_t(ov[2] != depth);
    const uint32_t best = n0 + n01 + n012;
    float bestAxX, bestAxY, bestCdoa;
    switch (best) {   // register-friendly indexing
    case 0: bestAxX = axX[0]; bestAxY = axY[0]; bestCdoa = cdoa[0]; break;
    case 1: bestAxX = axX[1]; bestAxY = axY[1]; bestCdoa = cdoa[1]; break;
    case 2: bestAxX = axX[2]; bestAxY = axY[2]; bestCdoa = cdoa[2]; break;
    default: bestAxX = axX[3]; bestAxY = axY[3]; bestCdoa = cdoa[3]; break;
    }
    const V2 normal = flip_if_negative(v2(bestAxX, bestAxY), bestCdoa);
    const bool refIsA = best < 2;
    const V2 posRef = refIsA ? A.pos : B.pos, posInc = refIsA ? B.pos : A.pos;
    const float hwRef = refIsA ? hwA : hwB, hhRef = refIsA ? hhA : hhB;
    const float hwInc = refIsA ? hwB : hwA, hhInc = refIsA ? hhB : hhA;
    const V2 rightRef = refIsA ? rightA : rightB, upRef = refIsA ? upA : upB;
    const V2 rightInc = refIsA ? rightB : rightA, upInc = refIsA ? upB : upA;
    const V2 refNormal = refIsA ? normal : -normal;
    const float sign = copysignf(1.0f, refIsA ? bestCdoa : -bestCdoa);
    const bool useX = best == 0 || best == 2;
    V2 rfc, sideDir;
    if (useX) { rfc = posRef + rightRef * (sign * hwRef); sideDir = upRef; }
    else { rfc = posRef + upRef * (sign * hhRef); sideDir = rightRef; }
    const V2 eo = sideDir * (useX ? hhRef : hwRef);
    const V2 refStart = rfc + eo, refEnd = rfc - eo;
    V2 c0, c1;
    {
        const bool axisIsUp = (best & 1u) != 0;
        const float sideTerm = (best == 0 || best == 3) ? -relSin : relSin;
        const float dotX = sign * (axisIsUp ? sideTerm : relCos);
        const float dotY = sign * (axisIsUp ? relCos : sideTerm);
        const bool useXi = fabsf(dotX) > fabsf(dotY);
        const float incSign = -copysignf(1.0f, useXi ? dotX : dotY);
        V2 fc, off;
        if (useXi) { fc = posInc + rightInc * (incSign * hwInc); off = upInc * hhInc; }
        else { fc = posInc + upInc * (incSign * hhInc); off = rightInc * hwInc; }
        c0 = fc + off; c1 = fc - off;
    }
    if (clip_segment(c0, c1, refStart, -sideDir)) return false;
    if (clip_segment(c0, c1, refEnd, sideDir)) return false;
    const float refPlaneDist = dot(rfc, refNormal);
    const uint32_t idBase = best << 1;
    uint32_t cnt = 0;
    if (dot(c0, refNormal) <= refPlaneDist + SAT_EPSILON) { out.p[cnt] = c0; out.id[cnt] = idBase | 0u; cnt++; }
    if (dot(c1, refNormal) <= refPlaneDist + SAT_EPSILON) { out.p[cnt] = c1; out.id[cnt] = idBase | 1u; cnt++; }
    if (cnt == 0) return false;
    out.n = normal; out.depth = depth; out.count = cnt;
    return true;
}

// collisionBoxPolygon (BoxPolygon.cpp:14-319). A box, B polygon; works in the polygon's frame.
__device__ __forceinline__ bool collide_box_polygon(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const float cA = A.c, sA = A.s, cB = B.c, sB = B.s, hwA = A.hw, hhA = A.hh;
    const uint32_t nv = B.nv;
    const V2 rightB = v2(cB, sB), upB = v2(-sB, cB);
    const float relCos = cA * cB + sA * sB;
    const float relSin = cA * sB - sA * cB;
    const V2 rA = v2(relCos, -relSin), uA = v2(relSin, relCos);
    const V2 dBA = A.pos - B.pos;
    const V2 bc = v2(dot(dBA, rightB), dot(dBA, upB));
    V2 nl;
    float depth, bestFacing, pcxd, pcyd;
    int bestType;
    uint32_t bestIndex = 0;
    {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (uint32_t k = 0; k < nv; k++) { const float p = dot(ld2(B.verts, k), rA); mn = rfminf(mn, p); mx = rfmaxf(mx, p); }
        const float bcp = dot(bc, rA);
        mn -= bcp; mx -= bcp;
        const float overlap = hwA + rfminf(-mn, mx);
        if (overlap < 0.0f) return false;
        pcxd = mn + mx;
        depth = overlap; nl = flip_if_negative(rA, pcxd); bestType = 0; bestFacing = -fabsf(pcxd);
    }
    {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (uint32_t k = 0; k < nv; k++) { const float p = dot(ld2(B.verts, k), uA); mn = rfminf(mn, p); mx = rfmaxf(mx, p); }
        const float bcp = dot(bc, uA);
        mn -= bcp; mx -= bcp;
        const float overlap = hhA + rfminf(-mn, mx);
        if (overlap < 0.0f) return false;
        pcyd = mn + mx;
        const float facing = -fabsf(pcyd);
        if (overlap < depth || (overlap == depth && facing < bestFacing)) {
            depth = overlap; nl = flip_if_negative(uA, pcyd); bestType = 1; bestFacing = facing;
        }
    }
    const V2 pcr = v2(pcxd * rA.x + pcyd * uA.x, pcxd * rA.y + pcyd * uA.y);
    for (uint32_t i = 0; i < nv; i++) {
        const V2 ax = ld2(B.normals, i);
        const float boxRadius = hwA * fabsf(dot(ax, rA)) + hhA * fabsf(dot(ax, uA));
        const float bcp = dot(bc, ax);
        const float overlap = dot(ax, ld2(B.verts, i)) - (bcp - boxRadius);
        if (overlap < 0.0f) return false;
        const float facing = dot(ax, pcr);
        if (overlap < depth || (overlap == depth && facing < bestFacing)) {
            depth = overlap; nl = -ax; bestType = 2; bestIndex = i; bestFacing = facing;
        }
    }
    const bool refIsBox = bestType != 2;
    V2 rnl, rfc, sd, rs, re, c0, c1;
    uint32_t ie, ie2;
    if (refIsBox) {
        rnl = nl;
        const bool useX = bestType == 0;
        const float sign = useX ? dot(rnl, rA) : dot(rnl, uA);
        if (useX) { rfc = bc + rA * (sign * hwA); sd = uA; }
        else { rfc = bc + uA * (sign * hhA); sd = rA; }
        const V2 eo = sd * (useX ? hhA : hwA);
        rs = rfc + eo; re = rfc - eo;
        ie = 0;
        float minDot = FLT_MAX;
        for (uint32_t i = 0; i < nv; i++) {
            const float d = dot(rnl, ld2(B.normals, i));
            if (d < minDot) { minDot = d; ie = i; }
        }
        ie2 = next_index(ie, nv);
        c0 = ld2(B.verts, ie); c1 = ld2(B.verts, ie2);
    } else {
        rnl = -nl;
        const uint32_t i0 = bestIndex, i1 = next_index(i0, nv);
        rs = ld2(B.verts, i0); re = ld2(B.verts, i1);
        rfc = (rs + re) * 0.5f;
        const V2 edge = re - rs;
        const float len2 = dot(edge, edge);
        sd = edge * (-1.0f / sqrtf(len2));
        const float dotX = dot(rnl, rA), dotY = dot(rnl, uA);
        const bool useX = fabsf(dotX) > fabsf(dotY);
        const float sign = -copysignf(1.0f, useX ? dotX : dotY);
        // BOX_INCIDENT_EDGE_IDS[useX][sign > 0] (Narrow/Constants.h:34-37): {{1,2},{0,3}}, {{3,2},{0,1}}.
        const bool pos = sign > 0.0f;
        ie = pos ? 0u : (useX ? 3u : 1u);
        ie2 = pos ? (useX ? 1u : 3u) : 2u;
        V2 fc, off;
        if (useX) { fc = bc + rA * (sign * hwA); off = uA * hhA; }
        else { fc = bc + uA * (sign * hhA); off = rA * hwA; }
        c0 = fc + off; c1 = fc - off;
    }
    if (clip_segment(c0, c1, rs, -sd)) return false;
    if (clip_segment(c0, c1, re, sd)) return false;
    const uint32_t tag = refIsBox ? REFERENCE_BODY_TAG : 0u;
    const float refPlaneDist = dot(rfc, rnl);
    uint32_t cnt = 0;
    if (dot(c0, rnl) <= refPlaneDist + SAT_EPSILON) {
        out.p[cnt] = (B.pos + rightB * c0.x) + upB * c0.y; out.id[cnt] = tag | ie; cnt++;
    }
    if (dot(c1, rnl) <= refPlaneDist + SAT_EPSILON) {
        out.p[cnt] = (B.pos + rightB * c1.x) + upB * c1.y; out.id[cnt] = tag | ie2; cnt++;
    }
    if (cnt == 0) return false;
    out.n = rightB * nl.x + upB * nl.y; out.depth = depth; out.count = cnt;
    return true;
}

// collisionPolygonPolygon (PolygonPolygon.cpp:18-235). B's vertices are brought into A's frame.
__device__ __forceinline__ bool collide_polygon_polygon(const ColliderView& A, const ColliderView& B, Contact& out)
{
    V2 vB[MAX_POLYGON_VERTICES];
    const float cA = A.c, sA = A.s, cB = B.c, sB = B.s;
    const uint32_t nA = A.nv, nB = B.nv;
    const V2 rightA = v2(cA, sA), upA = v2(-sA, cA);
    const V2 cd = B.pos - A.pos;
    const V2 bdl = v2(dot(cd, rightA), dot(cd, upA));
    const float relCos = cA * cB + sA * sB;
    const float relSin = cA * sB - sA * cB;
    for (uint32_t i = 0; i < nB; i++) {
        const V2 v = ld2(B.verts, i);
        vB[i] = v2(bdl.x + relCos * v.x - relSin * v.y, bdl.y + relSin * v.x + relCos * v.y);
    }
    V2 nl = v2(0.0f, 0.0f);
    float depth = FLT_MAX, bestFacing = FLT_MAX;
    bool bestIsB = false;
    uint32_t bestIndex = 0;
    for (uint32_t i = 0; i < nA; i++) {
        const V2 ax = ld2(A.normals, i);
        float minB = FLT_MAX;
        for (uint32_t j = 0; j < nB; j++) minB = rfminf(minB, dot(vB[j], ax));
        const float overlap = dot(ld2(A.verts, i), ax) - minB;
        if (overlap < 0.0f) return false;
        const float facing = -dot(ax, bdl);
        if (overlap > depth) continue;
        if (overlap < depth || facing < bestFacing) { depth = overlap; nl = ax; bestIsB = false; bestIndex = i; bestFacing = facing; }
    }
    for (uint32_t i = 0; i < nB; i++) {
        const V2 nb = ld2(B.normals, i);
        const V2 ax = v2(relCos * nb.x - relSin * nb.y, relSin * nb.x + relCos * nb.y);
        float minA = FLT_MAX;
        for (uint32_t j = 0; j < nA; j++) minA = rfminf(minA, dot(ld2(A.verts, j), ax));
        const float overlap = dot(vB[i], ax) - minA;
        if (overlap < 0.0f) return false;
        const float facing = dot(ax, bdl);
        if (overlap > depth) continue;
        if (overlap < depth || facing < bestFacing) { depth = overlap; nl = -ax; bestIsB = true; bestIndex = i; bestFacing = facing; }
    }
    const bool refIsA = !bestIsB;
    const uint32_t refCount = refIsA ? nA : nB, incCount = refIsA ? nB : nA;
    const V2 rnl = refIsA ? nl : -nl;
    const uint32_t i0 = bestIndex, i1 = next_index(i0, refCount);
    const V2 rs = refIsA ? ld2(A.verts, i0) : vB[i0];
    const V2 re = refIsA ? ld2(A.verts, i1) : vB[i1];
    const V2 rfc = (rs + re) * 0.5f;
    const V2 edge = re - rs;
    const float len2 = dot(edge, edge);
    const V2 sideDir = edge * (1.0f / sqrtf(len2));
    uint32_t ie = 0;
    float minDot = FLT_MAX;
    for (uint32_t i = 0; i < incCount; i++) {
        V2 n;
        if (refIsA) { const V2 nb = ld2(B.normals, i); n = v2(relCos * nb.x - relSin * nb.y, relSin * nb.x + relCos * nb.y); }
        else n = ld2(A.normals, i);
        const float d = dot(rnl, n);
        if (d < minDot) { minDot = d; ie = i; }
    }
    const uint32_t ie2 = next_index(ie, incCount);
    V2 c0 = refIsA ? vB[ie] : ld2(A.verts, ie);
    V2 c1 = refIsA ? vB[ie2] : ld2(A.verts, ie2);
    if (clip_segment(c0, c1, rs, sideDir)) return false;
    if (clip_segment(c0, c1, re, -sideDir)) return false;
    const float refPlaneDist = dot(rfc, rnl);
    const uint32_t tag = refIsA ? REFERENCE_BODY_TAG : 0u;
    uint32_t cnt = 0;
    if (dot(c0, rnl) <= refPlaneDist + SAT_EPSILON) {
        out.p[cnt] = (A.pos + rightA * c0.x) + upA * c0.y; out.id[cnt] = tag | ie; cnt++;
    }
    if (dot(c1, rnl) <= refPlaneDist + SAT_EPSILON) {
        out.p[cnt] = (A.pos + rightA * c1.x) + upA * c1.y; out.id[cnt] = tag | ie2; cnt++;
    }
    if (cnt == 0) return false;
    out.n = rightA * nl.x + upA * nl.y; out.depth = depth; out.count = cnt;
    return true;
}

// collisionPolygonPolygon for one pair on a group of NARROW_GROUP lanes (lane = this lane's index in the group,
// mask = the group's lanes in the warp). Lanes share the two polygons' vertices (A local, B in A's frame) through
// the group's shared-memory tiles sA / sB, each lane projects its own axes, and group shuffles pick the separating
// axis and the incident edge. The sequential choice keeps the axis with the smallest (overlap, facing), the first
// one on ties (A's axes before B's), and the incident edge with the smallest dot, the first on ties: exactly the
// lexicographic minima the reductions below take, so the result equals collide_polygon_polygon bit for bit. Every
// lane returns the hit flag; the contact is valid on lane 0 of the group.
constexpr uint32_t NARROW_GROUP = 8;

__device__ __forceinline__ bool sat_better(float ov, float fac, uint32_t ord, float bov, float bfac, uint32_t bord)
{
    if (ov != bov) return ov < bov;
    if (fac != bfac) return fac < bfac;
    return ord < bord;
}

__device__ __forceinline__ bool collide_polygon_polygon_group(const ColliderView& A, const ColliderView& B,
                                                              Contact& out, uint32_t lane, uint32_t mask,
                                                              V2* sA, V2* sB)
{
    const float cA = A.c, sAn = A.s, cB = B.c, sBn = B.s;
    const uint32_t nA = A.nv, nB = B.nv;
    const V2 rightA = v2(cA, sAn), upA = v2(-sAn, cA);
    const V2 cd = B.pos - A.pos;
    const V2 bdl = v2(dot(cd, rightA), dot(cd, upA));
    const float relCos = cA * cB + sAn * sBn;
    const float relSin = cA * sBn - sAn * cB;
    for (uint32_t k = lane; k < nB; k += NARROW_GROUP) {
        const V2 v = ld2(B.verts, k);
        sB[k] = v2(bdl.x + relCos * v.x - relSin * v.y, bdl.y + relSin * v.x + relCos * v.y);
    }
    for (uint32_t k = lane; k < nA; k += NARROW_GROUP) sA[k] = ld2(A.verts, k);
    __syncwarp(mask);
    bool separated = false;
    float bov = FLT_MAX, bfac = FLT_MAX;
    uint32_t bord = 0xFFFFFFFFu;
    for (uint32_t i = lane; i < nA; i += NARROW_GROUP) {
        const V2 ax = ld2(A.normals, i);
        float minB = FLT_MAX;
        for (uint32_t j = 0; j < nB; j++) minB = rfminf(minB, dot(sB[j], ax));
        const float overlap = dot(sA[i], ax) - minB;
        if (overlap < 0.0f) separated = true;
        const float facing = -dot(ax, bdl);
        if (sat_better(overlap, facing, i, bov, bfac, bord)) { bov = overlap; bfac = facing; bord = i; }
    }
    for (uint32_t i = lane; i < nB; i += NARROW_GROUP) {
        const V2 nb = ld2(B.normals, i);
        const V2 ax = v2(relCos * nb.x - relSin * nb.y, relSin * nb.x + relCos * nb.y);
        float minA = FLT_MAX;
        for (uint32_t j = 0; j < nA; j++) minA = rfminf(minA, dot(sA[j], ax));
        const float overlap = dot(sB[i], ax) - minA;
        if (overlap < 0.0f) separated = true;
        const float facing = dot(ax, bdl);
        const uint32_t ord = MAX_POLYGON_VERTICES + i;
        if (sat_better(overlap, facing, ord, bov, bfac, bord)) { bov = overlap; bfac = facing; bord = ord; }
    }
    if (__any_sync(mask, separated)) return false;
#pragma unroll
    for (uint32_t o = NARROW_GROUP / 2; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(mask, bov, o), fac = __shfl_xor_sync(mask, bfac, o);
        const uint32_t ord = __shfl_xor_sync(mask, bord, o);
        if (sat_better(ov, fac, ord, bov, bfac, bord)) { bov = ov; bfac = fac; bord = ord; }
    }
    const bool refIsA = bord < MAX_POLYGON_VERTICES;
    const uint32_t bestIndex = refIsA ? bord : bord - MAX_POLYGON_VERTICES;
    V2 nl;
    if (refIsA) {
        nl = ld2(A.normals, bestIndex);
    } else {
        const V2 nb = ld2(B.normals, bestIndex);
        nl = -v2(relCos * nb.x - relSin * nb.y, relSin * nb.x + relCos * nb.y);
    }
    const float depth = bov;
    const uint32_t refCount = refIsA ? nA : nB, incCount = refIsA ? nB : nA;
    const V2 rnl = refIsA ? nl : -nl;
    float bd = FLT_MAX;
    uint32_t bi = 0xFFFFFFFFu;
    for (uint32_t i = lane; i < incCount; i += NARROW_GROUP) {
        V2 n;
        if (refIsA) { const V2 nb = ld2(B.normals, i); n = v2(relCos * nb.x - relSin * nb.y, relSin * nb.x + relCos * nb.y); }
        else n = ld2(A.normals, i);
        const float d = dot(rnl, n);
        if (d < bd || (d == bd && i < bi && d < FLT_MAX)) { bd = d; bi = i; }
    }
#pragma unroll
    for (uint32_t o = NARROW_GROUP / 2; o > 0; o >>= 1) {
        const float d = __shfl_xor_sync(mask, bd, o);
        const uint32_t i = __shfl_xor_sync(mask, bi, o);
        if (d < bd || (d == bd && i < bi && d < FLT_MAX)) { bd = d; bi = i; }
    }
    // The sequential search starts at edge 0 with minDot = FLT_MAX and takes strictly smaller dots only, so with no
    // dot below FLT_MAX it keeps edge 0.
    const uint32_t ie = bi == 0xFFFFFFFFu ? 0u : bi;
    bool hit = false;
    if (lane == 0) {
        const uint32_t i0 = bestIndex, i1 = next_index(i0, refCount);
        const V2 rs = refIsA ? sA[i0] : sB[i0];
        const V2 re = refIsA ? sA[i1] : sB[i1];
        const V2 rfc = (rs + re) * 0.5f;
        const V2 edge = re - rs;
        const float len2 = dot(edge, edge);
        const V2 sideDir = edge * (1.0f / sqrtf(len2));
        const uint32_t ie2 = next_index(ie, incCount);
        V2 c0 = refIsA ? sB[ie] : sA[ie];
        V2 c1 = refIsA ? sB[ie2] : sA[ie2];
        if (!clip_segment(c0, c1, rs, sideDir) && !clip_segment(c0, c1, re, -sideDir)) {
            const float refPlaneDist = dot(rfc, rnl);
            const uint32_t tag = refIsA ? REFERENCE_BODY_TAG : 0u;
            uint32_t cnt = 0;
            if (dot(c0, rnl) <= refPlaneDist + SAT_EPSILON) {
                out.p[cnt] = (A.pos + rightA * c0.x) + upA * c0.y; out.id[cnt] = tag | ie; cnt++;
            }
            if (dot(c1, rnl) <= refPlaneDist + SAT_EPSILON) {
                out.p[cnt] = (A.pos + rightA * c1.x) + upA * c1.y; out.id[cnt] = tag | ie2; cnt++;
            }
            if (cnt > 0) {
                out.n = rightA * nl.x + upA * nl.y; out.depth = depth; out.count = cnt;
                hit = true;
            }
        }
    }
    return __shfl_sync(mask, hit ? 1u : 0u, __ffs(mask) - 1) != 0;
}

// ---------------------------------------------------------------------------------------------------------------
// Capsules: a core segment of half length hw along the collider's local x axis, swept by radius r
// (CollisionMethods/*Capsule*.cpp). clampValue (HelperMethods.h:111-114) is fmin(fmax(v, lo), hi).
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ float clamp_value(float v, float lo, float hi) { return rfminf(rfmaxf(v, lo), hi); }

// collisionCircleCapsule, the scalar path (CircleCapsule.cpp:148-203). The 8-lane batch (:55-146) computes the same
// manifold except when the circle's centre lies within ZERO_DIVISION_BOUNDARY of the core, where it picks the
// fallback normal's side from another expression; this routine takes the scalar one there.
__device__ __forceinline__ bool collide_circle_capsule(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const float radiusA = A.r, halfLengthB = B.hw, radiusB = B.r;
    const V2 axisB = v2(B.c, B.s);
    const V2 d = A.pos - B.pos;
    const float t = clamp_value(dot(d, axisB), -halfLengthB, halfLengthB);
    const V2 delta = axisB * t - d;
    const float radiusSum = radiusA + radiusB;
    const float squaredDistance = dot(delta, delta);
    if (squaredDistance >= radiusSum * radiusSum) return false;
    const float distance = sqrtf(squaredDistance);
    const float depth = radiusSum - distance;
    V2 normal;
    if (distance < ZERO_DIVISION_BOUNDARY) normal = flip_if_negative(v2(B.s, -B.c), d.x * B.s + d.y * B.c);
    else normal = delta * (1.0f / distance);
    out.n = normal;
    out.depth = depth;
    out.count = 1;
    out.p[0] = A.pos + normal * radiusA;
    out.id[0] = 0;
    return true;
}

// collisionCapsuleCapsule (CapsuleCapsule.cpp:23-157).
__device__ __forceinline__ bool collide_capsule_capsule(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const float halfLengthA = A.hw, halfLengthB = B.hw, radiusA = A.r, radiusB = B.r;
    const V2 positionA = A.pos, positionB = B.pos;
    const V2 centerDelta = positionB - positionA;
    const float radiusSum = radiusA + radiusB;
    const float reach = halfLengthA + halfLengthB + radiusSum;
    if (dot(centerDelta, centerDelta) >= reach * reach) return false;
    const V2 axisA = v2(A.c, A.s), axisB = v2(B.c, B.s);
    const float b = dot(axisA, axisB);
    const float centerAlongA = dot(centerDelta, axisA);
    const float c = -centerAlongA;
    const float f = -dot(axisB, centerDelta);
    const float sinSquared = 1.0f - b * b;
    const bool parallel = sinSquared < CAPSULE_PARALLEL_SIN_SQUARED;
    const float extentB = fabsf(b) * halfLengthB;
    const float overlapLo = rfmaxf(-halfLengthA, centerAlongA - extentB);
    const float overlapHi = rfminf(halfLengthA, centerAlongA + extentB);
    const bool hasOverlap = parallel && (overlapHi - overlapLo >= ZERO_DIVISION_BOUNDARY);
    float s, t;
    if (hasOverlap) {
        s = 0.5f * (overlapLo + overlapHi);
        t = clamp_value(b * s + f, -halfLengthB, halfLengthB);
    } else {
        s = parallel ? 0.0f : clamp_value((b * f - c) / sinSquared, -halfLengthA, halfLengthA);
        t = b * s + f;
        t = clamp_value(t, -halfLengthB, halfLengthB);
        s = clamp_value(b * t - c, -halfLengthA, halfLengthA);
    }
    const V2 pointA = positionA + axisA * s;
    const V2 pointB = positionB + axisB * t;
    const V2 delta = pointB - pointA;
    const float squaredDistance = dot(delta, delta);
    if (squaredDistance >= radiusSum * radiusSum) return false;
    V2 normal;
    float depth;
    if (squaredDistance >= ZERO_DIVISION_BOUNDARY_SQUARED) {
        const float distance = sqrtf(squaredDistance);
        normal = delta * (1.0f / distance);
        depth = radiusSum - distance;
    } else {
        // Core segments intersect: separate along the cheaper of the two side axes.
        const V2 sideA = v2(-axisA.y, axisA.x), sideB = v2(-axisB.y, axisB.x);
        const float offsetA = dot(centerDelta, sideA);
        const float offsetB = dot(centerDelta, sideB);
        const float depthA = fabsf(dot(axisB, sideA)) * halfLengthB - fabsf(offsetA);
        const float depthB = fabsf(dot(axisA, sideB)) * halfLengthA - fabsf(offsetB);
        if (depthA <= depthB) { normal = flip_if_negative(sideA, offsetA); depth = depthA; }
        else { normal = flip_if_negative(sideB, offsetB); depth = depthB; }
        depth += radiusSum;
    }
    uint32_t count = 0;
    if (hasOverlap) {
        // Side by side: one contact at each end of the overlap, if within reach.
        const V2 sideB = v2(-axisB.y, axisB.x);
        const float ends[2] = {overlapLo, overlapHi};
        float minGap = FLT_MAX;
        for (uint32_t k = 0; k < 2; k++) {
            const V2 p = positionA + axisA * ends[k];
            const float gap = fabsf(dot(p - positionB, sideB));
            if (gap >= radiusSum) continue;
            out.p[count] = p + normal * radiusA;
            out.id[count] = k;
            count++;
            minGap = rfminf(minGap, gap);
        }
        if (count != 0) depth = radiusSum - minGap;
    }
    if (count == 0) {
        out.p[0] = pointA + normal * radiusA;
        out.id[0] = 2;
        count = 1;
    }
    out.n = normal;
    out.depth = depth;
    out.count = count;
    return true;
}

// collisionBoxCapsule (BoxCapsule.cpp:26-242): box A, capsule B, normal from the box to the capsule.
__device__ __forceinline__ bool collide_box_capsule(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const V2 halfExtents = v2(A.hw, A.hh);
    const V2 positionA = A.pos, rightA = v2(A.c, A.s), positionB = B.pos, axisB = v2(B.c, B.s);
    const float halfLengthB = B.hw, radius = B.r;
    const V2 upA = v2(-rightA.y, rightA.x);
    const V2 centerDelta = positionB - positionA;
    // Capsule pose in box-local space, folded into the +,+ quadrant.
    const float localX = dot(centerDelta, rightA);
    const float localY = dot(centerDelta, upA);
    const float sx = copysignf(1.0f, localX);
    const float sy = copysignf(1.0f, localY);
    const V2 center = v2(fabsf(localX), fabsf(localY));
    const V2 axis = v2((rightA.x * axisB.x + rightA.y * axisB.y) * sx, (rightA.x * axisB.y - rightA.y * axisB.x) * sy);
    const float absAxisX = fabsf(axis.x), absAxisY = fabsf(axis.y);
    const float sepX = center.x - halfLengthB * absAxisX - halfExtents.x;
    const float sepY = center.y - halfLengthB * absAxisY - halfExtents.y;
    const float faceSeparation = rfmaxf(sepX, sepY);
    if (faceSeparation >= radius) return false;
    const V2 sideAxis = v2(-axis.y, axis.x);
    const float sideOffset = dot(sideAxis, center);
    const float sideSeparation = fabsf(sideOffset) - (halfExtents.x * absAxisY + halfExtents.y * absAxisX);
    if (sideSeparation >= radius) return false;
    const bool sideWins = sideSeparation > faceSeparation + SAT_EPSILON;
    const bool swap = !sideWins && sepY > sepX;
    // Working frame: reference face at x = ext.x.
    const V2 ext = swap ? v2(halfExtents.y, halfExtents.x) : halfExtents;
    const V2 dir = swap ? v2(axis.y, axis.x) : axis;
    const V2 mid = swap ? v2(center.y, center.x) : center;
    const V2 basisX = rightA * sx, basisY = upA * sy;
    const V2 worldX = swap ? basisY : basisX;
    const V2 worldY = swap ? basisX : basisY;
    const V2 halfCore = dir * halfLengthB;
    const V2 s0 = mid - halfCore, s1 = mid + halfCore;
    const float length = halfLengthB * 2.0f;
    auto coreDistSquared = [&](V2 w) {
        const V2 d = s0 + dir * rfminf(rfmaxf(dot(w - s0, dir), 0.0f), length) - w;
        return dot(d, d);
    };
    V2 normal = v2(1.0f, 0.0f);
    float depth = 0.0f;
    uint32_t count = 0;
    V2 point0 = v2(0.0f, 0.0f), point1 = v2(0.0f, 0.0f);
    uint32_t id0 = 0, id1 = 0;
    bool faceContact = false;
    bool cornerPosX = true, cornerPosY = true;
    V2 vertexNormal = v2(1.0f, 0.0f);
    float vertexSeparation = faceSeparation;
    if (sideWins) {
        vertexNormal = sideOffset >= 0.0f ? sideAxis : -sideAxis;
        vertexSeparation = sideSeparation;
        cornerPosX = vertexNormal.x >= 0.0f;
        cornerPosY = vertexNormal.y >= 0.0f;
    } else {
        do {
            V2 c0 = s0, c1 = s1;
            float e0 = s0.x - ext.x, e1 = s1.x - ext.x;
            if (faceSeparation > 0.0f) {
                const float minY = rfminf(s0.y, s1.y), maxY = rfmaxf(s0.y, s1.y);
                if (minY > ext.y) break;
                const bool beyondLow = minY < -ext.y, beyondHigh = maxY > ext.y;
                if (beyondLow || beyondHigh) {
                    const float invDy = 1.0f / (s1.y - s0.y);
                    const float tA = (-ext.y - s0.y) * invDy;
                    const float tB = (ext.y - s0.y) * invDy;
                    const float tLow = rfmaxf(0.0f, rfminf(tA, tB));
                    const float tHigh = rfminf(1.0f, rfmaxf(tA, tB));
                    const V2 span = s1 - s0;
                    c0 = s0 + span * tLow;
                    c1 = s0 + span * tHigh;
                    e0 = c0.x - ext.x;
                    e1 = c1.x - ext.x;
                    const float minE = rfminf(e0, e1);
                    const float faceDistSquared = minE * minE;
                    if (beyondLow && coreDistSquared(v2(ext.x, -ext.y)) + SAT_EPSILON < faceDistSquared) {
                        cornerPosY = false;
                        break;
                    }
                    if (beyondHigh && coreDistSquared(ext) + SAT_EPSILON < faceDistSquared) break;
                }
            }
            const V2 clipped = c1 - c0;
            const bool hasSecond = dot(clipped, clipped) >= ZERO_DIVISION_BOUNDARY_SQUARED;
            const float contactLimit = radius + SAT_EPSILON;
            const uint32_t faceId = swap ? (sy < 0.0f ? 0u : 2u) : (sx < 0.0f ? 3u : 1u);
            const uint32_t idBase = REFERENCE_BODY_TAG | (faceId << 1);
            if (e0 <= contactLimit) { point0 = v2(c0.x - radius, c0.y); id0 = idBase; count = 1; }
            if (hasSecond && e1 <= contactLimit) {
                const V2 p = v2(c1.x - radius, c1.y);
                if (count == 0) { point0 = p; id0 = idBase | 1u; }
                else { point1 = p; id1 = idBase | 1u; }
                count++;
            }
            if (count == 0) return false;
            depth = radius - rfminf(e0, e1);
            faceContact = true;
        } while (false);
    }
    if (!faceContact) {
        // Single contact between a box corner and the capsule core.
        const V2 w = v2(cornerPosX ? ext.x : -ext.x, cornerPosY ? ext.y : -ext.y);
        const V2 q = s0 + dir * rfminf(rfmaxf(dot(w - s0, dir), 0.0f), length);
        normal = vertexNormal;
        depth = radius - vertexSeparation;
        if (vertexSeparation > 0.0f) {
            const V2 d = q - w;
            const float distSquared = dot(d, d);
            if (distSquared >= radius * radius) return false;
            if (distSquared >= ZERO_DIVISION_BOUNDARY_SQUARED) {
                const float distance = sqrtf(distSquared);
                normal = d * (1.0f / distance);
                depth = radius - distance;
            }
        }
        // Corner id in real box space (undo the swap, then the fold). Corner order: (-,-), (+,-), (+,+), (-,+).
        const bool foldedPosX = swap ? cornerPosY : cornerPosX;
        const bool foldedPosY = swap ? cornerPosX : cornerPosY;
        const bool realPosX = foldedPosX != (sx < 0.0f);
        const bool realPosY = foldedPosY != (sy < 0.0f);
        const uint32_t vertexId = (realPosY ? 2u : 0u) | ((realPosX != realPosY) ? 1u : 0u);
        count = 1;
        point0 = q - normal * radius;
        id0 = CAPSULE_VERTEX_CONTACT_TAG | vertexId;
    }
    out.n = worldX * normal.x + worldY * normal.y;
    out.p[0] = positionA + worldX * point0.x + worldY * point0.y;
    if (count > 1) out.p[1] = positionA + worldX * point1.x + worldY * point1.y;
    out.id[0] = id0;
    out.id[1] = id1;
    out.depth = depth;
    out.count = count;
    return true;
}

// collisionPolygonCapsule (PolygonCapsule.cpp:27-240): polygon A, capsule B, normal from the polygon to the capsule.
__device__ __forceinline__ bool collide_polygon_capsule(const ColliderView& A, const ColliderView& B, Contact& out)
{
    const uint32_t vertexCount = A.nv;
    const V2 positionA = A.pos, rightA = v2(A.c, A.s), positionB = B.pos, axisB = v2(B.c, B.s);
    const float halfLengthB = B.hw, radius = B.r;
    const V2 upA = v2(-rightA.y, rightA.x);
    const V2 centerDelta = positionB - positionA;
    const V2 centerLocal = v2(dot(centerDelta, rightA), dot(centerDelta, upA));
    const V2 axis = v2(rightA.x * axisB.x + rightA.y * axisB.y, rightA.x * axisB.y - rightA.y * axisB.x);
    const V2 halfCore = axis * halfLengthB;
    const V2 s0 = centerLocal - halfCore, s1 = centerLocal + halfCore;
    const float length = halfLengthB * 2.0f;
    const V2 sideAxis = v2(-axis.y, axis.x);
    float faceSeparation = -FLT_MAX;
    uint32_t faceIndex = 0;
    float minSide = FLT_MAX, maxSide = -FLT_MAX;
    uint32_t minSideVertex = 0, maxSideVertex = 0;
    for (uint32_t i = 0; i < vertexCount; i++) {
        const V2 v = ld2(A.verts, i), n = ld2(A.normals, i);
        const float separation = rfminf(dot(n, s0 - v), dot(n, s1 - v));
        if (separation >= radius) return false;
        if (separation > faceSeparation) { faceSeparation = separation; faceIndex = i; }
        const float side = dot(v, sideAxis);
        if (side < minSide) { minSide = side; minSideVertex = i; }
        if (side > maxSide) { maxSide = side; maxSideVertex = i; }
    }
    const float sideOffset = dot(sideAxis, centerLocal);
    const float sidePlus = sideOffset - maxSide;
    const float sideMinus = minSide - sideOffset;
    const float sideSeparation = rfmaxf(sidePlus, sideMinus);
    if (sideSeparation >= radius) return false;
    auto coreDistSquared = [&](V2 w) {
        const V2 d = s0 + axis * rfminf(rfmaxf(dot(w - s0, axis), 0.0f), length) - w;
        return dot(d, d);
    };
    V2 normal = v2(0.0f, 0.0f);
    float depth = 0.0f;
    uint32_t count = 0;
    V2 point0 = v2(0.0f, 0.0f), point1 = v2(0.0f, 0.0f);
    uint32_t id0 = 0, id1 = 0;
    bool faceContact = false;
    uint32_t vertexId = 0;
    V2 vertexNormal = v2(0.0f, 0.0f);
    float vertexSeparation = 0.0f;
    do {
        if (sideSeparation > faceSeparation + SAT_EPSILON) {
            const bool onPlusSide = sidePlus >= sideMinus;
            vertexId = onPlusSide ? maxSideVertex : minSideVertex;
            vertexNormal = onPlusSide ? sideAxis : -sideAxis;
            vertexSeparation = sideSeparation;
            break;
        }
        const uint32_t i0 = faceIndex, i1 = next_index(i0, vertexCount);
        const V2 a = ld2(A.verts, i0), b = ld2(A.verts, i1), n = ld2(A.normals, i0);
        const V2 tangent = v2(-n.y, n.x);
        vertexNormal = n;
        vertexSeparation = faceSeparation;
        V2 c0 = s0, c1 = s1;
        float e0 = dot(s0 - a, n), e1 = dot(s1 - a, n);
        if (faceSeparation > 0.0f) {
            const float edgeLength = dot(b - a, tangent);
            const float t0 = dot(s0 - a, tangent), t1 = dot(s1 - a, tangent);
            const bool beyondStart = rfminf(t0, t1) < 0.0f;
            const bool beyondEnd = rfmaxf(t0, t1) > edgeLength;
            if (beyondStart || beyondEnd) {
                if (clip_segment(c0, c1, a, tangent)) { vertexId = i0; break; }
                if (clip_segment(c0, c1, b, -tangent)) { vertexId = i1; break; }
                e0 = dot(c0 - a, n);
                e1 = dot(c1 - a, n);
                const float minE = rfminf(e0, e1);
                const float faceDistSquared = minE * minE;
                if (beyondStart && coreDistSquared(a) + SAT_EPSILON < faceDistSquared) { vertexId = i0; break; }
                if (beyondEnd && coreDistSquared(b) + SAT_EPSILON < faceDistSquared) { vertexId = i1; break; }
            }
        }
        const V2 span = c1 - c0;
        const bool hasSecond = dot(span, span) >= ZERO_DIVISION_BOUNDARY_SQUARED;
        const float contactLimit = radius + SAT_EPSILON;
        const uint32_t idBase = REFERENCE_BODY_TAG | (i0 << 1);
        if (e0 <= contactLimit) { point0 = c0 - n * radius; id0 = idBase; count = 1; }
        if (hasSecond && e1 <= contactLimit) {
            const V2 p = c1 - n * radius;
            if (count == 0) { point0 = p; id0 = idBase | 1u; }
            else { point1 = p; id1 = idBase | 1u; }
            count++;
        }
        if (count == 0) return false;
        normal = n;
        depth = radius - rfminf(e0, e1);
        faceContact = true;
    } while (false);
    if (!faceContact) {
        const V2 w = ld2(A.verts, vertexId);
        const V2 q = s0 + axis * rfminf(rfmaxf(dot(w - s0, axis), 0.0f), length);
        normal = vertexNormal;
        depth = radius - vertexSeparation;
        if (vertexSeparation > 0.0f) {
            const V2 d = q - w;
            const float distSquared = dot(d, d);
            if (distSquared >= radius * radius) return false;
            if (distSquared >= ZERO_DIVISION_BOUNDARY_SQUARED) {
                const float distance = sqrtf(distSquared);
                normal = d * (1.0f / distance);
                depth = radius - distance;
            }
        }
        count = 1;
        point0 = q - normal * radius;
        id0 = CAPSULE_VERTEX_CONTACT_TAG | vertexId;
    }
    out.n = rightA * normal.x + upA * normal.y;
    out.p[0] = positionA + rightA * point0.x + upA * point0.y;
    if (count > 1) out.p[1] = positionA + rightA * point1.x + upA * point1.y;
    out.id[0] = id0;
    out.id[1] = id1;
    out.depth = depth;
    out.count = count;
    return true;
}

// Dispatch on the (ordered) shape-type pair: typeA <= typeB.
__device__ __forceinline__ bool collide(const ColliderView& A, const ColliderView& B, Contact& out)
{
    if (B.type == SHAPE_CAPSULE) {
        if (A.type == SHAPE_CIRCLE) return collide_circle_capsule(A, B, out);
        if (A.type == SHAPE_BOX) return collide_box_capsule(A, B, out);
        if (A.type == SHAPE_POLYGON) return collide_polygon_capsule(A, B, out);
        return collide_capsule_capsule(A, B, out);
    }
    if (A.type == SHAPE_CIRCLE) {
        if (B.type == SHAPE_CIRCLE) return collide_circle_circle(A, B, out);
        if (B.type == SHAPE_BOX) return collide_circle_box(A, B, out);
        return collide_circle_polygon(A, B, out);
    }
    if (A.type == SHAPE_BOX) {
        if (B.type == SHAPE_BOX) return collide_box_box(A, B, out);
        return collide_box_polygon(A, B, out);
    }
    return collide_polygon_polygon(A, B, out);
}

}  // namespace ag2d
