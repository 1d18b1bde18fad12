/* CPU restatement of PS_AGONY2D's per-step collision and contact pipeline (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY — see ag2d_oracle.h. Compiled with -O2 -ffp-contract=off so that every a*b+c stays two
 * roundings, as in the reference's parity build; fmaf() appears only where the reference's SIMD path issues an
 * FMA instruction (Ecstasy Simd::negMulAdd).
 *
 * Reference paths are relative to PhysicsSimulation-Agony/PS_AGONY2D/.
 */
#include "ag2d_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Constants.h:7-14 (double constants rounded to float) */
#define ORA_FULL_PI 3.14159265358979323846
static const float HALF_PI_F = (float)(ORA_FULL_PI * 0.5);
static const float INV_HALF_PI_F = (float)(1.0 / (ORA_FULL_PI * 0.5));
static const float TWO_PI_F = (float)(ORA_FULL_PI * 2.0);
static const float INV_TWO_PI_F = (float)(1.0 / (ORA_FULL_PI * 2.0));

/* FastCosSin.cpp:10-14 */
static const float COEF0 = (float)9.9999999999953215e-01;
static const float COEF1 = (float)-1.6666666534403832e-01;
static const float COEF2 = (float)8.3332302391869520e-03;
static const float COEF3 = (float)-1.9818200679665358e-04;
static const float COEF4 = (float)2.6182346015248291e-06;

/* Narrow/Constants.h:7-37 */
#define ZERO_DIVISION_BOUNDARY 1e-4f
#define ZERO_DIVISION_BOUNDARY_SQUARED 1e-8f
#define SAT_EPSILON 1e-4f
#define REFERENCE_BODY_TAG 0x80000000u

/* Width of the reference's float SIMD register (AVX2: 8 lanes). Elements [0, n & ~7) of a range take the SIMD
 * path, the rest the scalar tail. */
#define SIMD_LANES 8u

static inline uint32_t simd_body_count(uint32_t n) { return n & ~(SIMD_LANES - 1u); }

/* ------------------------------------------------------------------------------------------------------------ */
/* Integration (Integration/Integrator.cpp:140-299; call order Simulation.cpp:392-407)                        */
/* ------------------------------------------------------------------------------------------------------------ */

static void damp_angular(ora_world *w, uint32_t begin, uint32_t end, float dtPart, float damping_setting)
{
    /* Integrator.cpp:253-299: skipped unless 0 <= damping < 1. */
    if (!(damping_setting >= 0.0f && damping_setting < 1.0f)) return;
    const float damping = powf(damping_setting, dtPart);
    const uint32_t simd = begin + simd_body_count(end - begin);
    for (uint32_t i = begin; i < end; i++) {
        const float av = w->angVel[i];
        const int movable = w->invInertia[i] != 0.0f;
        const float nv = av * damping;
        if (i < simd) {
            w->angVel[i] = movable ? nv : av;                       /* blendv */
        } else {
            const float m = (float)movable;
            w->angVel[i] = m * nv + (1.0f - m) * av;
        }
    }
}

void ora_integrate_velocity_verlet(ora_world *w, uint32_t begin, uint32_t end, float dt, float gx, float gy,
                                   float angular_damping)
{
    const float halfDT = dt * 0.5f;
    const float gdx = gx * halfDT, gdy = gy * halfDT;
    const uint32_t simd = begin + simd_body_count(end - begin);

    /* integratePhase1_VelocityVerlet (Integrator.cpp:140-180): half velocity step for movable bodies. */
    for (uint32_t i = begin; i < end; i++) {
        const int movable = w->invMass[i] != 0.0f;
        if (i < simd) {
            w->velX[i] += movable ? gdx : 0.0f;                      /* gravityDelta & mask */
            w->velY[i] += movable ? gdy : 0.0f;
        } else {
            w->velX[i] += gdx * (float)movable;
            w->velY[i] += gdy * (float)movable;
        }
    }
    damp_angular(w, begin, end, halfDT, angular_damping);

    /* integratePhase2_VelocityVerlet (Integrator.cpp:182-250): full position step, then half velocity step. */
    for (uint32_t i = begin; i < end; i++) {
        w->comX[i] = w->velX[i] * dt + w->comX[i];
        w->comY[i] = w->velY[i] * dt + w->comY[i];
        w->rot[i] = w->angVel[i] * dt + w->rot[i];
        const int movable = w->invMass[i] != 0.0f;
        if (i < simd) {
            w->velX[i] += movable ? gdx : 0.0f;
            w->velY[i] += movable ? gdy : 0.0f;
        } else {
            w->velX[i] += gdx * (float)movable;
            w->velY[i] += gdy * (float)movable;
        }
    }
    damp_angular(w, begin, end, halfDT, angular_damping);
}

/* wrapBodyRotations (SimulationImpl/LeftOutFunctions.cpp:13-60). The SIMD body subtracts with a fused
 * negative multiply-add; the scalar tail with a separate multiply and subtract, and uses the double-rounded
 * 1/(2 pi) constant where the SIMD body uses 1.0f / TWO_PI computed in float. */
void ora_wrap_body_rotations(ora_world *w, uint32_t begin, uint32_t end)
{
    const float invTwoPiSimd = 1.0f / TWO_PI_F;
    const uint32_t simd = begin + simd_body_count(end - begin);
    for (uint32_t i = begin; i < end; i++) {
        float rot = w->rot[i];
        float wc;
        if (i < simd) {
            wc = truncf(rot * invTwoPiSimd);
            rot = fmaf(-wc, TWO_PI_F, rot);
            if (rot < 0.0f) { rot += TWO_PI_F; wc -= 1.0f; } else { rot += 0.0f; wc -= 0.0f; }
            w->wrapCount[i] = w->wrapCount[i] + wc;
        } else {
            wc = truncf(rot * INV_TWO_PI_F);
            rot -= wc * TWO_PI_F;
            const float neg = (float)(rot < 0.0f);
            rot += neg * TWO_PI_F;
            wc -= neg;
            w->wrapCount[i] += wc;
        }
        w->rot[i] = rot;
    }
}

static void wrap_collider_range(float *rot, uint32_t begin, uint32_t end)
{
    /* wrapColliderRotations (LeftOutFunctions.cpp:62-102): same as the body wrap without the wrap count. */
    const float invTwoPiSimd = 1.0f / TWO_PI_F;
    const uint32_t simd = begin + simd_body_count(end - begin);
    for (uint32_t i = begin; i < end; i++) {
        float r = rot[i];
        if (i < simd) {
            const float wc = truncf(r * invTwoPiSimd);
            r = fmaf(-wc, TWO_PI_F, r);
            r += (r < 0.0f) ? TWO_PI_F : 0.0f;
        } else {
            const float wc = truncf(r * INV_TWO_PI_F);
            r -= wc * TWO_PI_F;
            const float neg = (float)(r < 0.0f);
            r += neg * TWO_PI_F;
        }
        rot[i] = r;
    }
}

/* FastCosSin::order5Array (FastCosSin.cpp:26-109). Quadrant by truncation, mirrored argument, odd degree-5
 * polynomial for sin clamped to 1, cos = sqrt(1 - sin^2). The SIMD body applies the quadrant signs by flipping
 * sign bits ((q & 2) and ((q + 1) & 2)); the scalar tail multiplies by 1 - 2 * (q >> 1) etc. The two agree for
 * q in [0, 3]; both forms are kept for the q = 4 edge (an input a few ulp below 2 pi). */
void ora_fastcossin_array(const float *in, float *out_cos, float *out_sin, uint32_t n)
{
    const uint32_t simd = simd_body_count(n);
    for (uint32_t i = 0; i < n; i++) {
        const float x = in[i];
        const int q = (int)(x * INV_HALF_PI_F);
        const float u = x - (float)q * HALF_PI_F;
        const float mirror = (float)(q & 1);
        const float a = mirror * (HALF_PI_F - 2.0f * u) + u;
        const float a2 = a * a;
        float s = COEF4;
        s = s * a2 + COEF3;
        s = s * a2 + COEF2;
        s = s * a2 + COEF1;
        s = s * a2 + COEF0;
        s = s * a;
        s = (s < 1.0f) ? s : 1.0f;
        const float c = sqrtf(1.0f - s * s);
        float so, co;
        if (i < simd) {
            uint32_t sb, cb;
            memcpy(&sb, &s, 4);
            memcpy(&cb, &c, 4);
            sb ^= ((uint32_t)(q & 2)) << 30;
            cb ^= ((uint32_t)((q + 1) & 2)) << 30;
            memcpy(&so, &sb, 4);
            memcpy(&co, &cb, 4);
        } else {
            const float sinSign = 1.0f - 2.0f * (float)(q >> 1);
            const float cosSign = 1.0f - 2.0f * (float)(((q + 1) >> 1) & 1);
            so = sinSign * s;
            co = cosSign * c;
        }
        out_sin[i] = so;
        out_cos[i] = co;
    }
}

/* Integrator::computeRotationCosSin (Integrator.cpp:301-311). */
void ora_body_cossin(ora_world *w, uint32_t begin, uint32_t end)
{
    ora_fastcossin_array(w->rot + begin, w->rotCos + begin, w->rotSin + begin, end - begin);
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Collider poses and AABBs (Simulation.cpp:673-736; SimulationImpl/ColliderAABBBuilder.cpp:8-136)             */
/* ------------------------------------------------------------------------------------------------------------ */

void ora_collider_world_positions(ora_world *w, uint32_t begin, uint32_t end)
{
    for (uint32_t i = begin; i < end; i++) {
        const uint32_t b = w->bodyIndex[i];
        const float offX = w->comOffX[i], offY = w->comOffY[i];
        const float c = w->rotCos[b], s = w->rotSin[b];
        w->worldX[i] = w->comX[b] + (offX * c - offY * s);
        w->worldY[i] = w->comY[b] + (offX * s + offY * c);
    }
}

void ora_collider_world_rotations(ora_world *w, uint32_t begin, uint32_t end)
{
    if (begin == end) return;
    for (uint32_t i = begin; i < end; i++) w->worldRot[i] = w->rot[w->bodyIndex[i]] + w->localRot[i];
    wrap_collider_range(w->worldRot, begin, end);
    ora_fastcossin_array(w->worldRot + begin, w->worldCos + begin, w->worldSin + begin, end - begin);
}

void ora_collider_aabbs(ora_world *w, uint32_t begin, uint32_t end)
{
    for (uint32_t i = begin; i < end; i++) {
        const uint32_t si = w->shapeIndex[i];
        const float x = w->worldX[i], y = w->worldY[i];
        switch (w->shapeType[i]) {
        case ORA_CIRCLE: { /* ColliderAABBBuilder.cpp:8-38 */
            const float r = w->circleRadius[si];
            w->minX[i] = x - r; w->minY[i] = y - r; w->maxX[i] = x + r; w->maxY[i] = y + r;
            break;
        }
        case ORA_BOX: { /* :40-82 */
            const float hw = w->boxHalfW[si], hh = w->boxHalfH[si];
            const float ac = fabsf(w->worldCos[i]), as = fabsf(w->worldSin[i]);
            const float ex = ac * hw + as * hh;
            const float ey = as * hw + ac * hh;
            w->minX[i] = x - ex; w->minY[i] = y - ey; w->maxX[i] = x + ex; w->maxY[i] = y + ey;
            break;
        }
        case ORA_POLYGON: { /* :84-136 */
            const float c = w->worldCos[i], s = w->worldSin[i];
            const float *v = w->polyVerts + 2u * w->polyOffset[si];
            const uint32_t nv = w->polyCount[si];
            float mnx = FLT_MAX, mny = FLT_MAX, mxx = -FLT_MAX, mxy = -FLT_MAX;
            for (uint32_t k = 0; k < nv; k++) {
                const float wx = c * v[2 * k] - s * v[2 * k + 1];
                const float wy = s * v[2 * k] + c * v[2 * k + 1];
                mnx = fminf(mnx, wx); mxx = fmaxf(mxx, wx);
                mny = fminf(mny, wy); mxy = fmaxf(mxy, wy);
            }
            w->minX[i] = x + mnx; w->minY[i] = y + mny; w->maxX[i] = x + mxx; w->maxY[i] = y + mxy;
            break;
        }
        default:
            break;
        }
    }
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Morton keys and sort (CollisionDetection/Broad/BvhTree.cpp:27-40, 148-354)                                   */
/* ------------------------------------------------------------------------------------------------------------ */

static inline uint32_t part1by1(uint32_t x)
{
    x &= 0x0000ffffu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

void ora_morton_codes(const ora_world *w, uint32_t begin, uint32_t end, uint32_t *out_codes, float *out_bounds4)
{
    /* gatherCentroids (:148-188): 2 x centroid and the union of the AABBs. */
    float bminX = FLT_MAX, bminY = FLT_MAX, bmaxX = -FLT_MAX, bmaxY = -FLT_MAX;
    for (uint32_t i = begin; i < end; i++) {
        bminX = fminf(bminX, w->minX[i]); bminY = fminf(bminY, w->minY[i]);
        bmaxX = fmaxf(bmaxX, w->maxX[i]); bmaxY = fmaxf(bmaxY, w->maxY[i]);
    }
    if (out_bounds4) { out_bounds4[0] = bminX; out_bounds4[1] = bminY; out_bounds4[2] = bmaxX; out_bounds4[3] = bmaxY; }
    /* transformCentroids (:191-250). */
    const float kEps = 1e-5f;
    const float maxX = fmaxf(bmaxX, bminX + kEps);
    const float maxY = fmaxf(bmaxY, bminY + kEps);
    const float clampMax = 65535.0f;
    const float scaleX = clampMax / (maxX - bminX);
    const float scaleY = clampMax / (maxY - bminY);
    const float negScaledMinX = -bminX * scaleX;
    const float negScaledMinY = -bminY * scaleY;
    const float halfScaleX = scaleX * 0.5f;
    const float halfScaleY = scaleY * 0.5f;
    for (uint32_t i = begin; i < end; i++) {
        const float cx = w->minX[i] + w->maxX[i];
        const float cy = w->minY[i] + w->maxY[i];
        float tx = cx * halfScaleX + negScaledMinX;
        float ty = cy * halfScaleY + negScaledMinY;
        tx = tx < 0.0f ? 0.0f : (tx > clampMax ? clampMax : tx);
        ty = ty < 0.0f ? 0.0f : (ty > clampMax ? clampMax : ty);
        /* computeMortonCodes (:252-280): truncate, interleave, y in the odd bits. */
        out_codes[i - begin] = (part1by1((uint32_t)ty) << 1) | part1by1((uint32_t)tx);
    }
}

/* sortByMortonCodes (:282-354): stable 4 x 8-bit LSD radix sort of {key, collider index}. */
void ora_sort_by_morton(const uint32_t *codes, uint32_t begin, uint32_t n, uint32_t *out_sorted_colliders,
                        uint32_t *out_sorted_codes)
{
    uint32_t *ka = malloc(sizeof(uint32_t) * (n ? n : 1)), *ia = malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *kb = malloc(sizeof(uint32_t) * (n ? n : 1)), *ib = malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; i++) { ka[i] = codes[i]; ia[i] = begin + i; }
    for (uint32_t shift = 0; shift < 32; shift += 8) {
        uint32_t count[256] = {0};
        for (uint32_t i = 0; i < n; i++) count[(ka[i] >> shift) & 0xFFu]++;
        uint32_t sum = 0;
        for (uint32_t d = 0; d < 256; d++) { const uint32_t c = count[d]; count[d] = sum; sum += c; }
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t dst = count[(ka[i] >> shift) & 0xFFu]++;
            kb[dst] = ka[i]; ib[dst] = ia[i];
        }
        uint32_t *t = ka; ka = kb; kb = t;
        t = ia; ia = ib; ib = t;
    }
    for (uint32_t i = 0; i < n; i++) { out_sorted_colliders[i] = ia[i]; out_sorted_codes[i] = ka[i]; }
    free(ka); free(ia); free(kb); free(ib);
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Broad phase pair set (BroadPhaseCollisionDetector.cpp:197-244; BvhNode.h:33-38; LeafPairTesting.h:71-203)    */
/* The reference's pair set does not depend on its tree: a pair is reported iff the AABBs overlap strictly,     */
/* one collider is dynamic, and (dynamic-dynamic) the owners differ. This restatement finds the same set by a   */
/* sweep over x.                                                                                                 */
/* ------------------------------------------------------------------------------------------------------------ */

static const ora_world *g_sort_world;
static int cmp_minx(const void *pa, const void *pb)
{
    const uint32_t a = *(const uint32_t *)pa, b = *(const uint32_t *)pb;
    const float xa = g_sort_world->minX[a], xb = g_sort_world->minX[b];
    if (xa < xb) return -1;
    if (xa > xb) return 1;
    return (a < b) ? -1 : (a > b);
}

static int cmp_pair(const void *pa, const void *pb)
{
    const uint32_t *a = pa, *b = pb;
    if (a[0] != b[0]) return a[0] < b[0] ? -1 : 1;
    if (a[1] != b[1]) return a[1] < b[1] ? -1 : 1;
    return 0;
}

int64_t ora_broad_pairs(const ora_world *w, uint32_t *out_pairs, int64_t cap)
{
    const uint32_t n = w->col_starts[3];
    const uint32_t dynBegin = w->col_starts[2];
    uint32_t *order = malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    g_sort_world = w;
    qsort(order, n, sizeof(uint32_t), cmp_minx);
    int64_t count = 0;
    for (uint32_t oi = 0; oi < n; oi++) {
        const uint32_t i = order[oi];
        const int di = i >= dynBegin;
        for (uint32_t oj = oi + 1; oj < n; oj++) {
            const uint32_t j = order[oj];
            if (!(w->minX[j] < w->maxX[i])) break;
            const int dj = j >= dynBegin;
            if (!di && !dj) continue;
            if (!(w->minX[i] < w->maxX[j] && w->maxX[i] > w->minX[j] &&
                  w->minY[i] < w->maxY[j] && w->maxY[i] > w->minY[j])) continue;
            uint32_t a, b;
            if (di && dj) {
                if (w->bodyIndex[i] == w->bodyIndex[j]) continue;
                a = i < j ? i : j; b = i < j ? j : i;
            } else {
                a = di ? i : j; b = di ? j : i;
            }
            if (count < cap) { out_pairs[2 * count] = a; out_pairs[2 * count + 1] = b; }
            count++;
        }
    }
    free(order);
    if (count > cap) return -count;
    qsort(out_pairs, (size_t)count, 2 * sizeof(uint32_t), cmp_pair);
    return count;
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Narrow phase (CollisionDetection/Narrow/...)                                                                 */
/* ------------------------------------------------------------------------------------------------------------ */

typedef struct { float x, y; } v2;
static inline v2 mk(float x, float y) { v2 r = {x, y}; return r; }
static inline float dot2(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }  /* glm::dot: (a*b).x + (a*b).y */
static inline v2 sub2(v2 a, v2 b) { return mk(a.x - b.x, a.y - b.y); }
static inline v2 add2(v2 a, v2 b) { return mk(a.x + b.x, a.y + b.y); }
static inline v2 scl2(v2 a, float s) { return mk(a.x * s, a.y * s); }
static inline v2 neg2(v2 a) { return mk(-a.x, -a.y); }
static inline uint32_t next_index(uint32_t i, uint32_t n) { return i + 1 == n ? 0u : i + 1; }

static inline v2 vert(const ora_world *w, uint32_t si, uint32_t k)
{
    const float *p = w->polyVerts + 2u * (w->polyOffset[si] + k);
    return mk(p[0], p[1]);
}
static inline v2 nrm(const ora_world *w, uint32_t si, uint32_t k)
{
    const float *p = w->polyNormals + 2u * (w->polyOffset[si] + k);
    return mk(p[0], p[1]);
}

/* clipSegment (Narrow/HelperMethods.h:36-52). Returns 1 if both points are outside. */
static int clip_segment(v2 *p1, v2 *p2, v2 planePoint, v2 planeNormal)
{
    const float d1 = dot2(sub2(*p1, planePoint), planeNormal);
    const float d2 = dot2(sub2(*p2, planePoint), planeNormal);
    if (d1 >= 0.0f && d2 >= 0.0f) return 0;
    if (d1 < 0.0f && d2 < 0.0f) return 1;
    const float t = d1 / (d1 - d2);
    const v2 dir = sub2(*p2, *p1);
    const v2 inter = add2(*p1, scl2(dir, t));
    if (d1 >= 0.0f) *p2 = inter; else *p1 = inter;
    return 0;
}

static inline void flip_if_negative(v2 *v, float sign)
{
    /* flipSignIfNegative (HelperMethods.h:26-34): xor the sign bit of 'sign' into both components. */
    uint32_t sb, xb, yb;
    memcpy(&sb, &sign, 4); memcpy(&xb, &v->x, 4); memcpy(&yb, &v->y, 4);
    sb &= 0x80000000u; xb ^= sb; yb ^= sb;
    memcpy(&v->x, &xb, 4); memcpy(&v->y, &yb, 4);
}

static void emit(ora_manifold *m, uint32_t a, uint32_t b, v2 n, float depth, uint32_t count, v2 p0, v2 p1,
                 uint32_t id0, uint32_t id1)
{
    memset(m, 0, sizeof(*m));
    m->a = a; m->b = b; m->nx = n.x; m->ny = n.y; m->depth = depth; m->count = count;
    m->px[0] = p0.x; m->py[0] = p0.y; m->id[0] = id0;
    if (count > 1) { m->px[1] = p1.x; m->py[1] = p1.y; m->id[1] = id1; }
}

/* collisionCircleCircle (CollisionMethods/CircleCircle.cpp:14-179). */
static int circle_circle(const ora_world *w, uint32_t a, uint32_t b, ora_manifold *out)
{
    const v2 pA = mk(w->worldX[a], w->worldY[a]), pB = mk(w->worldX[b], w->worldY[b]);
    const float rA = w->circleRadius[w->shapeIndex[a]], rB = w->circleRadius[w->shapeIndex[b]];
    const v2 d = sub2(pB, pA);
    const float rs = rA + rB;
    const float sq = dot2(d, d);
    if (!(sq < rs * rs)) return 0;
    const float dist = sqrtf(sq);
    const float depth = rs - dist;
    v2 n;
    if (dist < ZERO_DIVISION_BOUNDARY) n = mk(1.0f, 0.0f);
    else { const float inv = 1.0f / dist; n = scl2(d, inv); }
    emit(out, a, b, n, depth, 1, add2(pA, scl2(n, rA)), mk(0, 0), 0, 0);
    return 1;
}

/* collisionCircleBox (CollisionMethods/CircleBox.cpp:9-120). A circle, B box. */
static int circle_box(const ora_world *w, uint32_t a, uint32_t b, ora_manifold *out)
{
    const v2 pA = mk(w->worldX[a], w->worldY[a]), pB = mk(w->worldX[b], w->worldY[b]);
    const float rA = w->circleRadius[w->shapeIndex[a]];
    const float hw = w->boxHalfW[w->shapeIndex[b]], hh = w->boxHalfH[w->shapeIndex[b]];
    const float cB = w->worldCos[b], sB = w->worldSin[b];
    const v2 dg = sub2(pA, pB);
    const v2 loc = mk(dg.x * cB + dg.y * sB, dg.x * -sB + dg.y * cB);
    const v2 cl = mk(fminf(fmaxf(loc.x, -hw), hw), fminf(fmaxf(loc.y, -hh), hh));
    const v2 dl = sub2(cl, loc);
    const float sq = dot2(dl, dl);
    if (sq >= rA * rA) return 0;
    if (sq >= ZERO_DIVISION_BOUNDARY_SQUARED) {
        const float dist = sqrtf(sq);
        const float inv = 1.0f / dist;
        const v2 wd = mk(cB * dl.x - sB * dl.y, sB * dl.x + cB * dl.y);
        const v2 n = scl2(wd, inv);
        uint32_t id = 0;
        id |= (uint32_t)(loc.x > hw);
        id |= (uint32_t)(loc.x < -hw) << 1;
        id |= (uint32_t)(loc.y > hh) << 2;
        id |= (uint32_t)(loc.y < -hh) << 3;
        emit(out, a, b, n, rA - dist, 1, add2(pA, scl2(n, rA)), mk(0, 0), id, 0);
        return 1;
    }
    const float dx = hw - fabsf(loc.x);
    const float dy = hh - fabsf(loc.y);
    const int useY = dy <= dx;
    const float minPen = useY ? dy : dx;
    const float sign = copysignf(1.0f, useY ? loc.y : loc.x);
    const v2 nl = mk(useY ? 0.0f : sign, useY ? sign : 0.0f);
    const uint32_t id = 1u << ((uint32_t)(sign <= 0.0f) + ((uint32_t)useY << 1));
    const v2 n = neg2(mk(cB * nl.x - sB * nl.y, sB * nl.x + cB * nl.y));
    emit(out, a, b, n, rA + minPen, 1, add2(pA, scl2(n, rA)), mk(0, 0), id, 0);
    return 1;
}

/* collisionCirclePolygon (CollisionMethods/CirclePolygon.cpp:10-103) with findSupportEdge and
 * closestPointOnSegment (HelperMethods.h:73-109). A circle, B polygon. */
static int circle_polygon(const ora_world *w, uint32_t a, uint32_t b, ora_manifold *out)
{
    const v2 pA = mk(w->worldX[a], w->worldY[a]), pB = mk(w->worldX[b], w->worldY[b]);
    const float cB = w->worldCos[b], sB = w->worldSin[b];
    const float rA = w->circleRadius[w->shapeIndex[a]];
    const uint32_t si = w->shapeIndex[b];
    const uint32_t nv = w->polyCount[si];
    const v2 dg = sub2(pA, pB);
    const v2 loc = mk(dg.x * cB + dg.y * sB, dg.x * -sB + dg.y * cB);
    float maxSep = -FLT_MAX;
    uint32_t edge = 0;
    for (uint32_t i = 0; i < nv; i++) {
        const float sep = dot2(nrm(w, si, i), sub2(loc, vert(w, si, i)));
        if (sep > rA) return 0;
        if (sep > maxSep) { maxSep = sep; edge = i; }
    }
    v2 nl;
    float separation;
    if (maxSep >= ZERO_DIVISION_BOUNDARY) {
        const v2 va = vert(w, si, edge), vb = vert(w, si, next_index(edge, nv));
        const v2 ab = sub2(vb, va);
        const float denom = dot2(ab, ab);
        v2 cp;
        if (denom < ZERO_DIVISION_BOUNDARY_SQUARED) cp = va;
        else {
            const float t = dot2(sub2(loc, va), ab) / denom;
            cp = add2(va, scl2(ab, fminf(fmaxf(t, 0.0f), 1.0f)));
        }
        const v2 cpd = sub2(loc, cp);
        const float d2 = dot2(cpd, cpd);
        if (d2 > rA * rA) return 0;
        if (d2 < ZERO_DIVISION_BOUNDARY_SQUARED) { separation = 0.0f; nl = nrm(w, si, edge); }
        else { separation = sqrtf(d2); nl = scl2(cpd, 1.0f / separation); }
    } else {
        nl = nrm(w, si, edge);
        separation = maxSep;
    }
    const v2 n = neg2(mk(cB * nl.x - sB * nl.y, sB * nl.x + cB * nl.y));
    emit(out, a, b, n, rA - separation, 1, add2(pA, scl2(n, rA)), mk(0, 0), edge, 0);
    return 1;
}

/* collisionBoxBox (CollisionMethods/BoxBox.cpp:13-227): 4-axis SAT (lanes A right, A up, B right, B up), lowest
 * lane wins ties, reference face on the winning axis, incident face by the relative rotation, two clips. */
static int box_box(const ora_world *w, uint32_t a, uint32_t b, ora_manifold *out)
{
    const v2 pA = mk(w->worldX[a], w->worldY[a]), pB = mk(w->worldX[b], w->worldY[b]);
    const float cA = w->worldCos[a], sA = w->worldSin[a], cB = w->worldCos[b], sB = w->worldSin[b];
    const float hwA = w->boxHalfW[w->shapeIndex[a]], hhA = w->boxHalfH[w->shapeIndex[a]];
    const float hwB = w->boxHalfW[w->shapeIndex[b]], hhB = w->boxHalfH[w->shapeIndex[b]];
    const v2 rightA = mk(cA, sA), upA = mk(-sA, cA), rightB = mk(cB, sB), upB = mk(-sB, cB);
    const float relCos = cA * cB + sA * sB;
    const float relSin = cA * sB - sA * cB;
    const float arc = fabsf(relCos), ars = fabsf(relSin);
    const v2 cd = sub2(pB, pA);
    const float hwL[4] = {hwB, hwB, hwA, hwA}, hhL[4] = {hhB, hhB, hhA, hhA}, hwhL[4] = {hwA, hhA, hwB, hhB};
    const float cs1[4] = {arc, ars, arc, ars}, cs2[4] = {ars, arc, ars, arc};
    const float axX[4] = {cA, -sA, cB, -sB}, axY[4] = {sA, cA, sB, cB};
    float ov[4], cdoa[4];
    for (int k = 0; k < 4; k++) {
        const float rsum = hwL[k] * cs1[k] + hhL[k] * cs2[k] + hwhL[k];
        cdoa[k] = cd.x * axX[k] + cd.y * axY[k];
        ov[k] = rsum - fabsf(cdoa[k]);
    }
    for (int k = 0; k < 4; k++) if (ov[k] < 0.0f) return 0;
    const float depth = fminf(fminf(ov[0], ov[1]), fminf(ov[2], ov[3]));
    const uint32_t n0 = ov[0] != depth;
    const uint32_t n01 = n0 & (uint32_t)(ov[1] != depth);
    const uint32_t n012 = n01 & (uint32_t)(ov[2] != depth);
    const uint32_t best = n0 + n01 + n012;
    v2 normal = mk(axX[best], axY[best]);
    flip_if_negative(&normal, cdoa[best]);
    const int refIsA = best < 2;
    v2 posRef, posInc, rightRef, upRef, rightInc, upInc, refNormal;
    float hwRef, hhRef, hwInc, hhInc;
    if (refIsA) {
        posRef = pA; hwRef = hwA; hhRef = hhA; rightRef = rightA; upRef = upA;
        posInc = pB; hwInc = hwB; hhInc = hhB; rightInc = rightB; upInc = upB;
        refNormal = normal;
    } else {
        posRef = pB; hwRef = hwB; hhRef = hhB; rightRef = rightB; upRef = upB;
        posInc = pA; hwInc = hwA; hhInc = hhA; rightInc = rightA; upInc = upA;
        refNormal = neg2(normal);
    }
    const float sign = copysignf(1.0f, refIsA ? cdoa[best] : -cdoa[best]);
    v2 rfc, sideDir;
    const int useX = best == 0 || best == 2;
    if (useX) { rfc = add2(posRef, scl2(rightRef, sign * hwRef)); sideDir = upRef; }
    else { rfc = add2(posRef, scl2(upRef, sign * hhRef)); sideDir = rightRef; }
    const v2 eo = scl2(sideDir, useX ? hhRef : hwRef);
    const v2 refStart = add2(rfc, eo), refEnd = sub2(rfc, eo);
    v2 incStart, incEnd;
    {
        const int axisIsUp = (best & 1u) != 0;
        const float sideTerm = (best == 0 || best == 3) ? -relSin : relSin;
        const float dotX = sign * (axisIsUp ? sideTerm : relCos);
        const float dotY = sign * (axisIsUp ? relCos : sideTerm);
        const int useXi = fabsf(dotX) > fabsf(dotY);
        const float incSign = -copysignf(1.0f, useXi ? dotX : dotY);
        v2 fc, off;
        if (useXi) { fc = add2(posInc, scl2(rightInc, incSign * hwInc)); off = scl2(upInc, hhInc); }
        else { fc = add2(posInc, scl2(upInc, incSign * hhInc)); off = scl2(rightInc, hwInc); }
        incStart = add2(fc, off); incEnd = sub2(fc, off);
    }
    v2 c0 = incStart, c1 = incEnd;
    if (clip_segment(&c0, &c1, refStart, neg2(sideDir))) return 0;
    if (clip_segment(&c0, &c1, refEnd, sideDir)) return 0;
    const float refPlaneDist = dot2(rfc, refNormal);
    const uint32_t idBase = best << 1;
    v2 pts[2]; uint32_t ids[2]; uint32_t cnt = 0;
    const v2 cl[2] = {c0, c1};
    for (uint32_t i = 0; i < 2; i++) {
        if (dot2(cl[i], refNormal) <= refPlaneDist + SAT_EPSILON) { pts[cnt] = cl[i]; ids[cnt] = idBase | i; cnt++; }
    }
    if (cnt == 0) return 0;
    emit(out, a, b, normal, depth, cnt, pts[0], cnt > 1 ? pts[1] : mk(0, 0), ids[0], cnt > 1 ? ids[1] : 0);
    return 1;
}

/* collisionBoxPolygon (CollisionMethods/BoxPolygon.cpp:14-319): SAT in the polygon's frame (box X, box Y, then
 * polygon edges; ties go to the better "facing"), reference/incident selection, two clips. A box, B polygon. */
static int box_polygon(const ora_world *w, uint32_t a, uint32_t b, ora_manifold *out)
{
    static const uint32_t BOX_INCIDENT_EDGE_IDS[2][2][2] = {{{1, 2}, {0, 3}}, {{3, 2}, {0, 1}}};
    const v2 pA = mk(w->worldX[a], w->worldY[a]), pB = mk(w->worldX[b], w->worldY[b]);
    const float cA = w->worldCos[a], sA = w->worldSin[a], cB = w->worldCos[b], sB = w->worldSin[b];
    const float hwA = w->boxHalfW[w->shapeIndex[a]], hhA = w->boxHalfH[w->shapeIndex[a]];
    const uint32_t si = w->shapeIndex[b];
    const uint32_t nv = w->polyCount[si];
    const v2 rightB = mk(cB, sB), upB = mk(-sB, cB);
    const float relCos = cA * cB + sA * sB;
    const float relSin = cA * sB - sA * cB;
    const v2 rA = mk(relCos, -relSin), uA = mk(relSin, relCos);
    const v2 dBA = sub2(pA, pB);
    const v2 bc = mk(dot2(dBA, rightB), dot2(dBA, upB));
    v2 nl;
    float depth, bestFacing;
    int bestType; /* 0 box right, 1 box up, 2 polygon edge */
    uint32_t bestIndex = 0;
    float pcxd, pcyd;
    {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (uint32_t k = 0; k < nv; k++) { const float p = dot2(vert(w, si, k), rA); mn = fminf(mn, p); mx = fmaxf(mx, p); }
        const float bcp = dot2(bc, rA);
        mn -= bcp; mx -= bcp;
        const float overlap = hwA + fminf(-mn, mx);
        if (overlap < 0.0f) return 0;
        pcxd = mn + mx;
        depth = overlap; nl = rA; flip_if_negative(&nl, pcxd); bestType = 0; bestFacing = -fabsf(pcxd);
    }
    {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (uint32_t k = 0; k < nv; k++) { const float p = dot2(vert(w, si, k), uA); mn = fminf(mn, p); mx = fmaxf(mx, p); }
        const float bcp = dot2(bc, uA);
        mn -= bcp; mx -= bcp;
        const float overlap = hhA + fminf(-mn, mx);
        if (overlap < 0.0f) return 0;
        pcyd = mn + mx;
        const float facing = -fabsf(pcyd);
        if (overlap < depth || (overlap == depth && facing < bestFacing)) {
            depth = overlap; nl = uA; flip_if_negative(&nl, pcyd); bestType = 1; bestFacing = facing;
        }
    }
    const v2 pcr = mk(pcxd * rA.x + pcyd * uA.x, pcxd * rA.y + pcyd * uA.y);
    for (uint32_t i = 0; i < nv; i++) {
        const v2 ax = nrm(w, si, i);
        const float boxRadius = hwA * fabsf(dot2(ax, rA)) + hhA * fabsf(dot2(ax, uA));
        const float bcp = dot2(bc, ax);
        const float overlap = dot2(ax, vert(w, si, i)) - (bcp - boxRadius);
        if (overlap < 0.0f) return 0;
        const float facing = dot2(ax, pcr);
        if (overlap < depth || (overlap == depth && facing < bestFacing)) {
            depth = overlap; nl = neg2(ax); bestType = 2; bestIndex = i; bestFacing = facing;
        }
    }
    const int refIsBox = bestType != 2;
    v2 rnl, rfc, sd, rs, re, incS, incE;
    uint32_t ie, ie2;
    if (refIsBox) {
        rnl = nl;
        const int useX = bestType == 0;
        const float sign = useX ? dot2(rnl, rA) : dot2(rnl, uA);
        if (useX) { rfc = add2(bc, scl2(rA, sign * hwA)); sd = uA; }
        else { rfc = add2(bc, scl2(uA, sign * hhA)); sd = rA; }
        const v2 eo = scl2(sd, useX ? hhA : hwA);
        rs = add2(rfc, eo); re = sub2(rfc, eo);
        ie = 0;
        float minDot = FLT_MAX;
        for (uint32_t i = 0; i < nv; i++) {
            const float d = dot2(rnl, nrm(w, si, i));
            if (d < minDot) { minDot = d; ie = i; }
        }
        ie2 = next_index(ie, nv);
        incS = vert(w, si, ie); incE = vert(w, si, ie2);
    } else {
        rnl = neg2(nl);
        const uint32_t i0 = bestIndex, i1 = next_index(i0, nv);
        rs = vert(w, si, i0); re = vert(w, si, i1);
        rfc = scl2(add2(rs, re), 0.5f);
        const v2 edge = sub2(re, rs);
        const float len2 = dot2(edge, edge);
        sd = scl2(edge, -1.0f / sqrtf(len2));
        const float dotX = dot2(rnl, rA), dotY = dot2(rnl, uA);
        const int useX = fabsf(dotX) > fabsf(dotY);
        const float sign = -copysignf(1.0f, useX ? dotX : dotY);
        ie = BOX_INCIDENT_EDGE_IDS[useX][sign > 0.0f][0];
        ie2 = BOX_INCIDENT_EDGE_IDS[useX][sign > 0.0f][1];
        v2 fc, off;
        if (useX) { fc = add2(bc, scl2(rA, sign * hwA)); off = scl2(uA, hhA); }
        else { fc = add2(bc, scl2(uA, sign * hhA)); off = scl2(rA, hwA); }
        incS = add2(fc, off); incE = sub2(fc, off);
    }
    v2 c0 = incS, c1 = incE;
    if (clip_segment(&c0, &c1, rs, neg2(sd))) return 0;
    if (clip_segment(&c0, &c1, re, sd)) return 0;
    const uint32_t tag = refIsBox ? REFERENCE_BODY_TAG : 0u;
    const uint32_t id1 = tag | ie, id2 = tag | ie2;
    const float refPlaneDist = dot2(rfc, rnl);
    const v2 nw = add2(scl2(rightB, nl.x), scl2(upB, nl.y));
    v2 pts[2]; uint32_t ids[2]; uint32_t cnt = 0;
    const v2 cl[2] = {c0, c1};
    for (uint32_t i = 0; i < 2; i++) {
        if (dot2(cl[i], rnl) <= refPlaneDist + SAT_EPSILON) {
            pts[cnt] = add2(add2(pB, scl2(rightB, cl[i].x)), scl2(upB, cl[i].y));
            ids[cnt] = i == 0 ? id1 : id2;
            cnt++;
        }
    }
    if (cnt == 0) return 0;
    emit(out, a, b, nw, depth, cnt, pts[0], cnt > 1 ? pts[1] : mk(0, 0), ids[0], cnt > 1 ? ids[1] : 0);
    return 1;
}

/* collisionPolygonPolygon (CollisionMethods/PolygonPolygon.cpp:18-235): B's vertices into A's frame, SAT over A's
 * then B's edge normals (strictly smaller overlap wins, ties go to the smaller "facing"), reference/incident
 * edges, two clips, contacts within SAT_EPSILON of the reference face. */
static int polygon_polygon(const ora_world *w, uint32_t a, uint32_t b, ora_manifold *out)
{
    v2 vB[16], nBA[16];
    const v2 pA = mk(w->worldX[a], w->worldY[a]), pB = mk(w->worldX[b], w->worldY[b]);
    const float cA = w->worldCos[a], sA = w->worldSin[a], cB = w->worldCos[b], sB = w->worldSin[b];
    const uint32_t sa = w->shapeIndex[a], sb = w->shapeIndex[b];
    const uint32_t nA = w->polyCount[sa], nB = w->polyCount[sb];
    const v2 rightA = mk(cA, sA), upA = mk(-sA, cA);
    const v2 cd = sub2(pB, pA);
    const v2 bdl = mk(dot2(cd, rightA), dot2(cd, upA));
    const float relCos = cA * cB + sA * sB;
    const float relSin = cA * sB - sA * cB;
    for (uint32_t i = 0; i < nB; i++) {
        const v2 v = vert(w, sb, i);
        vB[i] = mk(bdl.x + relCos * v.x - relSin * v.y, bdl.y + relSin * v.x + relCos * v.y);
    }
    v2 nl = mk(0, 0);
    float depth = FLT_MAX, bestFacing = FLT_MAX;
    int bestIsB = 0;
    uint32_t bestIndex = 0;
    for (uint32_t i = 0; i < nA; i++) {
        const v2 ax = nrm(w, sa, i);
        float minB = FLT_MAX;
        for (uint32_t j = 0; j < nB; j++) minB = fminf(minB, dot2(vB[j], ax));
        const float overlap = dot2(vert(w, sa, i), ax) - minB;
        if (overlap < 0.0f) return 0;
        const float facing = -dot2(ax, bdl);
        if (overlap > depth) continue;
        if (overlap < depth || facing < bestFacing) {
            depth = overlap; nl = ax; bestIsB = 0; bestIndex = i; bestFacing = facing;
        }
    }
    for (uint32_t i = 0; i < nB; i++) {
        const v2 nb = nrm(w, sb, i);
        const v2 ax = mk(relCos * nb.x - relSin * nb.y, relSin * nb.x + relCos * nb.y);
        nBA[i] = ax;
        float minA = FLT_MAX;
        for (uint32_t j = 0; j < nA; j++) minA = fminf(minA, dot2(vert(w, sa, j), ax));
        const float overlap = dot2(vB[i], ax) - minA;
        if (overlap < 0.0f) return 0;
        const float facing = dot2(ax, bdl);
        if (overlap > depth) continue;
        if (overlap < depth || facing < bestFacing) {
            depth = overlap; nl = neg2(ax); bestIsB = 1; bestIndex = i; bestFacing = facing;
        }
    }
    const int refIsA = !bestIsB;
    const uint32_t refCount = refIsA ? nA : nB, incCount = refIsA ? nB : nA;
    const v2 rnl = refIsA ? nl : neg2(nl);
    const uint32_t i0 = bestIndex, i1 = next_index(i0, refCount);
    const v2 rs = refIsA ? vert(w, sa, i0) : vB[i0];
    const v2 re = refIsA ? vert(w, sa, i1) : vB[i1];
    const v2 rfc = scl2(add2(rs, re), 0.5f);
    const v2 edge = sub2(re, rs);
    const float len2 = dot2(edge, edge);
    const v2 sideDir = scl2(edge, 1.0f / sqrtf(len2));
    uint32_t ie = 0;
    float minDot = FLT_MAX;
    for (uint32_t i = 0; i < incCount; i++) {
        const v2 n = refIsA ? nBA[i] : nrm(w, sa, i);
        const float d = dot2(rnl, n);
        if (d < minDot) { minDot = d; ie = i; }
    }
    const uint32_t ie2 = next_index(ie, incCount);
    v2 c0 = refIsA ? vB[ie] : vert(w, sa, ie);
    v2 c1 = refIsA ? vB[ie2] : vert(w, sa, ie2);
    if (clip_segment(&c0, &c1, rs, sideDir)) return 0;
    if (clip_segment(&c0, &c1, re, neg2(sideDir))) return 0;
    const float refPlaneDist = dot2(rfc, rnl);
    const uint32_t tag = refIsA ? REFERENCE_BODY_TAG : 0u;
    const uint32_t id1 = tag | ie, id2 = tag | ie2;
    const v2 nw = add2(scl2(rightA, nl.x), scl2(upA, nl.y));
    v2 pts[2]; uint32_t ids[2]; uint32_t cnt = 0;
    const v2 cl[2] = {c0, c1};
    for (uint32_t i = 0; i < 2; i++) {
        if (dot2(cl[i], rnl) <= refPlaneDist + SAT_EPSILON) {
            pts[cnt] = add2(add2(pA, scl2(rightA, cl[i].x)), scl2(upA, cl[i].y));
            ids[cnt] = i == 0 ? id1 : id2;
            cnt++;
        }
    }
    if (cnt == 0) return 0;
    emit(out, a, b, nw, depth, cnt, pts[0], cnt > 1 ? pts[1] : mk(0, 0), ids[0], cnt > 1 ? ids[1] : 0);
    return 1;
}

int64_t ora_narrow(const ora_world *w, const uint32_t *pairs, int64_t n_pairs, ora_manifold *out)
{
    int64_t m = 0;
    for (int64_t p = 0; p < n_pairs; p++) {
        /* processPairs orientation (NarrowPhaseCollisionDetector.cpp:649-668): lower shape type first; equal
         * types put the higher dense collider index first. */
        uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
        uint32_t ta = w->shapeType[a], tb = w->shapeType[b];
        if (ta > tb) { uint32_t t = a; a = b; b = t; t = ta; ta = tb; tb = t; }
        else if (ta == tb && b > a) { uint32_t t = a; a = b; b = t; }
        int hit = 0;
        if (ta == ORA_CIRCLE && tb == ORA_CIRCLE) hit = circle_circle(w, a, b, out + m);
        else if (ta == ORA_CIRCLE && tb == ORA_BOX) hit = circle_box(w, a, b, out + m);
        else if (ta == ORA_CIRCLE && tb == ORA_POLYGON) hit = circle_polygon(w, a, b, out + m);
        else if (ta == ORA_BOX && tb == ORA_BOX) hit = box_box(w, a, b, out + m);
        else if (ta == ORA_BOX && tb == ORA_POLYGON) hit = box_polygon(w, a, b, out + m);
        else if (ta == ORA_POLYGON && tb == ORA_POLYGON) hit = polygon_polygon(w, a, b, out + m);
        m += hit;
    }
    return m;
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Warm start (NarrowPhaseCollisionDetector.cpp:272-297 rebuildContactCache, :692-767 finalizeResults;           */
/* makePairKey .h:216-219). A linear scan replaces the hash table: same lookup result, last insert wins.         */
/* ------------------------------------------------------------------------------------------------------------ */

void ora_warm_start(const ora_manifold *prev, const uint32_t *prev_slotA, const uint32_t *prev_slotB, int64_t n_prev,
                    ora_manifold *cur, const uint32_t *cur_slotA, const uint32_t *cur_slotB, int64_t n_cur)
{
    for (int64_t c = 0; c < n_cur; c++) {
        const uint32_t ka = cur_slotA[c] < cur_slotB[c] ? cur_slotA[c] : cur_slotB[c];
        const uint32_t kb = cur_slotA[c] < cur_slotB[c] ? cur_slotB[c] : cur_slotA[c];
        int64_t found = -1;
        for (int64_t p = 0; p < n_prev; p++) {
            const ora_manifold *pm = prev + p;
            const float lanes[4] = {pm->jn[0], pm->jt[0], pm->jn[1], pm->jt[1]};
            uint32_t mask = 0;
            for (int k = 0; k < 4; k++) mask |= (uint32_t)(lanes[k] != 0.0f) << k;
            mask &= (1u << (2u * pm->count)) - 1u;
            if (!mask) continue;
            const uint32_t pa = prev_slotA[p] < prev_slotB[p] ? prev_slotA[p] : prev_slotB[p];
            const uint32_t pb = prev_slotA[p] < prev_slotB[p] ? prev_slotB[p] : prev_slotA[p];
            if (pa == ka && pb == kb) found = p;
        }
        if (found < 0) continue;
        const ora_manifold *pm = prev + found;
        if (prev_slotA[found] != cur_slotA[c] || prev_slotB[found] != cur_slotB[c]) continue;
        for (uint32_t i = 0; i < cur[c].count; i++) {
            const uint32_t id = cur[c].id[i];
            if (pm->count > 0 && id == pm->id[0]) { cur[c].jn[i] = pm->jn[0]; cur[c].jt[i] = pm->jt[0]; }
            else if (pm->count > 1 && id == pm->id[1]) { cur[c].jn[i] = pm->jn[1]; cur[c].jt[i] = pm->jt[1]; }
        }
    }
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Contact solver (Solving/BodyCollisionSolver.cpp:229-980) for REAL = float and REAL = double                   */
/* ------------------------------------------------------------------------------------------------------------ */

#define REAL float
#define RSFX _f32
#include "ora_solver.inc"
#undef REAL
#undef RSFX
#define REAL double
#define RSFX _f64
#include "ora_solver.inc"
#undef REAL
#undef RSFX

void ora_solve(ora_world *w, ora_manifold *m, int64_t n, const int64_t *order, uint32_t vel_iters, uint32_t pos_iters)
{
    const uint32_t nb = w->n_bodies;
    float *vel = malloc(sizeof(float) * 3 * (nb ? nb : 1));
    float *pos = malloc(sizeof(float) * 2 * (nb ? nb : 1));
    float *imp = malloc(sizeof(float) * 4 * (n ? n : 1));
    for (uint32_t i = 0; i < nb; i++) {
        vel[3 * i] = w->velX[i]; vel[3 * i + 1] = w->velY[i]; vel[3 * i + 2] = w->angVel[i];
        pos[2 * i] = w->comX[i]; pos[2 * i + 1] = w->comY[i];
    }
    solve_f32(w, m, n, order, vel_iters, pos_iters, vel, pos, imp);
    for (uint32_t i = 0; i < nb; i++) {
        w->velX[i] = vel[3 * i]; w->velY[i] = vel[3 * i + 1]; w->angVel[i] = vel[3 * i + 2];
        w->comX[i] = pos[2 * i]; w->comY[i] = pos[2 * i + 1];
    }
    for (int64_t c = 0; c < n; c++) {
        m[c].jn[0] = imp[4 * c]; m[c].jt[0] = imp[4 * c + 1]; m[c].jn[1] = imp[4 * c + 2]; m[c].jt[1] = imp[4 * c + 3];
    }
    free(vel); free(pos); free(imp);
}

void ora_solve_f64(ora_world *w, ora_manifold *m, int64_t n, const int64_t *order, uint32_t vel_iters,
                   uint32_t pos_iters, double *io_vel, double *io_pos, double *out_impulses)
{
    solve_f64(w, m, n, order, vel_iters, pos_iters, io_vel, io_pos, out_impulses);
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Collision events (Solving/BodyCollisionSolver.cpp:320-387)                                                    */
/* ------------------------------------------------------------------------------------------------------------ */

int64_t ora_collision_events(const ora_world *w, const ora_manifold *m, int64_t n, const uint32_t *callback,
                             const float *threshold, ora_event *out, int64_t cap)
{
    int64_t k = 0;
    for (int64_t c = 0; c < n; c++) {
        const ora_manifold *d = m + c;
        const uint32_t bA = w->bodyIndex[d->a], bB = w->bodyIndex[d->b];
        const float cAx = w->comX[bA], cAy = w->comY[bA], cBx = w->comX[bB], cBy = w->comY[bB];
        const float iIA = w->invInertia[bA], iIB = w->invInertia[bB];
        const float effMass = w->invMass[bA] + w->invMass[bB];
        const float vAx = w->velX[bA], vAy = w->velY[bA], wA = w->angVel[bA];
        const float vBx = w->velX[bB], vBy = w->velY[bB], wB = w->angVel[bB];
        /* :320-350 the per-point terms of the constraint data; impactImpulse = fmax(impactImpulse, negVn * nm). */
        float impact = 0.0f;
        for (uint32_t i = 0; i < d->count; i++) {
            const float rAx = d->px[i] - cAx, rAy = d->py[i] - cAy, rBx = d->px[i] - cBx, rBy = d->py[i] - cBy;
            const float rAn = (-rAy) * d->nx + rAx * d->ny;
            const float rBn = (-rBy) * d->nx + rBx * d->ny;
            const float nd = effMass + rAn * rAn * iIA + rBn * rBn * iIB;
            const float nm = nd > 0.0f ? 1.0f / nd : 0.0f;
            const float negVn = -(((vBx - vAx) * d->nx + (vBy - vAy) * d->ny) + rBn * wB - rAn * wA);
            impact = rmax_f32(impact, negVn * nm);
        }
        /* :353-387 the event of each side whose collider opted in at a threshold the impulse reaches. */
        if (impact <= 0.0f) continue;
        const uint32_t cbA = callback[d->a], cbB = callback[d->b];
        const int fireA = cbA != 0 && impact >= threshold[d->a];
        const int fireB = cbB != 0 && impact >= threshold[d->b];
        if (!fireA && !fireB) continue;
        const float px = d->count > 1 ? (d->px[0] + d->px[1]) * 0.5f : d->px[0];
        const float py = d->count > 1 ? (d->py[0] + d->py[1]) * 0.5f : d->py[0];
        if (fireA) {
            if (k < cap) {
                ora_event e = {d->a, d->b, bA, bB, cbA, px, py, d->nx, d->ny, impact};
                out[k] = e;
            }
            k++;
        }
        if (fireB) {
            if (k < cap) {
                ora_event e = {d->b, d->a, bB, bA, cbB, px, py, -d->nx, -d->ny, impact};
                out[k] = e;
            }
            k++;
        }
    }
    return k <= cap ? k : -k;
}

/* ------------------------------------------------------------------------------------------------------------ */
/* Islands and sleeping (IslandManager.cpp:7-116; ObjectManager.cpp:1438-1491)                                   */
/* ------------------------------------------------------------------------------------------------------------ */

static uint32_t dsu_find(int32_t *parent, uint32_t x)
{
    while (parent[x] >= 0) {
        const uint32_t p = (uint32_t)parent[x];
        const int32_t gp = parent[p];
        if (gp < 0) return p;
        parent[x] = gp;
        x = (uint32_t)gp;
    }
    return x;
}

uint32_t ora_islands(const ora_world *w, const uint32_t *edges, int64_t n_edges, uint32_t *out_island_id)
{
    const uint32_t db = w->body_starts[2], de = w->body_starts[3];
    const uint32_t count = de - db;
    int32_t *parent = malloc(sizeof(int32_t) * (count ? count : 1));
    uint32_t *rootToId = malloc(sizeof(uint32_t) * (count ? count : 1));
    for (uint32_t i = 0; i < count; i++) parent[i] = -1;
    for (int64_t e = 0; e < n_edges; e++) {
        const uint32_t a = edges[2 * e] - db, b = edges[2 * e + 1] - db;
        if (a >= count || b >= count) continue;
        uint32_t ra = dsu_find(parent, a), rb = dsu_find(parent, b);
        if (ra == rb) continue;
        if (parent[ra] > parent[rb]) { const uint32_t t = ra; ra = rb; rb = t; }
        parent[ra] += parent[rb];
        parent[rb] = (int32_t)ra;
    }
    uint32_t k = 0;
    for (uint32_t i = 0; i < count; i++) if (parent[i] < 0) rootToId[i] = k++;
    for (uint32_t i = 0; i < w->n_bodies; i++) out_island_id[i] = 0xFFFFFFFFu;
    for (uint32_t i = 0; i < count; i++) out_island_id[db + i] = rootToId[dsu_find(parent, i)];
    free(parent); free(rootToId);
    return k;
}

void ora_update_sleeping(ora_world *w, const uint32_t *island_id, uint32_t island_count, float dt,
                         float speed_threshold, float time_threshold, uint8_t *out_sleep)
{
    const uint32_t db = w->body_starts[2], de = w->body_starts[3];
    uint32_t *flags = malloc(sizeof(uint32_t) * (island_count + 1));
    for (uint32_t i = 0; i < island_count; i++) flags[i] = 1;
    flags[island_count] = 0;
    for (uint32_t i = 0; i < w->n_bodies; i++) out_sleep[i] = 0;
    for (uint32_t i = db; i < de; i++) {
        const float speed = sqrtf(w->velX[i] * w->velX[i] + w->velY[i] * w->velY[i]) + fabsf(w->angVel[i]) * w->boundRadius[i];
        const int quiet = speed <= speed_threshold;
        const float timer = (w->sleepTimer[i] + dt) * (float)quiet;
        w->sleepTimer[i] = timer;
        const uint32_t slot = island_id[i] < island_count ? island_id[i] : island_count;
        flags[slot] &= (uint32_t)quiet & (uint32_t)(timer >= time_threshold);
    }
    for (uint32_t i = db; i < de; i++) {
        const uint32_t slot = island_id[i] < island_count ? island_id[i] : island_count;
        if (flags[slot]) out_sleep[i] = 1;
    }
    free(flags);
}
