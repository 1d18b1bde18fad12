// Graph colouring + sequential-impulse solver as one device routine over a "team" of threads that share a barrier:
// a thread-block cluster (hardware barrier.cluster, large single worlds), one CTA (batched small worlds) or a
// cooperative grid (very large worlds). The per-constraint arithmetic (prep/warm/velocity/position) below is shared
// by every variant.
#pragma once

#include <cooperative_groups.h>

#include "ag2d_kernels.cuh"

namespace ag2d {

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------------------------------------------
// Sequential-impulse solver (Solving/BodyCollisionSolver.cpp): computeConstraintData (:229-390), applyWarmStarting
// (:416-490), solveVelocityConstraints (:492-928; one-contact path, two-contact 2x2 block LCP with iterative
// fallback, iterative friction), solvePositionConstraints (:930-980), scatterImpulses (:392-414). A team runs every
// pass colour by colour with its barrier between colours.
// ---------------------------------------------------------------------------------------------------------------
// Body state seen by the solver, with the colouring words of each body (the round's highest priority and the mask of
// colours taken around the body): global memory indexed by body, or a team's contiguous body range staged in shared
// memory.
struct GlobalBodies {
    float4* vel;
    float4* pos;
    unsigned long long* maxW;    // [bodies], zeroed before the call
    unsigned long long* maskW;   // [bodies], zeroed before the call
    __device__ __forceinline__ float4 v(uint32_t b) const { return vel[b]; }
    __device__ __forceinline__ float4 p(uint32_t b) const { return pos[b]; }
    __device__ __forceinline__ void setV(uint32_t b, const float4& x) const { vel[b] = x; }
    __device__ __forceinline__ void setP(uint32_t b, const float4& x) const { pos[b] = x; }
    __device__ __forceinline__ float invMass(uint32_t b) const { return __ldcg(&vel[b].w); }
    __device__ __forceinline__ unsigned long long* maxWord(uint32_t b) const { return maxW + b; }
    __device__ __forceinline__ unsigned long long* maskWord(uint32_t b) const { return maskW + b; }
    static __device__ __forceinline__ unsigned long long ldWord(const unsigned long long* p) { return __ldcg(p); }
    __device__ __forceinline__ bool stage(uint32_t, uint32_t) const { return false; }
};
// Bodies [base, base + count) in shared memory. With 'lazy' set the colouring words occupy the front of the body
// cache while the team colours (inverse masses then come from global memory), and stage() loads the velocities and
// poses over them once the colours are known: 32 bytes of shared memory a body instead of 48, so more teams fit on
// an SM. Otherwise the team loaded the bodies before colouring and the words have a region of their own.
struct SharedBodies {
    float4* vel;                 // shared: bodies [base, base + count)
    float4* pos;
    unsigned long long* maxW;    // shared, zeroed by the team before colouring
    unsigned long long* maskW;
    uint32_t base;
    uint32_t count = 0;
    const float4* gvel = nullptr;   // lazy: the global velocities (inverse masses while colouring)
    const float4* gpos = nullptr;
    __device__ __forceinline__ float4 v(uint32_t b) const { return vel[b - base]; }
    __device__ __forceinline__ float4 p(uint32_t b) const { return pos[b - base]; }
    __device__ __forceinline__ void setV(uint32_t b, const float4& x) const { vel[b - base] = x; }
    __device__ __forceinline__ void setP(uint32_t b, const float4& x) const { pos[b - base] = x; }
    __device__ __forceinline__ float invMass(uint32_t b) const
    {
        return gvel ? __ldg(&gvel[b].w) : vel[b - base].w;
    }
    // Loads the body cache over the colouring words (lazy only); the caller synchronises the team after it.
    __device__ __forceinline__ bool stage(uint32_t rank, uint32_t size) const
    {
        if (!gvel) return false;
        for (uint32_t i = rank; i < count; i += size) {
            vel[i] = gvel[base + i];
            pos[i] = gpos[base + i];
        }
        return true;
    }
    __device__ __forceinline__ unsigned long long* maxWord(uint32_t b) const { return maxW + (b - base); }
    __device__ __forceinline__ unsigned long long* maskWord(uint32_t b) const { return maskW + (b - base); }
    static __device__ __forceinline__ unsigned long long ldWord(const unsigned long long* p)
    {
        return *static_cast<const volatile unsigned long long*>(p);
    }
};

template <class Bodies>
__device__ __forceinline__ void prep_constraint(const DeviceWorld& w, const Bodies& B, const Manifold& m, uint32_t mi,
                                                Constraint& k)
{
    const uint32_t bA = w.cbody[m.a], bB = w.cbody[m.b];
    const float4 vA = B.v(bA), vB = B.v(bB), pA = B.p(bA), pB = B.p(bB);
    k.bodyA = bA; k.bodyB = bB; k.count = m.count; k.manifold = mi;
    k.nx = m.nx; k.ny = m.ny;
    k.imA = vA.w; k.imB = vB.w; k.iIA = pA.w; k.iIB = pB.w;
    k.jn0 = m.jn0; k.jt0 = m.jt0; k.jn1 = m.jn1; k.jt1 = m.jt1;
    k.penBase = m.depth + ((pB.x - pA.x) * m.nx + (pB.y - pA.y) * m.ny) - 0.001f;
    const float4 matA = w.materials[w.cmat[m.a]], matB = w.materials[w.cmat[m.b]];
    const float e = (matA.x + matB.x) * 0.5f;
    k.sf = sqrtf(rfmaxf(0.0f, matA.y * matB.y));
    k.df = sqrtf(rfmaxf(0.0f, matA.z * matB.z));
    const float effMass = k.imA + k.imB;
    const float tx = -m.ny, ty = m.nx;
    float rAn[2] = {0, 0}, rBn[2] = {0, 0}, rAt[2] = {0, 0}, rBt[2] = {0, 0}, nm[2] = {0, 0}, tm[2] = {0, 0}, bias[2] = {0, 0};
#pragma unroll
    for (uint32_t i = 0; i < 2; i++) {
        if (i >= m.count) break;
        const float px = i == 0 ? m.px0 : m.px1, py = i == 0 ? m.py0 : m.py1;
        const float rAx = px - pA.x, rAy = py - pA.y, rBx = px - pB.x, rBy = py - pB.y;
        rAn[i] = (-rAy) * m.nx + rAx * m.ny;
        rBn[i] = (-rBy) * m.nx + rBx * m.ny;
        rAt[i] = (-rAy) * tx + rAx * ty;
        rBt[i] = (-rBy) * tx + rBx * ty;
        const float nd = effMass + rAn[i] * rAn[i] * k.iIA + rBn[i] * rBn[i] * k.iIB;
        nm[i] = nd > 0.0f ? 1.0f / nd : 0.0f;
        const float td = effMass + rAt[i] * rAt[i] * k.iIA + rBt[i] * rBt[i] * k.iIB;
        tm[i] = td > 0.0f ? 1.0f / td : 0.0f;
        const float negVn = -(((vB.x - vA.x) * m.nx + (vB.y - vA.y) * m.ny) + rBn[i] * vB.z - rAn[i] * vA.z);
        bias[i] = (negVn > 0.0f) ? e * negVn : 0.0f;
    }
    k.rAn0 = rAn[0]; k.rBn0 = rBn[0]; k.rAt0 = rAt[0]; k.rBt0 = rBt[0]; k.nm0 = nm[0]; k.tm0 = tm[0]; k.bias0 = bias[0];
    k.rAn1 = rAn[1]; k.rBn1 = rBn[1]; k.rAt1 = rAt[1]; k.rBt1 = rBt[1]; k.nm1 = nm[1]; k.tm1 = tm[1]; k.bias1 = bias[1];
    k.pad = 0.0f;
}

// Impact impulse of a manifold for collision events (BodyCollisionSolver.cpp:320-350): the largest over its points
// of the approach speed along the normal times the normal effective mass, from the velocities the constraint data
// is built from. The arithmetic is prep_constraint's (rAn, rBn, the normal mass and negVn, in the same order), so
// the value is the one the reference computes beside its constraint data.
__device__ __forceinline__ float impact_impulse(const Manifold& m, float4 vA, float4 vB, float4 pA, float4 pB)
{
    const float effMass = vA.w + vB.w;
    float impact = 0.0f;
#pragma unroll
    for (uint32_t i = 0; i < 2; i++) {
        if (i >= m.count) break;
        const float px = i == 0 ? m.px0 : m.px1, py = i == 0 ? m.py0 : m.py1;
        const float rAx = px - pA.x, rAy = py - pA.y, rBx = px - pB.x, rBy = py - pB.y;
        const float rAn = (-rAy) * m.nx + rAx * m.ny;
        const float rBn = (-rBy) * m.nx + rBx * m.ny;
        const float nd = effMass + rAn * rAn * pA.w + rBn * rBn * pB.w;
        const float nm = nd > 0.0f ? 1.0f / nd : 0.0f;
        const float negVn = -(((vB.x - vA.x) * m.nx + (vB.y - vA.y) * m.ny) + rBn * vB.z - rAn * vA.z);
        impact = rfmaxf(impact, negVn * nm);   // std::fmax: a NaN product leaves the running value
    }
    return impact;
}

template <class Bodies>
__device__ __forceinline__ void warm_constraint(const Bodies& B, const Constraint& k)
{
    float4 vA = B.v(k.bodyA), vB = B.v(k.bodyB);
    const float tx = -k.ny, ty = k.nx;
    const float jn0 = k.count > 0 ? k.jn0 : 0.0f, jt0 = k.count > 0 ? k.jt0 : 0.0f;
    const float jn1 = k.count > 1 ? k.jn1 : 0.0f, jt1 = k.count > 1 ? k.jt1 : 0.0f;
    const float sn = jn0 + jn1, st = jt0 + jt1;
    const float ix = sn * k.nx + st * tx, iy = sn * k.ny + st * ty;
    vA.x = vA.x - ix * k.imA; vA.y = vA.y - iy * k.imA;
    vB.x = vB.x + ix * k.imB; vB.y = vB.y + iy * k.imB;
    vA.z = vA.z - (jn0 * k.rAn0 + jt0 * k.rAt0 + jn1 * k.rAn1 + jt1 * k.rAt1) * k.iIA;
    vB.z = vB.z + (jn0 * k.rBn0 + jt0 * k.rBt0 + jn1 * k.rBn1 + jt1 * k.rBt1) * k.iIB;
    if (k.imA > 0.0f) B.setV(k.bodyA, vA);
    if (k.imB > 0.0f) B.setV(k.bodyB, vB);
}

// One velocity iteration of one constraint on its two bodies' velocities held in registers.
__device__ __forceinline__ void velocity_solve(Constraint& k, float4& vA, float4& vB)
{
    const float imA = k.imA, imB = k.imB, iIA = k.iIA, iIB = k.iIB;
    const float nx = k.nx, ny = k.ny, tx = -ny, ty = nx;
    if (k.count == 1) {
        float jnSingle = 0.0f;
        {
            const float vn = ((vB.x - vA.x) * nx + (vB.y - vA.y) * ny) + k.rBn0 * vB.z - k.rAn0 * vA.z;
            if (!(vn > 0.0f && k.jn0 == 0.0f)) {
                const float jn = (k.bias0 - vn) * k.nm0;
                const float old = k.jn0;
                k.jn0 = rfmaxf(0.0f, old + jn);
                const float dj = k.jn0 - old;
                jnSingle = k.jn0;
                const float ix = dj * nx, iy = dj * ny;
                vA.x = vA.x - ix * imA; vA.y = vA.y - iy * imA;
                vA.z = vA.z - dj * k.rAn0 * iIA;
                vB.x = vB.x + ix * imB; vB.y = vB.y + iy * imB;
                vB.z = vB.z + dj * k.rBn0 * iIB;
            }
        }
        {
            const float slip = ((vB.x - vA.x) * tx + (vB.y - vA.y) * ty) + k.rBt0 * vB.z - k.rAt0 * vA.z;
            const float jt = -slip * k.tm0;
            const float old = k.jt0;
            const float target = old + jt;
            if (fabsf(target) <= jnSingle * k.sf) k.jt0 = target;
            else { const float maxD = jnSingle * k.df; k.jt0 = glm_clamp(target, -maxD, maxD); }
            const float dj = k.jt0 - old;
            const float ix = dj * tx, iy = dj * ty;
            vA.x = vA.x - ix * imA; vA.y = vA.y - iy * imA;
            vA.z = vA.z - dj * k.rAt0 * iIA;
            vB.x = vB.x + ix * imB; vB.y = vB.y + iy * imB;
            vB.z = vB.z + dj * k.rBt0 * iIB;
        }
    } else {
        const float effMass = imA + imB;
        float jnArr0 = 0.0f, jnArr1 = 0.0f;
        bool ok = false;
        {
            const float dvn = (vB.x - vA.x) * nx + (vB.y - vA.y) * ny;
            const float vn0 = dvn + k.rBn0 * vB.z - k.rAn0 * vA.z;
            const float vn1 = dvn + k.rBn1 * vB.z - k.rAn1 * vA.z;
            const float a0 = k.jn0, a1 = k.jn1;
            const float K00 = effMass + k.rAn0 * k.rAn0 * iIA + k.rBn0 * k.rBn0 * iIB;
            const float K11 = effMass + k.rAn1 * k.rAn1 * iIA + k.rBn1 * k.rBn1 * iIB;
            const float K01 = effMass + k.rAn0 * k.rAn1 * iIA + k.rBn0 * k.rBn1 * iIB;
            const float b0 = k.bias0 - vn0 + K00 * a0 + K01 * a1;
            const float b1 = k.bias1 - vn1 + K01 * a0 + K11 * a1;
            const float EPS = 1e-6f;
            float x0 = 0.0f, x1 = 0.0f;
            const float det = K00 * K11 - K01 * K01;
            const float maxK = rfmaxf(K00, K11);
            if (maxK * maxK < 1000.0f * det) {
                const float invDet = 1.0f / det;
                const float s0 = (K11 * b0 - K01 * b1) * invDet;
                const float s1 = (K00 * b1 - K01 * b0) * invDet;
                if (s0 >= -EPS && s1 >= -EPS) { x0 = rfmaxf(s0, 0.0f); x1 = rfmaxf(s1, 0.0f); ok = true; }
            }
            if (!ok && K11 > 0.0f) {
                const float s1 = b1 / K11;
                if (s1 >= -EPS && (K01 * s1 - b0) >= -EPS) { x0 = 0.0f; x1 = rfmaxf(s1, 0.0f); ok = true; }
            }
            if (!ok && K00 > 0.0f) {
                const float s0 = b0 / K00;
                if (s0 >= -EPS && (K01 * s0 - b1) >= -EPS) { x0 = rfmaxf(s0, 0.0f); x1 = 0.0f; ok = true; }
            }
            if (!ok && b0 <= EPS && b1 <= EPS) { x0 = 0.0f; x1 = 0.0f; ok = true; }
            if (ok) {
                const float d0 = x0 - a0, d1 = x1 - a1;
                k.jn0 = x0; k.jn1 = x1;
                jnArr0 = x0; jnArr1 = x1;
                const float sum = d0 + d1;
                const float sA = sum * imA, sB = sum * imB;
                vA.x = vA.x - nx * sA; vA.y = vA.y - ny * sA;
                vB.x = vB.x + nx * sB; vB.y = vB.y + ny * sB;
                vA.z = vA.z - (d0 * k.rAn0 + d1 * k.rAn1) * iIA;
                vB.z = vB.z + (d0 * k.rBn0 + d1 * k.rBn1) * iIB;
            }
        }
        if (!ok) {
#pragma unroll
            for (uint32_t i = 0; i < 2; i++) {
                const float rAn = i == 0 ? k.rAn0 : k.rAn1, rBn = i == 0 ? k.rBn0 : k.rBn1;
                const float bias = i == 0 ? k.bias0 : k.bias1, nmass = i == 0 ? k.nm0 : k.nm1;
                const float vn = ((vB.x - vA.x) * nx + (vB.y - vA.y) * ny) + rBn * vB.z - rAn * vA.z;
                const float jn = (bias - vn) * nmass;
                const float old = i == 0 ? k.jn0 : k.jn1;
                const float acc = rfmaxf(0.0f, old + jn);
                if (i == 0) { k.jn0 = acc; jnArr0 = acc; } else { k.jn1 = acc; jnArr1 = acc; }
                const float dj = acc - old;
                const float ix = dj * nx, iy = dj * ny;
                vA.x = vA.x - ix * imA; vA.y = vA.y - iy * imA;
                vA.z = vA.z - dj * rAn * iIA;
                vB.x = vB.x + ix * imB; vB.y = vB.y + iy * imB;
                vB.z = vB.z + dj * rBn * iIB;
            }
        }
#pragma unroll
        for (uint32_t i = 0; i < 2; i++) {
            const float rAt = i == 0 ? k.rAt0 : k.rAt1, rBt = i == 0 ? k.rBt0 : k.rBt1;
            const float tmass = i == 0 ? k.tm0 : k.tm1;
            const float slip = ((vB.x - vA.x) * tx + (vB.y - vA.y) * ty) + rBt * vB.z - rAt * vA.z;
            const float jt = -slip * tmass;
            const float old = i == 0 ? k.jt0 : k.jt1;
            const float target = old + jt;
            const float jn = i == 0 ? jnArr0 : jnArr1;
            float acc;
            if (fabsf(target) <= jn * k.sf) acc = target;
            else { const float maxD = jn * k.df; acc = glm_clamp(target, -maxD, maxD); }
            if (i == 0) k.jt0 = acc; else k.jt1 = acc;
            const float dj = acc - old;
            const float ix = dj * tx, iy = dj * ty;
            vA.x = vA.x - ix * imA; vA.y = vA.y - iy * imA;
            vA.z = vA.z - dj * rAt * iIA;
            vB.x = vB.x + ix * imB; vB.y = vB.y + iy * imB;
            vB.z = vB.z + dj * rBt * iIB;
        }
    }
}

template <class Bodies>
__device__ __forceinline__ void velocity_constraint(const Bodies& B, Constraint& k)
{
    float4 vA = B.v(k.bodyA), vB = B.v(k.bodyB);
    velocity_solve(k, vA, vB);
    if (k.imA > 0.0f) B.setV(k.bodyA, vA);
    if (k.imB > 0.0f) B.setV(k.bodyB, vB);
}

template <class Bodies>
__device__ __forceinline__ void position_constraint(const Bodies& B, const Constraint& k)
{
    float4 pA = B.p(k.bodyA), pB = B.p(k.bodyB);
    const float pen = k.penBase - ((pB.x - pA.x) * k.nx + (pB.y - pA.y) * k.ny);
    if (pen <= 0.0f) return;
    const float imA = B.v(k.bodyA).w, imB = B.v(k.bodyB).w;
    const float total = pen / (imA + imB) * 0.5f;
    const float cA = imA * total, cB = imB * total;
    const float cAx = k.nx * cA, cAy = k.ny * cA, cBx = k.nx * cB, cBy = k.ny * cB;
    if (imA > 0.0f) { pA.x = pA.x - cAx; pA.y = pA.y - cAy; B.setP(k.bodyA, pA); }
    if (imB > 0.0f) { pB.x = pB.x + cBx; pB.y = pB.y + cBy; B.setP(k.bodyB, pB); }
}


__device__ __forceinline__ uint32_t priority_hash(uint32_t x)
{
    x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;   // murmur3 finalizer (bijective)
    return x;
}

// Colour word of a manifold: colour in the low bits, steps it has kept that colour in the high byte.
constexpr uint32_t COLOR_AGE_SHIFT = 24;
constexpr uint32_t COLOR_MASK = (1u << COLOR_AGE_SHIFT) - 1u;
constexpr uint32_t COLOR_KEEP_STEPS = 16;

// Colour counters: one per colour, then the lengths of the two uncoloured lists, then the colour count.
constexpr uint32_t COLOR_SLOTS = MAX_COLORS + 4;
// Colours 0..63 are chosen first-fit from a body's 64-bit mask of neighbouring colours; a manifold whose bodies see
// all 64 taken gets colour 64 + its round (unique to the round, so still conflict-free).
constexpr uint32_t MAX_ROUNDS = MAX_COLORS - 64;

// Scratch of one world's (or one team of worlds') colouring and solve.
struct SolveScratch {
    uint32_t* color;                  // [manifolds]
    uint32_t* order;                  // [manifolds] colour-major solving order
    unsigned long long* bodyMax;      // [bodies] global colouring words (GlobalBodies), zeroed before the call
    unsigned long long* bodyMask;     // [bodies] colours taken around each body, zeroed before the call
    uint32_t* colorCount;             // [COLOR_SLOTS], zeroed by the routine
    uint32_t* colorStart;             // [MAX_COLORS + 1]
    Constraint* cons;                 // [manifolds]
    const uint32_t* prio;             // [manifolds] colouring priorities, or null: priority_hash(index)
    uint4* listA;                     // [manifolds] uncoloured manifold records, ping
    uint4* listB;                     // [manifolds] uncoloured manifold records, pong
    uint2* pairBodies;                // [manifolds] the two bodies, bit 31 set when the body is dynamic
    const uint32_t* hint;             // [manifolds] colour of the same contact pair last step (NO_COLOR: none), or null
};

// Team barriers. ld() reads a colour counter written by other team members before the last barrier: global memory
// through L2 for the multi-CTA teams, shared memory for one CTA.
struct ClusterSync {
    __device__ __forceinline__ bool operator()() const { cg::this_cluster().sync(); return true; }
    static __device__ __forceinline__ uint32_t ld(const uint32_t* p) { return __ldcg(p); }
};
struct BlockSync {
    __device__ __forceinline__ bool operator()() const { __syncthreads(); return true; }
    static __device__ __forceinline__ uint32_t ld(const uint32_t* p) { return *static_cast<const volatile uint32_t*>(p); }
};
struct GridSync {
    uint32_t* bar;
    uint32_t* status;
    __device__ __forceinline__ bool operator()() const { return grid_barrier(bar, status); }
    static __device__ __forceinline__ uint32_t ld(const uint32_t* p) { return __ldcg(p); }
};

// Constraint records of a team kept in shared memory for the warm, velocity and position passes: seven float4
// fields per constraint, structure of arrays (q[f * cap + c]), so a warp's 16-byte accesses are contiguous. Body
// indices are stored relative to the team's first body (12 bits each, MAX_TEAM_BODY_CAP <= 4096). cap == 0: the
// records stay in global memory (SolveScratch::cons). The arithmetic on a record is the same either way.
struct ConsSmem {
    float4* q = nullptr;
    uint32_t cap = 0;
    uint32_t base = 0;
    static constexpr uint32_t FIELDS = 7;
    __device__ __forceinline__ void store(uint32_t c, const Constraint& k) const
    {
        const uint32_t packed = (k.bodyA - base) | (k.bodyB - base) << 12 | k.count << 24;
        q[c] = make_float4(__uint_as_float(packed), k.penBase, k.nx, k.ny);
        q[cap + c] = make_float4(k.jn0, k.jt0, k.jn1, k.jt1);
        q[2 * cap + c] = make_float4(k.rAn0, k.rBn0, k.rAt0, k.rBt0);
        q[3 * cap + c] = make_float4(k.rAn1, k.rBn1, k.rAt1, k.rBt1);
        q[4 * cap + c] = make_float4(k.nm0, k.tm0, k.bias0, k.nm1);
        q[5 * cap + c] = make_float4(k.tm1, k.bias1, k.sf, k.df);
        q[6 * cap + c] = make_float4(k.imA, k.imB, k.iIA, k.iIB);
    }
    __device__ __forceinline__ void loadHead(uint32_t c, Constraint& k) const
    {
        const float4 a = q[c];
        const uint32_t packed = __float_as_uint(a.x);
        k.bodyA = base + (packed & 0xFFFu);
        k.bodyB = base + ((packed >> 12) & 0xFFFu);
        k.count = packed >> 24;
        k.penBase = a.y; k.nx = a.z; k.ny = a.w;
    }
    __device__ __forceinline__ void load(uint32_t c, Constraint& k) const
    {
        loadHead(c, k);
        const float4 j = q[cap + c], r0 = q[2 * cap + c], r1 = q[3 * cap + c], m0 = q[4 * cap + c],
                     m1 = q[5 * cap + c], ms = q[6 * cap + c];
        k.jn0 = j.x; k.jt0 = j.y; k.jn1 = j.z; k.jt1 = j.w;
        k.rAn0 = r0.x; k.rBn0 = r0.y; k.rAt0 = r0.z; k.rBt0 = r0.w;
        k.rAn1 = r1.x; k.rBn1 = r1.y; k.rAt1 = r1.z; k.rBt1 = r1.w;
        k.nm0 = m0.x; k.tm0 = m0.y; k.bias0 = m0.z; k.nm1 = m0.w;
        k.tm1 = m1.x; k.bias1 = m1.y; k.sf = m1.z; k.df = m1.w;
        k.imA = ms.x; k.imB = ms.y; k.iIA = ms.z; k.iIB = ms.w;
    }
    __device__ __forceinline__ void storeImpulses(uint32_t c, const Constraint& k) const
    {
        q[cap + c] = make_float4(k.jn0, k.jt0, k.jn1, k.jt1);
    }
    __device__ __forceinline__ float4 impulses(uint32_t c) const { return q[cap + c]; }
};
constexpr uint32_t CONS_SMEM_BYTES = ConsSmem::FIELDS * sizeof(float4);

// Pulls the 128-byte constraint of slot c into L1 ahead of the pass that reads it.
__device__ __forceinline__ void prefetch_l1(const void* p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// The constraint slot this thread handles first in colour 'col' (or nothing), prefetched before the barrier that
// precedes that colour's pass.
template <class Sync>
__device__ __forceinline__ void prefetch_colour(const SolveScratch& s, uint32_t col, uint32_t ncol, uint32_t rank)
{
    if (col >= ncol) return;
    const uint32_t c = Sync::ld(s.colorStart + col) + rank;
    if (c < Sync::ld(s.colorStart + col + 1)) prefetch_l1(s.cons + c);
}

// Phases of the solve: what a phase does with its records.
constexpr uint32_t PHASE_WARM = 0, PHASE_VELOCITY = 1, PHASE_POSITION = 2;

// The fields a phase of 'kind' reads from global record c: the head (bodies, count, normal, masses) and, except
// for a position phase, the rest; a position phase takes the penetration base instead.
__device__ __forceinline__ void load_record(const Constraint* __restrict__ cons, uint32_t c, uint32_t kind,
                                            Constraint& k)
{
    const float4* q = reinterpret_cast<const float4*>(cons + c);
    const float4 h0 = q[0], h1 = q[1];
    k.bodyA = __float_as_uint(h0.x); k.bodyB = __float_as_uint(h0.y); k.count = __float_as_uint(h0.z);
    k.manifold = __float_as_uint(h0.w);
    k.nx = h1.x; k.ny = h1.y; k.imA = h1.z; k.imB = h1.w;
    if (kind == PHASE_POSITION) {
        k.penBase = cons[c].penBase;
        return;
    }
    const float4 h2 = q[2], j = q[3], r0 = q[4], m0 = q[5], r1 = q[6], m1 = q[7];
    k.iIA = h2.x; k.iIB = h2.y; k.sf = h2.z; k.df = h2.w;
    k.jn0 = j.x; k.jt0 = j.y; k.jn1 = j.z; k.jt1 = j.w;
    k.rAn0 = r0.x; k.rBn0 = r0.y; k.rAt0 = r0.z; k.rBt0 = r0.w;
    k.nm0 = m0.x; k.tm0 = m0.y; k.bias0 = m0.z; k.penBase = m0.w;
    k.rAn1 = r1.x; k.rBn1 = r1.y; k.rAt1 = r1.z; k.rBt1 = r1.w;
    k.nm1 = m1.x; k.tm1 = m1.y; k.bias1 = m1.z; k.pad = m1.w;
}

// One phase's step on a record held in registers; a velocity step writes the record's impulses back.
template <class Bodies>
__device__ __forceinline__ void solve_record(const Bodies& B, Constraint* __restrict__ cons, uint32_t c, uint32_t kind,
                                             Constraint& k)
{
    if (kind == PHASE_WARM) {
        warm_constraint(B, k);
    } else if (kind == PHASE_VELOCITY) {
        velocity_constraint(B, k);
        *reinterpret_cast<float4*>(&cons[c].jn0) = make_float4(k.jn0, k.jt0, k.jn1, k.jt1);
    } else {
        position_constraint(B, k);
    }
}

// The warm, velocity and position passes with global records, pipelined: the passes are one sequence of phases
// (colour-major within each pass, the barrier between phases); in a phase this thread handles the records
// start + rank, + size, ... of the phase's colour, and the first of them is loaded one phase ahead. A record is
// written only by the thread that handles it (its impulses), so its load may cross the barrier, which orders the
// body state alone: the load is in flight while this phase computes and waits. Same arithmetic, same order as the
// unpipelined passes; more registers (two records live).
template <class Sync, class Bodies>
__device__ bool solve_passes_pipelined(const Bodies& B, const SolveScratch& s, uint32_t ncol, uint32_t velIters,
                                       uint32_t posIters, uint32_t rank, uint32_t size, Sync sync)
{
    const uint32_t nPhase = ncol * (1 + velIters + posIters);
    auto kindOf = [&](uint32_t ph) {
        const uint32_t p = ph / ncol;
        return p == 0 ? PHASE_WARM : (p <= velIters ? PHASE_VELOCITY : PHASE_POSITION);
    };
    constexpr uint32_t NO_REC = 0xFFFFFFFFu;
    Constraint nxt;
    uint32_t cNext = NO_REC;
    if (nPhase) {
        const uint32_t c0 = Sync::ld(s.colorStart) + rank;
        if (c0 < Sync::ld(s.colorStart + 1)) { load_record(s.cons, c0, kindOf(0), nxt); cNext = c0; }
    }
    for (uint32_t ph = 0; ph < nPhase; ph++) {
        const uint32_t col = ph % ncol, kind = kindOf(ph);
        const uint32_t end = Sync::ld(s.colorStart + col + 1);
        Constraint k = nxt;
        uint32_t c = cNext;   // NO_REC (above every end) when this thread has no record in the phase
        cNext = NO_REC;
        if (ph + 1 < nPhase) {
            const uint32_t col2 = (ph + 1) % ncol;
            const uint32_t c2 = Sync::ld(s.colorStart + col2) + rank;
            if (c2 < Sync::ld(s.colorStart + col2 + 1)) { load_record(s.cons, c2, kindOf(ph + 1), nxt); cNext = c2; }
        }
        while (c < end) {
            solve_record(B, s.cons, c, kind, k);
            // One colour: the next phase's record is this one, loaded before this phase's impulses.
            if (cNext == c) { nxt.jn0 = k.jn0; nxt.jt0 = k.jt0; nxt.jn1 = k.jn1; nxt.jt1 = k.jt1; }
            c += size;   // a colour larger than the team
            if (c < end) load_record(s.cons, c, kind, k);
        }
        if (!sync()) return false;
    }
    return true;
}

// Colouring followed by the colour-major solve. Colouring runs Jones-Plassmann rounds: in round r every uncoloured
// manifold whose priority is the largest on each of its dynamic bodies takes the smallest colour not yet taken
// around its dynamic bodies (first fit); winners of one round share no dynamic body, so the colours stay
// conflict-free and depend only on the manifold list and priorities. Each round visits only the manifolds still
// uncoloured (compacted into a list whose order does not affect the result). rank/size: this thread's index in the
// team. Returns false if the colouring ran out of colours or a barrier gave up.
// Colouring with carried colours: a manifold whose collider pair was solved last step (its hint) keeps that
// step's colour when it was a first-fit one (< 64) and has been kept for fewer than COLOR_KEEP_STEPS steps in a
// row (so each contact's place in the solving order is revisited regularly). Two kept manifolds of one colour
// cannot share a dynamic body: their predecessors were coloured together last step, and a body's dynamic flag
// (finite mass) does not change between steps. The other manifolds run the Jones-Plassmann rounds around the kept
// colours. With no hints every manifold runs the rounds. s.color holds colour | age << COLOR_AGE_SHIFT.
// s.pairBodies words: body index | PAIR_DYNAMIC (finite mass) | PAIR_KEPT (first word: colour carried over).
constexpr uint32_t PAIR_DYNAMIC = 0x80000000u, PAIR_KEPT = 0x40000000u, PAIR_BODY = 0x3FFFFFFFu;

template <class Sync, class Bodies, bool PIPELINED = false>
__device__ bool color_and_solve(const DeviceWorld& w, const Bodies& B, Manifold* __restrict__ m, uint32_t n,
                                const SolveScratch& s, uint32_t velIters, uint32_t posIters, uint32_t rank,
                                uint32_t size, Sync sync, uint32_t* __restrict__ outColors, uint32_t* __restrict__ status,
                                ConsSmem cs = ConsSmem{})
{
    for (uint32_t c = rank; c < COLOR_SLOTS; c += size) s.colorCount[c] = 0;
    uint32_t* const nColors = s.colorCount + MAX_COLORS + 3;
    // Each manifold's two bodies and whether they are dynamic, looked up once for all colouring rounds; kept
    // colours are counted and marked around their bodies here.
    constexpr uint32_t DYN = PAIR_DYNAMIC, KEPT = PAIR_KEPT;
    if (s.hint && !sync()) return false;   // the counters are zeroed before kept colours are counted
    uint32_t keptTop = 0;
    for (uint32_t i = rank; i < n; i += size) {
        const uint32_t bA = w.cbody[m[i].a], bB = w.cbody[m[i].b];
        const bool dA = B.invMass(bA) > 0.0f, dB = B.invMass(bB) > 0.0f;
        const uint32_t hw = s.hint ? s.hint[i] : NO_COLOR;
        const uint32_t h = hw & COLOR_MASK, age = hw >> COLOR_AGE_SHIFT;
        const bool kept = hw != NO_COLOR && h < 64 && age + 1 < COLOR_KEEP_STEPS;
        if (kept) {
            s.color[i] = h | (age + 1) << COLOR_AGE_SHIFT;
            atomicAdd(s.colorCount + h, 1u);
            keptTop = max(keptTop, h + 1);
            if (dA) atomicOr(B.maskWord(bA), 1ull << h);
            if (dB) atomicOr(B.maskWord(bB), 1ull << h);
        }
        s.pairBodies[i] = make_uint2(bA | (dA ? DYN : 0u) | (kept ? KEPT : 0u), bB | (dB ? DYN : 0u));
    }
    if (s.hint) {
        for (int o = 16; o > 0; o >>= 1) keptTop = max(keptTop, __shfl_xor_sync(0xffffffffu, keptTop, o));
        if ((threadIdx.x & 31) == 0 && keptTop) atomicMax(nColors, keptTop);
    }
    if (!sync()) return false;
    uint32_t len = n;
    const uint4* in = nullptr;   // round 0 visits every manifold; later rounds the uncoloured records
    // Record j of this round: {manifold, priority, body A | dynamic bit, body B | dynamic bit}. In round 0 a kept
    // manifold's record carries the KEPT bit and takes no part.
    auto rec = [&](uint32_t j) -> uint4 {
        if (in) return in[j];
        const uint2 pb = s.pairBodies[j];
        return make_uint4(j, s.prio ? s.prio[j] : priority_hash(j), pb.x, pb.y);
    };
    constexpr uint32_t BATCH = 4;   // records loaded together per thread (independent loads in flight)
    for (uint32_t r = 0; r < MAX_ROUNDS && len > 0; r++) {
        uint4* out = (r & 1) ? s.listB : s.listA;
        uint32_t* outLen = s.colorCount + MAX_COLORS + 1 + (r & 1);
        // This counter was last read before the barrier that ended the previous round.
        if (rank == 0) *outLen = 0;
        const unsigned long long tag = static_cast<unsigned long long>(r + 1) << 32;
        for (uint32_t j0 = rank; j0 < len; j0 += BATCH * size) {
            uint4 e[BATCH];
#pragma unroll
            for (uint32_t u = 0; u < BATCH; u++) e[u] = j0 + u * size < len ? rec(j0 + u * size) : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (uint32_t u = 0; u < BATCH; u++) {
                if (j0 + u * size >= len) break;
                if (e[u].z & KEPT) continue;
                const unsigned long long key = tag | e[u].y;
                if (e[u].z & DYN) atomicMax(B.maxWord(e[u].z & ~DYN), key);
                if (e[u].w & DYN) atomicMax(B.maxWord(e[u].w & ~DYN), key);
            }
        }
        if (!sync()) return false;
        uint32_t top = 0;
        for (uint32_t j0 = rank; j0 < len; j0 += BATCH * size) {
            uint4 e[BATCH];
#pragma unroll
            for (uint32_t u = 0; u < BATCH; u++) e[u] = j0 + u * size < len ? rec(j0 + u * size) : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (uint32_t u = 0; u < BATCH; u++) {
                if (j0 + u * size >= len) break;
                if (e[u].z & KEPT) continue;
                const uint32_t i = e[u].x;
                const unsigned long long key = tag | e[u].y;
                const uint32_t bA = e[u].z & ~DYN, bB = e[u].w & ~DYN;
                const bool dA = (e[u].z & DYN) != 0, dB = (e[u].w & DYN) != 0;
                if ((!dA || B.ldWord(B.maxWord(bA)) == key) && (!dB || B.ldWord(B.maxWord(bB)) == key)) {
                    const unsigned long long used = (dA ? B.ldWord(B.maskWord(bA)) : 0ull) |
                                                    (dB ? B.ldWord(B.maskWord(bB)) : 0ull);
                    const uint32_t c = used == ~0ull ? 64u + r : uint32_t(__ffsll(static_cast<long long>(~used)) - 1);
                    s.color[i] = c;
                    atomicAdd(s.colorCount + c, 1u);
                    top = max(top, c + 1);
                    if (c < 64) {
                        if (dA) atomicOr(B.maskWord(bA), 1ull << c);
                        if (dB) atomicOr(B.maskWord(bB), 1ull << c);
                    }
                } else {
                    out[atomicAdd(outLen, 1u)] = e[u];
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
        if ((threadIdx.x & 31) == 0 && top) atomicMax(nColors, top);
        if (!sync()) return false;
        len = Sync::ld(outLen);
        in = out;
    }
    if (len > 0) { if (rank == 0) atomicOr(status, STATUS_COLOR_OVERFLOW); return false; }
    const uint32_t ncol = Sync::ld(nColors);
    if (rank == 0) {
        uint32_t run = 0;
        for (uint32_t c = 0; c < ncol; c++) { s.colorStart[c] = run; run += s.colorCount[c]; s.colorCount[c] = 0; }
        s.colorStart[ncol] = run;
        atomicMax(outColors, ncol);
    }
    if (!sync()) return false;
    for (uint32_t i = rank; i < n; i += size) {
        const uint32_t c = s.color[i] & COLOR_MASK;
        s.order[Sync::ld(s.colorStart + c) + atomicAdd(s.colorCount + c, 1u)] = i;
    }
    if (!sync()) return false;
    // The colouring words are no longer needed: a lazily staged body cache is loaded over them now.
    if (B.stage(rank, size) && !sync()) return false;
    // Constraint build for every manifold before any velocity changes (computeConstraintData). The records go to
    // shared memory when the team's fit there (the colouring words they overwrite are no longer needed).
    const bool onChip = cs.cap >= n && cs.q != nullptr;
    for (uint32_t c = rank; c < n; c += size) {
        const uint32_t mi = __ldcg(s.order + c);
        Constraint k;
        prep_constraint(w, B, m[mi], mi, k);
        if (onChip) cs.store(c, k);
        else s.cons[c] = k;
    }
    if (!sync()) return false;
    bool passesDone = false;
    if constexpr (PIPELINED) {
        if (!onChip) {
            if (!solve_passes_pipelined(B, s, ncol, velIters, posIters, rank, size, sync)) return false;
            passesDone = true;
        }
    }
    if (!passesDone) {
        for (uint32_t col = 0; col < ncol; col++) {
            const uint32_t end = Sync::ld(s.colorStart + col + 1);
            for (uint32_t c = Sync::ld(s.colorStart + col) + rank; c < end; c += size) {
                if (onChip) {
                    Constraint k;
                    cs.load(c, k);
                    warm_constraint(B, k);
                } else {
                    warm_constraint(B, s.cons[c]);
                }
            }
            if (!sync()) return false;
        }
        for (uint32_t it = 0; it < velIters; it++) {
            for (uint32_t col = 0; col < ncol; col++) {
                const uint32_t end = Sync::ld(s.colorStart + col + 1);
                for (uint32_t c = Sync::ld(s.colorStart + col) + rank; c < end; c += size) {
                    Constraint k;
                    if (onChip) cs.load(c, k);
                    else k = s.cons[c];
                    velocity_constraint(B, k);
                    if (onChip) cs.storeImpulses(c, k);
                    else *reinterpret_cast<float4*>(&s.cons[c].jn0) = make_float4(k.jn0, k.jt0, k.jn1, k.jt1);
                }
                // The next pass's constraint: from the next colour, or colour 0 of the next iteration.
                if (!onChip) prefetch_colour<Sync>(s, col + 1 < ncol ? col + 1 : 0, ncol, rank);
                if (!sync()) return false;
            }
        }
        for (uint32_t it = 0; it < posIters; it++) {
            for (uint32_t col = 0; col < ncol; col++) {
                const uint32_t end = Sync::ld(s.colorStart + col + 1);
                for (uint32_t c = Sync::ld(s.colorStart + col) + rank; c < end; c += size) {
                    if (onChip) {
                        Constraint k;
                        cs.loadHead(c, k);
                        position_constraint(B, k);
                    } else {
                        position_constraint(B, s.cons[c]);
                    }
                }
                if (!onChip) prefetch_colour<Sync>(s, col + 1 < ncol ? col + 1 : 0, ncol, rank);
                if (!sync()) return false;
            }
        }
    }
    for (uint32_t c = rank; c < n; c += size) {
        if (onChip) {
            const float4 j = cs.impulses(c);
            Manifold& d = m[__ldcg(s.order + c)];
            d.jn0 = j.x; d.jt0 = j.y; d.jn1 = j.z; d.jt1 = j.w;
        } else {
            const Constraint& k = s.cons[c];
            Manifold& d = m[k.manifold];
            d.jn0 = k.jn0; d.jt0 = k.jt0; d.jn1 = k.jn1; d.jt1 = k.jt1;
        }
    }
    return true;
}

constexpr uint32_t SOLVE_CLUSTER_THREADS = 512;

__global__ void __launch_bounds__(SOLVE_CLUSTER_THREADS, 1)
k_color_solve_cluster(DeviceWorld w, Manifold* m, const uint32_t* nM, SolveScratch s, uint32_t velIters,
                      uint32_t posIters, StepCounters* counters);
__global__ void k_color_solve_grid(DeviceWorld w, Manifold* m, const uint32_t* nM, SolveScratch s, uint32_t velIters,
                                   uint32_t posIters, uint32_t* bar, StepCounters* counters);

// Batched worlds: teams of consecutive worlds (team k owns worlds [teamWorld[k], teamWorld[k + 1])), each coloured
// and solved by one CTA with __syncthreads between colours. Teams are taken from the work counter *nextTeam (zeroed
// before the launch) in 'teamOrder' order, largest first. Colouring priorities are world-local manifold indices, so
// the colours of a world do not depend on its team. The CTA size (64 to 512 threads) is a launch parameter;
// a team whose bodies fit 'bodyCap' keeps their state and colouring words in dynamic shared memory, and, when its
// manifolds fit 'consCap', its constraint records too (team_smem_bytes).
constexpr uint32_t MAX_TEAM_BODY_CAP = 4096;   // largest body range a team stages in shared memory
constexpr uint32_t TEAM_SMEM_MAX = 220 * 1024; // dynamic shared memory of a team CTA (sm_100 allows 227 KB in
                                               // all, the kernel's static arrays included)
// Dynamic shared memory of a team CTA: body velocities and poses, then one region holding first the colouring words
// (16 B a body) and then the constraint records (CONS_SMEM_BYTES each, consCap of them).
// With no records on chip (consCap 0) the colouring words share the body cache (SharedBodies, lazy): 32 B a body.
__host__ __device__ constexpr size_t team_smem_bytes(uint32_t bodyCap, uint32_t consCap)
{
    return consCap == 0 ? size_t(bodyCap) * 2 * sizeof(float4)
                        : size_t(bodyCap) * 2 * sizeof(float4) +
                              (size_t(bodyCap) * 16 > size_t(consCap) * CONS_SMEM_BYTES
                                   ? size_t(bodyCap) * 16
                                   : size_t(consCap) * CONS_SMEM_BYTES);
}
// Launch shapes of the CTAs that solve a world larger than the team size (one world each): threads per CTA and
// whether the global-record passes are pipelined (solve_passes_pipelined).
constexpr uint32_t BIG_TEAM_THREADS = 512;
struct TeamLaunch {
    DeviceWorld w;
    Manifold* m;
    const uint32_t* manSeg;
    const uint32_t* teamWorld;
    const uint32_t* teamOrder;
    uint32_t teams;
    uint32_t bodyCap;
    uint32_t consCap;   // constraint records a team keeps in shared memory (0: global memory)
    SolveScratch s;
    uint32_t velIters, posIters;
    uint32_t* nextTeam;
    StepCounters* counters;
    uint32_t* ufParent;   // non-null: each team also links its islands (union-find over its manifolds, roots the
                          // smallest body index) into this array, initialised to parent[b] = b before the launch
};
// Host side: launches the team solver with 'threads' per CTA; returns the launch error.
cudaError_t launch_color_solve_teams(uint32_t threads, bool pipelined, uint32_t grid, cudaStream_t stream,
                                     const TeamLaunch& a);
// Host side: co-resident CTAs per SM of the team solver at this CTA size and shared-memory capacities. Also raises
// the kernel's dynamic shared-memory limit to TEAM_SMEM_MAX (the limit is per kernel, shared by every engine in the
// process, so it is never lowered).
cudaError_t team_solver_blocks_per_sm(uint32_t threads, bool pipelined, uint32_t bodyCap, uint32_t consCap, int* out);

}  // namespace ag2d
