// Contact phase kernels: narrow phase, manifold compaction, warm-start hash, sleeping-island wake, solver graph
// colouring, the sequential-impulse solver, islands and sleep flags, and work-list rebuilds. Reference routines are
// cited per kernel (paths relative to PhysicsSimulation-Agony/PS_AGONY2D/).
#include "ag2d_kernels.cuh"

namespace ag2d {

__device__ __forceinline__ ColliderView collider_view(const DeviceWorld& w, uint32_t c)
{
    ColliderView v;
    const float4 p = w.cpose[c];
    v.pos = V2{p.x, p.y};
    v.c = p.z;
    v.s = p.w;
    const uint32_t packed = w.cshape[c];
    v.type = shape_type(packed);
    const uint32_t si = shape_index(packed);
    v.r = 0.0f; v.hw = 0.0f; v.hh = 0.0f; v.verts = nullptr; v.normals = nullptr; v.nv = 0;
    if (v.type == SHAPE_CIRCLE) {
        v.r = w.circleRadius[si];
    } else if (v.type == SHAPE_BOX) {
        const float2 h = w.boxHalf[si];
        v.hw = h.x; v.hh = h.y;
    } else {
        const uint32_t off = w.polyOffset[si];
        v.verts = w.polyVerts + off;
        v.normals = w.polyNormals + off;
        v.nv = w.polyCount[si];
    }
    return v;
}

// ---------------------------------------------------------------------------------------------------------------
// Narrow phase: NarrowPhaseCollisionDetector::processPairs orientation (NarrowPhaseCollisionDetector.cpp:649-668:
// lower shape type first, equal types put the higher collider index first) and the shape-pair method. One thread
// per candidate pair writes the pair's manifold slot and a hit flag; a scan then compacts hits in pair order.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_narrow(DeviceWorld w, const uint2* __restrict__ pairs, const uint32_t* __restrict__ nPairs,
                         uint32_t pairCap, Manifold* __restrict__ slots, uint32_t* __restrict__ hit)
{
    const uint32_t n = min(*nPairs, pairCap);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        uint32_t a = pairs[p].x, b = pairs[p].y;
        uint32_t ta = shape_type(w.cshape[a]), tb = shape_type(w.cshape[b]);
        if (ta > tb || (ta == tb && b > a)) { const uint32_t t = a; a = b; b = t; }
        const ColliderView A = collider_view(w, a), B = collider_view(w, b);
        Contact ct;
        const bool h = collide(A, B, ct);
        hit[p] = h ? 1u : 0u;
        if (h) {
            Manifold m;
            m.a = a; m.b = b; m.nx = ct.n.x; m.ny = ct.n.y; m.depth = ct.depth; m.count = ct.count;
            m.id0 = ct.id[0]; m.px0 = ct.p[0].x; m.py0 = ct.p[0].y;
            if (ct.count > 1) { m.id1 = ct.id[1]; m.px1 = ct.p[1].x; m.py1 = ct.p[1].y; }
            else { m.id1 = 0; m.px1 = 0.0f; m.py1 = 0.0f; }
            m.jn0 = 0.0f; m.jt0 = 0.0f; m.jn1 = 0.0f; m.jt1 = 0.0f;
            slots[p] = m;
        }
    }
}

__global__ void k_compact_manifolds(const Manifold* __restrict__ slots, const uint32_t* __restrict__ hit,
                                    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ nPairs,
                                    uint32_t pairCap, Manifold* __restrict__ out, uint32_t manifoldCap,
                                    uint32_t* __restrict__ nOut, StepCounters* counters)
{
    const uint32_t n = min(*nPairs, pairCap);
    const uint32_t total = n ? offsets[n - 1] + hit[n - 1] : 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *nOut = min(total, manifoldCap);
        counters->manifolds = total;
        if (total > manifoldCap) atomicOr(&counters->status, STATUS_MANIFOLD_OVERFLOW);
    }
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (hit[p] && offsets[p] < manifoldCap) out[offsets[p]] = slots[p];
}

// ---------------------------------------------------------------------------------------------------------------
// Warm start: the previous step's manifolds with a non-zero impulse on an active contact go into an
// open-addressing table keyed by the unordered collider pair (rebuildContactCache, NarrowPhaseCollisionDetector.cpp:
// 272-297; makePairKey .h:216-219); each new manifold of the same ordered pair takes the impulses of the previous
// contacts with equal ids (finalizeResults, :749-766).
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long pair_key(uint32_t a, uint32_t b)
{
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return (static_cast<unsigned long long>(lo) << 32) | hi;
}
__device__ __forceinline__ uint32_t slot_of(unsigned long long key, uint32_t capacity)
{
    const uint32_t shift = 64u - (31u - __clz(capacity));   // capacity is a power of two
    return static_cast<uint32_t>((key * 0x9E3779B97F4A7C15ull) >> shift) & (capacity - 1u);
}

__global__ void k_warm_insert(const Manifold* __restrict__ prev, const uint32_t* __restrict__ nPrev,
                              unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t capacity,
                              uint32_t* __restrict__ status)
{
    const uint32_t n = *nPrev;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Manifold m = prev[i];
        uint32_t mask = uint32_t(m.jn0 != 0.0f) | uint32_t(m.jt0 != 0.0f) << 1 | uint32_t(m.jn1 != 0.0f) << 2 |
                        uint32_t(m.jt1 != 0.0f) << 3;
        mask &= (1u << (2u * m.count)) - 1u;
        if (!mask) continue;
        const unsigned long long key = pair_key(m.a, m.b);
        uint32_t s = slot_of(key, capacity);
        uint32_t probes = 0;
        for (;;) {
            const unsigned long long old = atomicCAS(keys + s, ~0ull, key);
            if (old == ~0ull || old == key) { vals[s] = i; break; }
            s = (s + 1) & (capacity - 1u);
            if (++probes >= capacity) { atomicOr(status, STATUS_HASH_FULL); break; }
        }
    }
}

__global__ void k_warm_lookup(const Manifold* __restrict__ prev, Manifold* __restrict__ cur,
                              const uint32_t* __restrict__ nCur, const unsigned long long* __restrict__ keys,
                              const uint32_t* __restrict__ vals, uint32_t capacity, StepCounters* counters)
{
    const uint32_t n = *nCur;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Manifold& c = cur[i];
        const unsigned long long key = pair_key(c.a, c.b);
        uint32_t s = slot_of(key, capacity);
        uint32_t idx = NO_COLOR;
        for (uint32_t probes = 0; probes < capacity; probes++) {
            const unsigned long long k = keys[s];
            if (k == key) { idx = vals[s]; break; }
            if (k == ~0ull) break;
            s = (s + 1) & (capacity - 1u);
        }
        if (idx == NO_COLOR) continue;
        const Manifold p = prev[idx];
        if (p.a != c.a || p.b != c.b) continue;
        bool any = false;
        for (uint32_t k = 0; k < c.count; k++) {
            const uint32_t id = k == 0 ? c.id0 : c.id1;
            float jn, jt;
            if (p.count > 0 && id == p.id0) { jn = p.jn0; jt = p.jt0; }
            else if (p.count > 1 && id == p.id1) { jn = p.jn1; jt = p.jt1; }
            else continue;
            if (k == 0) { c.jn0 = jn; c.jt0 = jt; } else { c.jn1 = jn; c.jt1 = jt; }
            any = true;
        }
        if (any) atomicAdd(&counters->warmHits, 1u);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Wake: every sleeping body in a manifold wakes its whole island (ObjectManager::wakeIslandsOfContacts,
// SimulationImpl/ObjectManager.h:139-157; wakeOne resets the sleep timer, ObjectManager.cpp:1344-1361).
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_wake(DeviceWorld w, const Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                       uint32_t* __restrict__ wakeIsland, StepCounters* counters)
{
    const uint32_t n = *nM;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t bA = w.cbody[m[i].a], bB = w.cbody[m[i].b];
        // Island ids are body indices (the island's root); anything else is ignored rather than written.
        if (w.bstate[bA] == STATE_SLEEPING && w.sleepIsland[bA] < w.nBodies) wakeIsland[w.sleepIsland[bA]] = 1u;
        if (w.bstate[bB] == STATE_SLEEPING && w.sleepIsland[bB] < w.nBodies) wakeIsland[w.sleepIsland[bB]] = 1u;
    }
}

__global__ void k_wake_apply(DeviceWorld w, const uint32_t* __restrict__ wakeIsland, StepCounters* counters)
{
    uint32_t woke = 0;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.nBodies; b += gridDim.x * blockDim.x) {
        if (w.bstate[b] == STATE_SLEEPING && w.sleepIsland[b] < w.nBodies && wakeIsland[w.sleepIsland[b]]) {
            w.bstate[b] = STATE_DYNAMIC;
            w.sleepTimer[b] = 0.0f;
            woke++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) woke += __shfl_xor_sync(0xffffffffu, woke, o);
    if ((threadIdx.x & 31) == 0 && woke) {
        atomicAdd(&counters->woke, woke);
        counters->topoDirty = 1u;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Graph colouring for the parallel Gauss-Seidel solver. Two manifolds conflict when they share a body with
// non-zero inverse mass (static bodies are never written, the reference's planner makes the same exception:
// Solving/SolvingPlanner.cpp:85-88). Luby / Jones-Plassmann rounds: in round r a manifold takes colour r when its
// priority (a bijective hash of its index) is the largest among the uncoloured manifolds on each of its dynamic
// bodies. Deterministic; colours are independent sets, so solving colour after colour equals a sequential
// Gauss-Seidel sweep in colour-major order. Cooperative launch; grid barriers are bounded.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t priority_of(uint32_t x)
{
    x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;   // murmur3 finalizer
    return x;
}

__global__ void k_color(DeviceWorld w, const Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                        uint32_t* __restrict__ color, unsigned long long* __restrict__ bodyMax,
                        uint32_t* __restrict__ colorCount, uint32_t* __restrict__ colorStart,
                        uint32_t* __restrict__ order, uint32_t* __restrict__ bar, StepCounters* counters)
{
    const uint32_t n = *nM;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    __shared__ uint32_t doneShared;
    for (uint32_t i = gtid; i < n; i += gstride) color[i] = NO_COLOR;
    for (uint32_t c = gtid; c <= MAX_COLORS; c += gstride) colorCount[c] = 0;
    if (!grid_barrier(bar, &counters->status)) return;
    uint32_t rounds = 0;
    for (uint32_t r = 0; r < MAX_COLORS; r++) {
        rounds = r + 1;
        for (uint32_t i = gtid; i < n; i += gstride) {
            if (color[i] != NO_COLOR) continue;
            const unsigned long long key = (static_cast<unsigned long long>(r + 1) << 32) | priority_of(i);
            const uint32_t bA = w.cbody[m[i].a], bB = w.cbody[m[i].b];
            if (w.bvel[bA].w > 0.0f) atomicMax(bodyMax + bA, key);
            if (w.bvel[bB].w > 0.0f) atomicMax(bodyMax + bB, key);
        }
        if (!grid_barrier(bar, &counters->status)) return;
        uint32_t got = 0;
        for (uint32_t i = gtid; i < n; i += gstride) {
            if (color[i] != NO_COLOR) continue;
            const unsigned long long key = (static_cast<unsigned long long>(r + 1) << 32) | priority_of(i);
            const uint32_t bA = w.cbody[m[i].a], bB = w.cbody[m[i].b];
            const bool okA = !(w.bvel[bA].w > 0.0f) || __ldcg(bodyMax + bA) == key;
            const bool okB = !(w.bvel[bB].w > 0.0f) || __ldcg(bodyMax + bB) == key;
            if (okA && okB) { color[i] = r; got++; }
        }
        for (int o = 16; o > 0; o >>= 1) got += __shfl_xor_sync(0xffffffffu, got, o);
        if ((threadIdx.x & 31) == 0 && got) { atomicAdd(colorCount + r, got); atomicAdd(colorCount + MAX_COLORS, got); }
        if (!grid_barrier(bar, &counters->status)) return;
        if (threadIdx.x == 0) doneShared = __ldcg(colorCount + MAX_COLORS);
        __syncthreads();
        if (doneShared >= n) break;
    }
    if (doneShared < n) { if (gtid == 0) atomicOr(&counters->status, STATUS_COLOR_OVERFLOW); return; }
    // Colour offsets (exclusive scan by one thread: at most MAX_COLORS entries) and colour-major order.
    if (gtid == 0) {
        uint32_t run = 0;
        for (uint32_t c = 0; c < rounds; c++) { colorStart[c] = run; run += colorCount[c]; colorCount[c] = 0; }
        colorStart[rounds] = run;
        counters->colors = rounds;
        counters->barrierRounds = rounds;
    }
    if (!grid_barrier(bar, &counters->status)) return;
    for (uint32_t i = gtid; i < n; i += gstride) {
        const uint32_t c = color[i];
        order[colorStart[c] + atomicAdd(colorCount + c, 1u)] = i;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Sequential-impulse solver (Solving/BodyCollisionSolver.cpp): computeConstraintData (:229-390), applyWarmStarting
// (:416-490), solveVelocityConstraints (:492-928; one-contact path, two-contact 2x2 block LCP with iterative
// fallback, iterative friction), solvePositionConstraints (:930-980), scatterImpulses (:392-414). One cooperative
// kernel runs every pass colour by colour with a grid barrier between colours.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void prep_constraint(const DeviceWorld& w, const Manifold& m, uint32_t mi, Constraint& k)
{
    const uint32_t bA = w.cbody[m.a], bB = w.cbody[m.b];
    const float4 vA = w.bvel[bA], vB = w.bvel[bB], pA = w.bpos[bA], pB = w.bpos[bB];
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

__device__ __forceinline__ void warm_constraint(const DeviceWorld& w, const Constraint& k)
{
    float4 vA = w.bvel[k.bodyA], vB = w.bvel[k.bodyB];
    const float tx = -k.ny, ty = k.nx;
    const float jn0 = k.count > 0 ? k.jn0 : 0.0f, jt0 = k.count > 0 ? k.jt0 : 0.0f;
    const float jn1 = k.count > 1 ? k.jn1 : 0.0f, jt1 = k.count > 1 ? k.jt1 : 0.0f;
    const float sn = jn0 + jn1, st = jt0 + jt1;
    const float ix = sn * k.nx + st * tx, iy = sn * k.ny + st * ty;
    vA.x = vA.x - ix * k.imA; vA.y = vA.y - iy * k.imA;
    vB.x = vB.x + ix * k.imB; vB.y = vB.y + iy * k.imB;
    vA.z = vA.z - (jn0 * k.rAn0 + jt0 * k.rAt0 + jn1 * k.rAn1 + jt1 * k.rAt1) * k.iIA;
    vB.z = vB.z + (jn0 * k.rBn0 + jt0 * k.rBt0 + jn1 * k.rBn1 + jt1 * k.rBt1) * k.iIB;
    if (k.imA > 0.0f) w.bvel[k.bodyA] = vA;
    if (k.imB > 0.0f) w.bvel[k.bodyB] = vB;
}

__device__ __forceinline__ void velocity_constraint(const DeviceWorld& w, Constraint& k)
{
    float4 vA = w.bvel[k.bodyA], vB = w.bvel[k.bodyB];
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
    if (imA > 0.0f) w.bvel[k.bodyA] = vA;
    if (imB > 0.0f) w.bvel[k.bodyB] = vB;
}

__device__ __forceinline__ void position_constraint(const DeviceWorld& w, const Constraint& k)
{
    float4 pA = w.bpos[k.bodyA], pB = w.bpos[k.bodyB];
    const float pen = k.penBase - ((pB.x - pA.x) * k.nx + (pB.y - pA.y) * k.ny);
    if (pen <= 0.0f) return;
    const float imA = w.bvel[k.bodyA].w, imB = w.bvel[k.bodyB].w;
    const float total = pen / (imA + imB) * 0.5f;
    const float cA = imA * total, cB = imB * total;
    const float cAx = k.nx * cA, cAy = k.ny * cA, cBx = k.nx * cB, cBy = k.ny * cB;
    if (imA > 0.0f) { pA.x = pA.x - cAx; pA.y = pA.y - cAy; w.bpos[k.bodyA] = pA; }
    if (imB > 0.0f) { pB.x = pB.x + cBx; pB.y = pB.y + cBy; w.bpos[k.bodyB] = pB; }
}

__global__ void k_solve(DeviceWorld w, Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                        const uint32_t* __restrict__ order, const uint32_t* __restrict__ colorStart,
                        Constraint* __restrict__ cons, uint32_t velIters, uint32_t posIters,
                        uint32_t* __restrict__ bar, StepCounters* counters)
{
    const uint32_t n = *nM;
    if (n == 0) return;
    const uint32_t colors = counters->colors;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    for (uint32_t c = gtid; c < n; c += gstride) {
        Constraint k;
        prep_constraint(w, m[order[c]], order[c], k);
        cons[c] = k;
    }
    if (!grid_barrier(bar, &counters->status)) return;
    for (uint32_t col = 0; col < colors; col++) {
        const uint32_t end = colorStart[col + 1];
        for (uint32_t c = colorStart[col] + gtid; c < end; c += gstride) warm_constraint(w, cons[c]);
        if (!grid_barrier(bar, &counters->status)) return;
    }
    for (uint32_t it = 0; it < velIters; it++) {
        for (uint32_t col = 0; col < colors; col++) {
            const uint32_t end = colorStart[col + 1];
            for (uint32_t c = colorStart[col] + gtid; c < end; c += gstride) {
                Constraint k = cons[c];
                velocity_constraint(w, k);
                cons[c].jn0 = k.jn0; cons[c].jt0 = k.jt0; cons[c].jn1 = k.jn1; cons[c].jt1 = k.jt1;
            }
            if (!grid_barrier(bar, &counters->status)) return;
        }
    }
    for (uint32_t it = 0; it < posIters; it++) {
        for (uint32_t col = 0; col < colors; col++) {
            const uint32_t end = colorStart[col + 1];
            for (uint32_t c = colorStart[col] + gtid; c < end; c += gstride) position_constraint(w, cons[c]);
            if (!grid_barrier(bar, &counters->status)) return;
        }
    }
    for (uint32_t c = gtid; c < n; c += gstride) {
        const Constraint& k = cons[c];
        Manifold& d = m[k.manifold];
        d.jn0 = k.jn0; d.jt0 = k.jt0; d.jn1 = k.jn1; d.jt1 = k.jt1;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Islands and sleep (IslandManager.cpp:7-116, ObjectManager::updateSleeping ObjectManager.cpp:1438-1491).
// Union-find over manifolds whose bodies are both dynamic, linking the larger root under the smaller (the root is
// the island's smallest body index: a deterministic island id). A body is quiet when |v| + |w| * boundRadius is at
// most the speed threshold; its timer accumulates while quiet. An island sleeps when every member is quiet and has
// been for the time threshold.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x)
{
    uint32_t p = __ldcg(parent + x);
    while (p != x) {
        const uint32_t gp = __ldcg(parent + p);
        if (gp != p) atomicCAS(parent + x, p, gp);   // path halving, benign races
        x = p;
        p = gp;
    }
    return x;
}

__global__ void k_island_init(DeviceWorld w, uint32_t* __restrict__ parent, uint32_t* __restrict__ flag)
{
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.nBodies; b += gridDim.x * blockDim.x) {
        parent[b] = b;
        flag[b] = 1u;
    }
}

__global__ void k_island_union(DeviceWorld w, const Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                               uint32_t* __restrict__ parent)
{
    const uint32_t n = *nM;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t a = w.cbody[m[i].a], b = w.cbody[m[i].b];
        if (w.bstate[a] != STATE_DYNAMIC || w.bstate[b] != STATE_DYNAMIC) continue;
        for (uint32_t tries = 0; tries < 1u << 20; tries++) {
            uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
            if (ra == rb) break;
            if (ra < rb) { const uint32_t t = ra; ra = rb; rb = t; }   // link the larger root under the smaller
            if (atomicCAS(parent + ra, ra, rb) == ra) break;
        }
    }
}

__global__ void k_island_quiet(DeviceWorld w, uint32_t* __restrict__ parent, uint32_t* __restrict__ flag, float dt,
                               float speedThreshold, float timeThreshold)
{
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.nBodies; b += gridDim.x * blockDim.x) {
        if (w.bstate[b] != STATE_DYNAMIC) continue;
        const float4 v = w.bvel[b];
        const float speed = sqrtf(v.x * v.x + v.y * v.y) + fabsf(v.z) * w.boundRadius[b];
        const bool quiet = speed <= speedThreshold;
        const float timer = (w.sleepTimer[b] + dt) * float(quiet);
        w.sleepTimer[b] = timer;
        if (!(quiet && timer >= timeThreshold)) atomicAnd(flag + uf_find(parent, b), 0u);
    }
}

__global__ void k_island_sleep(DeviceWorld w, uint32_t* __restrict__ parent, const uint32_t* __restrict__ flag,
                               StepCounters* counters)
{
    uint32_t slept = 0;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.nBodies; b += gridDim.x * blockDim.x) {
        if (w.bstate[b] != STATE_DYNAMIC) continue;
        const uint32_t root = uf_find(parent, b);
        if (__ldcg(flag + root)) {
            w.bstate[b] = STATE_SLEEPING;
            w.sleepIsland[b] = root;
            w.sleepTimer[b] = 0.0f;
            slept++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) slept += __shfl_xor_sync(0xffffffffu, slept, o);
    if ((threadIdx.x & 31) == 0 && slept) {
        atomicAdd(&counters->slept, slept);
        counters->topoDirty = 1u;
    }
}

// Work-list flags from body states: dynamic bodies, dynamic colliders, static + sleeping colliders.
__global__ void k_state_flags(const uint8_t* __restrict__ bstate, const uint32_t* __restrict__ cbody,
                              uint32_t nBodies, uint32_t nColliders, uint32_t* __restrict__ bodyDyn,
                              uint32_t* __restrict__ colDyn, uint32_t* __restrict__ colOther)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nBodies; b += stride)
        bodyDyn[b] = bstate[b] == STATE_DYNAMIC;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nColliders; c += stride) {
        const bool dyn = bstate[cbody[c]] == STATE_DYNAMIC;
        colDyn[c] = dyn;
        colOther[c] = !dyn;
    }
}

__global__ void k_scatter_list(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ offset, uint32_t n,
                               uint32_t* __restrict__ list)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) list[offset[i]] = i;
}

}  // namespace ag2d
