// Spatial phase kernels: integration, collider poses + AABBs, Morton keys, onesweep radix sort, Karras LBVH build
// and refit, and the candidate-pair query. Reference routines cited per kernel (paths relative to
// PhysicsSimulation-Agony/PS_AGONY2D/).
#include "ag2d_ccd.cuh"
#include "ag2d_kernels.cuh"

namespace ag2d {

// ---------------------------------------------------------------------------------------------------------------
// Integration: Integrator::integratePhase1/2_VelocityVerlet + dampAngularVelocities (Integration/Integrator.cpp:
// 140-299, call order Simulation.cpp:392-407), wrapBodyRotations (LeftOutFunctions.cpp:13-60) and
// computeRotationCosSin (Integrator.cpp:301-311), fused per dynamic body. Elementwise: HBM-bound at 40 B/body.
// ---------------------------------------------------------------------------------------------------------------
// phase: 3 both halves; 1 the first (half kick and damping: Integrator::integratePhase1_VelocityVerlet +
// dampAngularVelocities); 2 the second (position step, half kick, damping, wrap, cos/sin). The body constraints
// run between the two (Simulation.cpp:399-404).
__global__ void k_integrate(DeviceWorld w, const uint32_t* __restrict__ dynBody, const uint8_t* __restrict__ dynSimd,
                            uint32_t nDyn, float dt, float gx, float gy,
                            float dampHalf /* damping^(dt/2), or >= 1 when damping is off */, uint32_t phase)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nDyn; k += gridDim.x * blockDim.x) {
        const uint32_t b = dynBody[k];
        const bool simd = dynSimd ? dynSimd[k] != 0 : k < (nDyn & ~7u);
        float4 v = w.bvel[b];
        float4 p = w.bpos[b];
        const float halfDT = dt * 0.5f;
        const float gdx = gx * halfDT, gdy = gy * halfDT;
        const bool movable = v.w != 0.0f;
        const bool angMovable = p.w != 0.0f;
        if (phase & 1u) {
            if (simd) { v.x += movable ? gdx : 0.0f; v.y += movable ? gdy : 0.0f; }
            else { v.x += gdx * float(movable); v.y += gdy * float(movable); }
            if (dampHalf < 1.0f) {
                const float nv = v.z * dampHalf;
                if (simd) v.z = angMovable ? nv : v.z;
                else { const float m = float(angMovable); v.z = m * nv + (1.0f - m) * v.z; }
            }
            if (!(phase & 2u)) {
                w.bvel[b] = v;
                continue;
            }
        }
        p.x = v.x * dt + p.x;
        p.y = v.y * dt + p.y;
        p.z = v.z * dt + p.z;
        if (simd) { v.x += movable ? gdx : 0.0f; v.y += movable ? gdy : 0.0f; }
        else { v.x += gdx * float(movable); v.y += gdy * float(movable); }
        if (dampHalf < 1.0f) {
            const float nv = v.z * dampHalf;
            if (simd) v.z = angMovable ? nv : v.z;
            else { const float m = float(angMovable); v.z = m * nv + (1.0f - m) * v.z; }
        }
        float wraps;
        p.z = wrap_angle(p.z, simd, wraps);
        w.wrapCount[b] = w.wrapCount[b] + wraps;
        float c, s;
        fast_cos_sin(p.z, simd, c, s);
        w.bvel[b] = v;
        w.bpos[b] = p;
        w.brot[b] = make_float2(c, s);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Collider world pose and AABB: computeColliderWorldPositions/Rotations (Simulation.cpp:673-736) and the shape
// AABB builders (SimulationImpl/ColliderAABBBuilder.cpp:8-136). 'list' selects the colliders with their SIMD-path
// flags (the k-th collider of its world's pass takes the reference's SIMD path iff k < (count & ~7)); null = every
// collider, classified by its index within its world's collider range (the reference's live-range pass), or only
// those of the worlds set in 'worldMask'.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ float4 collider_aabb(const DeviceWorld& w, uint32_t c, float x, float y, float cs, float sn)
{
    const uint32_t packed = w.cshape[c];
    const uint32_t si = shape_index(packed);
    switch (shape_type(packed)) {
    case SHAPE_CIRCLE: {
        const float r = w.circleRadius[si];
        return make_float4(x - r, y - r, x + r, y + r);
    }
    case SHAPE_BOX: {
        const float2 h = w.boxHalf[si];
        const float ac = fabsf(cs), as = fabsf(sn);
        const float ex = ac * h.x + as * h.y;
        const float ey = as * h.x + ac * h.y;
        return make_float4(x - ex, y - ey, x + ex, y + ey);
    }
    case SHAPE_CAPSULE: {   // buildCapsuleAABBs (ColliderAABBBuilder.cpp:138-175): (half length, radius)
        const float2 h = w.boxHalf[si];
        const float ex = fabsf(cs) * h.x + h.y;
        const float ey = fabsf(sn) * h.x + h.y;
        return make_float4(x - ex, y - ey, x + ex, y + ey);
    }
    default: {
        const uint32_t off = w.polyOffset[si], nv = w.polyCount[si];
        float mnx = FLT_MAX, mny = FLT_MAX, mxx = -FLT_MAX, mxy = -FLT_MAX;
        for (uint32_t k = 0; k < nv; k++) {
            const float2 v = w.polyVerts[off + k];
            const float wx = cs * v.x - sn * v.y;
            const float wy = sn * v.x + cs * v.y;
            mnx = rfminf(mnx, wx); mxx = rfmaxf(mxx, wx);
            mny = rfminf(mny, wy); mxy = rfmaxf(mxy, wy);
        }
        return make_float4(x + mnx, y + mny, x + mxx, y + mxy);
    }
    }
}

__global__ void k_collider_pose(DeviceWorld w, const uint32_t* __restrict__ list, const uint8_t* __restrict__ listSimd,
                                uint32_t n, const uint32_t* __restrict__ worldMask)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t c = list ? list[k] : k;
        if (worldMask && !worldMask[w.colWorld[c]]) continue;
        bool simd;
        if (list) {
            simd = listSimd ? listSimd[k] != 0 : k < (n & ~7u);
        } else if (w.colWorld) {
            const uint32_t wd = w.colWorld[c];
            const uint32_t lo = w.worldColStart[wd], hi = w.worldColStart[wd + 1];
            simd = (c - lo) < ((hi - lo) & ~7u);
        } else {
            simd = k < (n & ~7u);
        }
        const uint32_t b = w.cbody[c];
        const float4 off = w.coff[c];
        const float4 bp = w.bpos[b];
        const float2 br = w.brot[b];
        const float x = bp.x + (off.x * br.x - off.y * br.y);
        const float y = bp.y + (off.x * br.y + off.y * br.x);
        float wraps;
        const float rot = wrap_angle(bp.z + off.z, simd, wraps);
        float cs, sn;
        fast_cos_sin(rot, simd, cs, sn);
        w.cpose[c] = make_float4(x, y, cs, sn);
        w.cworldRot[c] = rot;
        w.caabb[c] = collider_aabb(w, c, x, y, cs, sn);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Tree bounds: the union of the AABBs of one tree's colliders (BvhTree::gatherCentroids, BvhTree.cpp:148-188).
// min/max are order-independent, so a block reduction plus ordered-integer atomics gives the sequential result
// (up to the sign of a zero bound).
// ---------------------------------------------------------------------------------------------------------------
// Per world (4 ordered words each). A warp whose lanes all belong to one world reduces first and issues one atomic
// per word; a warp that straddles worlds issues per-lane atomics.
__global__ void k_bounds(const float4* __restrict__ aabb, const uint32_t* __restrict__ list, uint32_t n,
                         const uint32_t* __restrict__ colWorld, uint32_t* __restrict__ bounds)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t base0 = blockIdx.x * blockDim.x;
    if (!colWorld) {
        // One world: per-thread running bounds over the grid-stride loop, then one block reduction and four
        // atomics per block (per-warp atomics on four addresses serialise at one L2 slice for large n).
        float mnx = FLT_MAX, mny = FLT_MAX, mxx = -FLT_MAX, mxy = -FLT_MAX;
        for (uint32_t k = base0 + threadIdx.x; k < n; k += stride) {
            const float4 a = aabb[list ? list[k] : k];
            mnx = fminf(mnx, a.x); mny = fminf(mny, a.y); mxx = fmaxf(mxx, a.z); mxy = fmaxf(mxy, a.w);
        }
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        __shared__ float4 part[32];
        const uint32_t warp = threadIdx.x >> 5, warps = (blockDim.x + 31) >> 5;
        if ((threadIdx.x & 31) == 0) part[warp] = make_float4(mnx, mny, mxx, mxy);
        __syncthreads();
        if (threadIdx.x == 0) {
            float4 r = part[0];
            for (uint32_t k = 1; k < warps; k++) {
                const float4 q = part[k];
                r = make_float4(fminf(r.x, q.x), fminf(r.y, q.y), fmaxf(r.z, q.z), fmaxf(r.w, q.w));
            }
            if (r.x <= r.z) {   // the block saw at least one collider
                atomicMin(bounds + 0, float_to_ordered(r.x));
                atomicMin(bounds + 1, float_to_ordered(r.y));
                atomicMax(bounds + 2, float_to_ordered(r.z));
                atomicMax(bounds + 3, float_to_ordered(r.w));
            }
        }
        return;
    }
    for (uint32_t base = base0; base < n; base += stride) {
        const uint32_t k = base + threadIdx.x;
        const bool valid = k < n;
        const uint32_t c = valid ? (list ? list[k] : k) : 0u;
        const float4 a = valid ? aabb[c] : make_float4(FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX);
        const uint32_t wd = valid ? (colWorld ? colWorld[c] : 0u) : 0xFFFFFFFFu;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        const uint32_t firstLane = __ffs(active) - 1;
        const uint32_t w0 = __shfl_sync(0xffffffffu, wd, firstLane);
        const bool uniform = __all_sync(0xffffffffu, !valid || wd == w0);
        if (uniform) {
            float mnx = a.x, mny = a.y, mxx = a.z, mxy = a.w;
            for (int o = 16; o > 0; o >>= 1) {
                mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
                mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
                mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
                mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
            }
            if ((threadIdx.x & 31) == firstLane && active) {
                uint32_t* b = bounds + 4 * w0;
                atomicMin(b + 0, float_to_ordered(mnx));
                atomicMin(b + 1, float_to_ordered(mny));
                atomicMax(b + 2, float_to_ordered(mxx));
                atomicMax(b + 3, float_to_ordered(mxy));
            }
        } else if (valid) {
            uint32_t* b = bounds + 4 * wd;
            atomicMin(b + 0, float_to_ordered(a.x));
            atomicMin(b + 1, float_to_ordered(a.y));
            atomicMax(b + 2, float_to_ordered(a.z));
            atomicMax(b + 3, float_to_ordered(a.w));
        }
    }
}

__global__ void k_bounds_init(uint32_t* bounds, uint32_t worlds)
{
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < worlds; w += gridDim.x * blockDim.x) {
        bounds[4 * w + 0] = float_to_ordered(FLT_MAX);
        bounds[4 * w + 1] = float_to_ordered(FLT_MAX);
        bounds[4 * w + 2] = float_to_ordered(-FLT_MAX);
        bounds[4 * w + 3] = float_to_ordered(-FLT_MAX);
    }
}

// Elements per world of a work list (for the per-world segment offsets of a tree or a manifold list).
__global__ void k_count_world(const uint32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ elemWorld,
                              uint32_t* __restrict__ counts)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        atomicAdd(counts + elemWorld[list ? list[k] : k], 1u);
}

// SIMD-path flag of each work-list entry: the rank of its element among its world's listed elements, against that
// world's (count & ~7). 'offsets' is the exclusive scan of the list flags over all elements, 'worldStart' the
// first element index of each world.
__global__ void k_simd_flags(const uint32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ offsets,
                             uint32_t nElems, const uint32_t* __restrict__ elemWorld,
                             const uint32_t* __restrict__ worldStart, uint32_t worlds, uint8_t* __restrict__ simd)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t w = elemWorld[list[k]];
        const uint32_t firstElem = worldStart[w], endElem = worldStart[w + 1];
        const uint32_t lo = offsets[firstElem];
        const uint32_t hi = endElem < nElems ? offsets[endElem] : n;
        simd[k] = (k - lo) < ((hi - lo) & ~7u) ? 1u : 0u;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Morton keys: transformCentroids + computeMortonCodes (BvhTree.cpp:191-280). 2 x centroid scaled into [0, 65535]
// per axis by the tree bounds, truncated, bits interleaved (y in the odd bits): a 32-bit key.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_morton(const float4* __restrict__ aabb, const uint32_t* __restrict__ list, uint32_t n,
                         const uint32_t* __restrict__ colWorld, const uint32_t* __restrict__ bounds,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* __restrict__ keyOf)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t c = list ? list[k] : k;
        const uint32_t* b = bounds + 4 * (colWorld ? colWorld[c] : 0u);
        const float bminX = ordered_to_float(b[0]), bminY = ordered_to_float(b[1]);
        const float bmaxX = ordered_to_float(b[2]), bmaxY = ordered_to_float(b[3]);
        const float kEps = 1e-5f;
        const float maxX = rfmaxf(bmaxX, bminX + kEps);
        const float maxY = rfmaxf(bmaxY, bminY + kEps);
        const float clampMax = 65535.0f;
        const float scaleX = clampMax / (maxX - bminX);
        const float scaleY = clampMax / (maxY - bminY);
        const float negScaledMinX = -bminX * scaleX;
        const float negScaledMinY = -bminY * scaleY;
        const float halfScaleX = scaleX * 0.5f;
        const float halfScaleY = scaleY * 0.5f;
        const float4 a = aabb[c];
        const float cx = a.x + a.z;
        const float cy = a.y + a.w;
        float tx = cx * halfScaleX + negScaledMinX;
        float ty = cy * halfScaleY + negScaledMinY;
        tx = tx < 0.0f ? 0.0f : (tx > clampMax ? clampMax : tx);
        ty = ty < 0.0f ? 0.0f : (ty > clampMax ? clampMax : ty);
        const uint32_t key = (part1by1(uint32_t(ty)) << 1) | part1by1(uint32_t(tx));
        keys[k] = key;
        vals[k] = c;
        if (keyOf) keyOf[c] = key;
    }
}

// After the Morton passes: the world id of each sorted element becomes the key of the next (stable) passes, so the
// final order is by (world, Morton key) with ties in collider order.
__global__ void k_world_keys(const uint32_t* __restrict__ vals, uint32_t n, const uint32_t* __restrict__ colWorld,
                             uint32_t* __restrict__ keys)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        keys[i] = colWorld[vals[i]];
}

// First index of every world's segment of a world-grouped list: segStart[w] = offsets[worldStart[w]] (the exclusive
// scan of the list flags over the elements), segStart[worlds] = the list length.
__global__ void k_seg_starts(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ worldStart,
                             uint32_t worlds, uint32_t nElems, const uint32_t* __restrict__ total,
                             uint32_t* __restrict__ segStart)
{
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w <= worlds; w += gridDim.x * blockDim.x) {
        const uint32_t e = worldStart[w];
        segStart[w] = (w == worlds || e >= nElems) ? *total : offsets[e];
    }
}

// Segment starts of the world-grouped manifold list (world of body a, non-decreasing): the thread at each world
// change fills the starts of every world in the gap, so worlds without manifolds get empty segments.
__global__ void k_manifold_segments(const Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                                    const uint32_t* __restrict__ cbody, const uint32_t* __restrict__ bodyWorld,
                                    uint32_t worlds, uint32_t* __restrict__ segStart)
{
    const uint32_t n = *nM;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        const int prev = i == 0 ? -1 : int(bodyWorld[cbody[m[i - 1].a]]);
        const int cur = i == n ? int(worlds) : int(bodyWorld[cbody[m[i].a]]);
        for (int w = prev + 1; w <= cur; w++) segStart[w] = i;
    }
}

// Sorted-order gathers for the tree: Morton key (after the world passes), world id and AABB of every leaf.
__global__ void k_tree_gather(const uint32_t* __restrict__ vals, uint32_t n, const uint32_t* __restrict__ keyOf,
                              const uint32_t* __restrict__ colWorld, const float4* __restrict__ caabb,
                              uint32_t* __restrict__ sortedKey, uint32_t* __restrict__ sortedWorld,
                              float4* __restrict__ leafAabb)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = vals[i];
        if (keyOf) sortedKey[i] = keyOf[c];
        if (colWorld) sortedWorld[i] = colWorld[c];
        leafAabb[i] = caabb[c];
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Onesweep LSD radix sort of (key, value) pairs, 8-bit digits, stable: the same permutation as
// BvhTree::sortByMortonCodes (BvhTree.cpp:282-354). One histogram pass for all four digits, then per digit one
// kernel that ranks a 4096-key tile (warp match-any ranking, striped so ranks follow input order), resolves the
// tile's global digit offsets by decoupled look-back over the preceding tiles, reorders the tile in shared
// memory and writes each digit's run contiguously.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_sort_histogram(const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t sh[4 * 256];
    for (uint32_t i = threadIdx.x; i < 4 * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        atomicAdd(&sh[0 * 256 + (k & 0xFF)], 1u);
        atomicAdd(&sh[1 * 256 + ((k >> 8) & 0xFF)], 1u);
        atomicAdd(&sh[2 * 256 + ((k >> 16) & 0xFF)], 1u);
        atomicAdd(&sh[3 * 256 + (k >> 24)], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 4 * 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// In-place exclusive scan of each 256-bin digit histogram; launched with 4 blocks of 256 threads.
__global__ void k_sort_digit_scan(uint32_t* hist)
{
    __shared__ uint32_t s[256];
    uint32_t* h = hist + blockIdx.x * 256;
    const uint32_t t = threadIdx.x;
    s[t] = h[t];
    __syncthreads();
    for (uint32_t o = 1; o < 256; o <<= 1) {
        const uint32_t v = t >= o ? s[t - o] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    h[t] = s[t] - h[t];
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_pass(
    const uint32_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn, uint32_t* __restrict__ keysOut,
    uint32_t* __restrict__ valsOut, uint32_t n, uint32_t shift, const uint32_t* __restrict__ digitBase,
    uint32_t* __restrict__ tileState, uint32_t* __restrict__ tileCounter, uint32_t* __restrict__ status)
{
    constexpr uint32_t WARPS = SORT_THREADS / 32;
    __shared__ uint32_t warpHist[WARPS][256];
    __shared__ uint32_t digitStart[256];     // exclusive scan of the tile's digit counts
    __shared__ uint32_t globalBase[256];     // global output position of the tile's first key of each digit
    __shared__ uint32_t smKey[SORT_TILE];
    __shared__ uint32_t smVal[SORT_TILE];
    __shared__ uint32_t tileSlot;

    if (threadIdx.x == 0) tileSlot = atomicAdd(tileCounter, 1u);   // tiles start in order: look-back progresses
    for (uint32_t i = threadIdx.x; i < WARPS * 256; i += SORT_THREADS) (&warpHist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = tileSlot;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t segBase = tile * SORT_TILE + warp * (SORT_ITEMS * 32);
    const uint32_t ltMask = (1u << lane) - 1u;

    uint32_t key[SORT_ITEMS], val[SORT_ITEMS], rank[SORT_ITEMS];
#pragma unroll
    for (uint32_t k = 0; k < SORT_ITEMS; k++) {
        const uint32_t idx = segBase + k * 32 + lane;
        const bool valid = idx < n;
        key[k] = valid ? keysIn[idx] : 0u;
        val[k] = valid ? valsIn[idx] : 0u;
        const uint32_t d = valid ? ((key[k] >> shift) & 0xFFu) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & ltMask);
        uint32_t base = 0;
        if (valid) base = warpHist[warp][d];
        __syncwarp();
        if (valid && before == 0) warpHist[warp][d] = base + __popc(peers);
        __syncwarp();
        rank[k] = base + before;
    }
    __syncthreads();

    // Per digit (one thread each): warp offsets within the tile, the tile aggregate, look-back.
    {
        const uint32_t d = threadIdx.x;
        uint32_t running = 0;
#pragma unroll
        for (uint32_t wi = 0; wi < WARPS; wi++) {
            const uint32_t c = warpHist[wi][d];
            warpHist[wi][d] = running;
            running += c;
        }
        volatile uint32_t* state = tileState;
        if (tile == 0) {
            state[d] = (2u << 30) | running;
            globalBase[d] = digitBase[d];
        } else {
            state[tile * 256 + d] = (1u << 30) | running;
            uint32_t prefix = 0;
            int32_t t = int32_t(tile) - 1;
            uint32_t spins = 0;
            // Look back over a window of LOOKBACK predecessors per round trip: their states are loaded together,
            // then summed newest first up to the first inclusive prefix; a tile not yet published restarts the
            // window at that tile. Tile 0 always publishes an inclusive prefix, so the walk ends there at the latest.
            // Only a window that makes no progress counts towards the spin limit.
            constexpr int32_t LOOKBACK = 8;
            bool done = false;
            while (!done && t >= 0) {
                uint32_t s[LOOKBACK];
#pragma unroll
                for (int32_t j = 0; j < LOOKBACK; j++) s[j] = t - j >= 0 ? state[(t - j) * 256 + d] : (2u << 30);
#pragma unroll
                for (int32_t j = 0; j < LOOKBACK; j++) {
                    const uint32_t flag = s[j] >> 30;
                    if (flag == 0) break;   // not published yet: reload from tile t
                    prefix += s[j] & 0x3FFFFFFFu;
                    t--;
                    if (flag == 2) { done = true; break; }
                }
                if (!done && t >= 0 && (s[0] >> 30) == 0 && ++spins > SPIN_LIMIT) {
                    atomicOr(status, STATUS_LOOKBACK_TIMEOUT);
                    break;
                }
            }
            __threadfence();
            state[tile * 256 + d] = (2u << 30) | (prefix + running);
            globalBase[d] = digitBase[d] + prefix;
        }
        digitStart[d] = running;   // scanned below
    }
    __syncthreads();
    // Exclusive scan of the 256 digit counts (digitStart holds counts).
    if (threadIdx.x < 32) {
        uint32_t local[8];
        uint32_t sum = 0;
#pragma unroll
        for (uint32_t j = 0; j < 8; j++) { local[j] = digitStart[lane * 8 + j]; sum += local[j]; }
        uint32_t incl = sum;
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t excl = incl - sum;
#pragma unroll
        for (uint32_t j = 0; j < 8; j++) { digitStart[lane * 8 + j] = excl; excl += local[j]; }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < SORT_ITEMS; k++) {
        const uint32_t idx = segBase + k * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[k] >> shift) & 0xFFu;
            const uint32_t pos = digitStart[d] + warpHist[warp][d] + rank[k];
            smKey[pos] = key[k];
            smVal[pos] = val[k];
        }
    }
    __syncthreads();
    const uint32_t tileBase = tile * SORT_TILE;
    const uint32_t tileN = n - tileBase < SORT_TILE ? n - tileBase : SORT_TILE;
    for (uint32_t i = threadIdx.x; i < tileN; i += SORT_THREADS) {
        const uint32_t k = smKey[i];
        const uint32_t d = (k >> shift) & 0xFFu;
        const uint32_t dst = globalBase[d] + (i - digitStart[d]);
        keysOut[dst] = k;
        valsOut[dst] = smVal[i];
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Karras LBVH over sorted keys (leaf = one collider). Internal node i spans [first, last] of the sorted order and
// splits at the highest differing bit; equal keys are ordered by index (key ++ index), as the reference's stable
// sort orders them. Children: >= 0 internal node, < 0 leaf ~rank. Worlds are independent segments [lo, hi) of the
// sorted order (sorted by world first): keys outside the segment count as unrelated (delta -1), so one build makes
// every world's tree, rooted at internal node lo.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ int lbvh_delta(const uint32_t* keys, int lo, int hi, int i, int j)
{
    if (j < lo || j >= hi) return -1;
    const uint32_t a = keys[i], b = keys[j];
    if (a != b) return __clz(a ^ b);
    // Index tie-break on segment-relative positions: a world's tree does not depend on where its segment starts.
    return 32 + __clz(uint32_t(i - lo) ^ uint32_t(j - lo));
}

// sortedWorld/segStart null: one segment [0, n).
__global__ void k_lbvh_build(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ sortedWorld,
                             const uint32_t* __restrict__ segStart, int n, int2* __restrict__ child,
                             int2* __restrict__ range, int* __restrict__ parent, int* __restrict__ leafParent,
                             float4* __restrict__ meet, NodeRec* __restrict__ rec)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int lo = 0, hi = n;
        if (sortedWorld) {
            const uint32_t wd = sortedWorld[i];
            lo = int(segStart[wd]);
            hi = int(segStart[wd + 1]);
        }
        if (hi - lo == 1) leafParent[i] = -1;
        if (i >= hi - 1) continue;
        meet[i] = make_float4(__uint_as_float(MEET_EMPTY), 0.0f, 0.0f, 0.0f);
        if (i == lo) parent[i] = -1;
        const int d = (lbvh_delta(keys, lo, hi, i, i + 1) - lbvh_delta(keys, lo, hi, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = lbvh_delta(keys, lo, hi, i, i - d);
        int lmax = 2;
        while (lbvh_delta(keys, lo, hi, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (lbvh_delta(keys, lo, hi, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = lbvh_delta(keys, lo, hi, i, j);
        int s = 0, t = l;
        do {
            t = (t + 1) >> 1;
            if (lbvh_delta(keys, lo, hi, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        const int gamma = i + s * d + (d < 0 ? -1 : 0);
        const int first = i < j ? i : j, last = i < j ? j : i;
        const int left = (first == gamma) ? ~gamma : gamma;
        const int right = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
        child[i] = make_int2(left, right);
        range[i] = make_int2(first, last);
        rec[i].child = make_int2(left, right);
        rec[i].last = make_int2(gamma, last);
        if (left < 0) leafParent[~left] = i; else parent[left] = i;
        if (right < 0) leafParent[~right] = i; else parent[right] = i;
    }
}

// Swaps a box into a node's meeting slot with one 16-byte atomic and returns what was there.
__device__ __forceinline__ float4 exchange_box(float4* slot, float4 v)
{
    const unsigned long long lo = uint64_t(__float_as_uint(v.x)) | uint64_t(__float_as_uint(v.y)) << 32;
    const unsigned long long hi = uint64_t(__float_as_uint(v.z)) | uint64_t(__float_as_uint(v.w)) << 32;
    unsigned long long rlo, rhi;
    asm volatile("{\n\t.reg .b128 d, s;\n\tmov.b128 s, {%2, %3};\n\t"
                 "atom.relaxed.gpu.global.exch.b128 d, [%4], s;\n\tmov.b128 {%0, %1}, d;\n\t}"
                 : "=l"(rlo), "=l"(rhi) : "l"(lo), "l"(hi), "l"(slot) : "memory");
    return make_float4(__uint_as_float(uint32_t(rlo)), __uint_as_float(uint32_t(rlo >> 32)),
                       __uint_as_float(uint32_t(rhi)), __uint_as_float(uint32_t(rhi >> 32)));
}

// ---------------------------------------------------------------------------------------------------------------
// Segmented sort of a world-grouped tree list: every world segment [segStart[w], segStart[w + 1]) is sorted by its
// Morton key in shared memory, one CTA per segment, by a bitonic network over (key << 32 | position) so that equal
// keys keep their list order: the result equals the stable (world, key, position) order of the global radix passes.
// A CTA takes only the segments of its size class (minSize, maxSize]; every segment of the list is written to the
// output arrays by exactly one class.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_segment_sort(const uint32_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
                               uint32_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut,
                               const uint32_t* __restrict__ segStart, uint32_t worlds, uint32_t minSize,
                               uint32_t maxSize)
{
    extern __shared__ unsigned long long sortTile[];
    for (uint32_t w = blockIdx.x; w < worlds; w += gridDim.x) {
        const uint32_t lo = segStart[w], n = segStart[w + 1] - lo;
        if (n <= minSize || n > maxSize) continue;
        uint32_t m = 1;
        while (m < n) m <<= 1;
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x)
            sortTile[i] = i < n ? (static_cast<unsigned long long>(keysIn[lo + i]) << 32 | i) : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= m; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                    const uint32_t p = i ^ j;
                    if (p > i) {
                        const unsigned long long a = sortTile[i], b = sortTile[p];
                        if ((a > b) == ((i & k) == 0)) { sortTile[i] = b; sortTile[p] = a; }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long e = sortTile[i];
            keysOut[lo + i] = uint32_t(e >> 32);
            valsOut[lo + i] = valsIn[lo + uint32_t(e)];
        }
        __syncthreads();
    }
}

// Bottom-up AABB refit (BvhTree::fitNodes equivalent). The two subtrees of a node meet in its slot: each swaps its
// bounds in with one 16-byte atomic exchange; the first finds the empty marker and stops, the second receives its
// sibling's bounds in the same operation (no flag, fence or second load on the chain), writes the node's record
// and bounds and carries on upwards.
__global__ void k_lbvh_refit(int n, const int2* __restrict__ child, const int* __restrict__ parent,
                             const int* __restrict__ leafParent, const float4* __restrict__ leafAabb,
                             float4* __restrict__ nodeAabb, float4* __restrict__ meet, NodeRec* __restrict__ rec)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int node = leafParent[i];   // -1 for the leaf of a one-collider segment
        int self = ~i;              // child encoding of the subtree this thread carries up
        float4 box = leafAabb[i];   // its bounds
        while (node >= 0) {
            // The tree links do not depend on the arrival: fetch them before the atomic.
            const int2 c = child[node];
            const int up = parent[node];
            const float4 o = exchange_box(meet + node, box);
            if (__float_as_uint(o.x) == MEET_EMPTY) break;   // first arrival: the sibling carries on
            const int side = c.x == self ? 0 : 1;
            const float4 a = side == 0 ? box : o;
            const float4 b = side == 0 ? o : box;
            __stcg(&rec[node].box[0], a);
            __stcg(&rec[node].box[1], b);
            box = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
            __stcg(nodeAabb + node, box);
            self = node;
            node = up;
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Pair query. For dynamic collider of sorted rank i: every dynamic collider of rank > i whose AABB strictly
// overlaps (BvhNode::overlaps, BvhNode.h:33-38) and has another owner body (LeafPairTesting.h:71-134), then every
// static/sleeping collider that overlaps (cross pairs, ordered (dynamic, other)). One traversal counts each query's
// pairs and keeps the first few; after a scan of the counts they land at their offsets: a deterministic pair list
// ordered by query rank and traversal order.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool strict_overlap(const float4& a, const float4& b)
{
    return a.x < b.z && a.z > b.x && a.y < b.w && a.w > b.y;
}

// All pairs of dynamic collider rank i, in traversal order; emit(k, pair) receives the k-th. Returns the count.
template <class Emit>
__device__ __forceinline__ uint32_t query_one(const TreeView& dyn, const TreeView& other,
                                              const uint32_t* __restrict__ cbody, int i, Emit emit,
                                              uint32_t* __restrict__ status)
{
    const int n = dyn.n;
    const float4 q = dyn.leafAabb[i];
    const uint32_t me = dyn.vals[i];
    const uint32_t myBody = cbody[me];
    // This collider's world: the segments of both trees it is tested against.
    int dlo = 0, dhi = n, olo = 0, ohi = other.n;
    if (dyn.sortedWorld) {
        const uint32_t wd = dyn.sortedWorld[i];
        dlo = int(dyn.segStart[wd]);
        dhi = int(dyn.segStart[wd + 1]);
        if (other.n > 0) {
            olo = int(other.segStart[wd]);
            ohi = int(other.segStart[wd + 1]);
        } else {
            ohi = 0;
        }
    }
    uint32_t count = 0;
    int stack[QUERY_STACK];
    // Self pairs within the dynamic tree.
    if (dhi - dlo > 1) {
        int sp = 0;
        stack[sp++] = dlo;
        while (sp > 0) {
            const int node = stack[--sp];
            const NodeRec r = dyn.rec[node];
#pragma unroll
            for (int side = 0; side < 2; side++) {
                const int ch = side == 0 ? r.child.x : r.child.y;
                const int last = side == 0 ? r.last.x : r.last.y;
                if (last <= i || !strict_overlap(q, r.box[side])) continue;   // every leaf below ranks <= i
                if (ch < 0) {
                    const uint32_t other_c = dyn.vals[~ch];
                    if (cbody[other_c] != myBody) emit(count++, make_uint2(me, other_c));
                } else if (sp < QUERY_STACK) {
                    stack[sp++] = ch;
                } else {
                    atomicOr(status, STATUS_STACK_OVERFLOW);
                }
            }
        }
    }
    // Cross pairs against the static + sleeping tree.
    if (ohi - olo == 1) {
        if (strict_overlap(q, other.leafAabb[olo])) emit(count++, make_uint2(me, other.vals[olo]));
    } else if (ohi - olo > 1 && strict_overlap(q, other.nodeAabb[olo])) {
        int sp = 0;
        stack[sp++] = olo;
        while (sp > 0) {
            const int node = stack[--sp];
            const NodeRec r = other.rec[node];
#pragma unroll
            for (int side = 0; side < 2; side++) {
                const int ch = side == 0 ? r.child.x : r.child.y;
                if (!strict_overlap(q, r.box[side])) continue;
                if (ch < 0) emit(count++, make_uint2(me, other.vals[~ch]));
                else if (sp < QUERY_STACK) stack[sp++] = ch;
                else atomicOr(status, STATUS_STACK_OVERFLOW);
            }
        }
    }
    return count;
}

// The pair query in one kernel: blocks take tiles of blockDim.x queries (dynamic colliders in sorted rank order) in
// ticket order (tileState and the ticket counter zeroed before the launch; at most QUERY_MAX_THREADS threads). Each
// thread traverses once, counting its query's pairs and keeping the first QUERY_STASH in shared memory; the tile
// scans the counts, takes its output offset from the decoupled look-back over the preceding tiles and writes the
// kept pairs in place. A query with more pairs than the stash holds traverses again for the rest, after its tile
// has published its prefix. The pairs come out ordered by query rank, then traversal order; the last tile writes
// the pair count.
__global__ void __launch_bounds__(QUERY_MAX_THREADS) k_query(TreeView dyn, TreeView other,
                                                             const uint32_t* __restrict__ cbody,
                                                             uint2* __restrict__ pairs, uint32_t pairCap,
                                                             uint32_t* __restrict__ total,
                                                             uint32_t* __restrict__ status,
                                                             uint32_t* __restrict__ tileState,
                                                             uint32_t* __restrict__ tileCounter)
{
    __shared__ uint2 kept[QUERY_STASH * QUERY_MAX_THREADS];   // [k][thread]
    __shared__ uint32_t warpBase[QUERY_MAX_THREADS / 32];
    __shared__ uint32_t tileSlot, tileBase;
    const uint32_t n = uint32_t(dyn.n);
    const uint32_t tiles = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    while (true) {
        if (threadIdx.x == 0) tileSlot = atomicAdd(tileCounter, 1u);
        __syncthreads();
        const uint32_t tile = tileSlot;
        if (tile >= tiles) return;
        const uint32_t i = tile * blockDim.x + threadIdx.x;
        uint32_t count = 0;
        if (i < n)
            count = query_one(dyn, other, cbody, int(i), [&](uint32_t k, uint2 pr) {
                if (k < QUERY_STASH) kept[k * blockDim.x + threadIdx.x] = pr;
            }, status);
        // Block scan of the counts: lane prefix within the warp, then the warps' totals.
        uint32_t incl = count;
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warpBase[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t c = lane < nWarps ? warpBase[lane] : 0u;
            uint32_t wi = c;
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            const uint32_t aggregate = __shfl_sync(0xffffffffu, wi, 31);
            if (lane < nWarps) warpBase[lane] = wi - c;
            volatile uint32_t* state = tileState;
            uint32_t prefix = 0;
            if (tile == 0) {
                if (lane == 0) state[0] = (2u << 30) | aggregate;
            } else {
                if (lane == 0) state[tile] = (1u << 30) | aggregate;
                prefix = scan_lookback(tile, tileState, status);
                if (lane == 0) state[tile] = (2u << 30) | (prefix + aggregate);
            }
            if (lane == 0) {
                tileBase = prefix;
                if (tile == tiles - 1) {
                    *total = prefix + aggregate;
                    if (prefix + aggregate > pairCap) atomicOr(status, STATUS_PAIR_OVERFLOW);
                }
            }
        }
        __syncthreads();
        const uint32_t out = tileBase + warpBase[warp] + incl - count;
        const uint32_t keptCount = min(count, QUERY_STASH);
        for (uint32_t k = 0; k < keptCount; k++)
            if (out + k < pairCap) pairs[out + k] = kept[k * blockDim.x + threadIdx.x];
        if (count > QUERY_STASH)
            query_one(dyn, other, cbody, int(i), [&](uint32_t k, uint2 pr) {
                if (k >= QUERY_STASH && out + k < pairCap) pairs[out + k] = pr;
            }, status);
        __syncthreads();   // tileSlot, tileBase, warpBase and the stash are reused by the next tile
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Continuous collision (ContinuousCollisionDetector::processShapeRange / resolve, ContinuousCollisionDetector.cpp:
// 303-531). Per dynamic collider: skip unless both the body and the collider moved more than fastFactor x min
// extent this step; sweep the core circle's AABB through the static colliders of its world's static + sleeping
// tree (sleeping ones are skipped: the reference sweeps the static tree only); keep the earliest time of impact per
// body. 'prevPos' holds each body's (x, y) and 'prevPose' each collider's world pose from before integration.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ float ccd_cast_core(const DeviceWorld& w, uint32_t c, V2 start, V2 d, float dd,
                                               float coreRadius, float best)
{
    const float4 pose = w.cpose[c];
    const float cs = pose.z, sn = pose.w;
    const float rx = start.x - pose.x, ry = start.y - pose.y;
    const V2 q0 = v2(cs * rx + sn * ry, cs * ry - sn * rx);
    const V2 dl = v2(cs * d.x + sn * d.y, cs * d.y - sn * d.x);
    const uint32_t packed = w.cshape[c];
    const uint32_t si = shape_index(packed);
    switch (shape_type(packed)) {
    case SHAPE_CIRCLE: return ccd_cast_circle(q0.x, q0.y, dl.x, dl.y, dd, w.circleRadius[si] + coreRadius, best);
    case SHAPE_BOX: {
        const float2 h = w.boxHalf[si];
        return ccd_cast_box(q0, dl, dd, h.x, h.y, coreRadius, best);
    }
    case SHAPE_CAPSULE: {
        const float2 h = w.boxHalf[si];
        return ccd_cast_capsule(q0, dl, dd, h.x, h.y, coreRadius, best);
    }
    default: {
        const uint32_t off = w.polyOffset[si];
        return ccd_cast_polygon(q0, dl, dd, w.polyVerts + off, w.polyNormals + off, w.polyCount[si], coreRadius, best);
    }
    }
}

__global__ void k_ccd_sweep(DeviceWorld w, const uint32_t* __restrict__ dynCol, uint32_t n, TreeView other,
                            const float4* __restrict__ prevPos, const float4* __restrict__ prevPose,
                            const float* __restrict__ minExtent, uint32_t* __restrict__ hitTime,
                            uint32_t* __restrict__ status)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t c = dynCol[k];
        const uint32_t body = w.cbody[c];
        const float4 com = w.bpos[body], pcom = prevPos[body];
        const float bodyDx = com.x - pcom.x, bodyDy = com.y - pcom.y;
        const float bodyDeltaSq = bodyDx * bodyDx + bodyDy * bodyDy;
        if (bodyDeltaSq <= CCD_MIN_DISPLACEMENT_SQ) continue;
        const float me = minExtent[c];
        if (me <= 0.0f) continue;
        const float threshold = CCD_FAST_FACTOR * me;
        const float thresholdSq = threshold * threshold;
        if (bodyDeltaSq <= thresholdSq) continue;
        const float4 pp = prevPose[c], cp = w.cpose[c];
        const V2 start = v2(pp.x, pp.y), end = v2(cp.x, cp.y);
        const V2 d = end - start;
        const float dd = dot(d, d);
        if (dd <= thresholdSq) continue;
        const float coreRadius = CCD_CORE_FRACTION * me;
        const float4 sweep = make_float4(rfminf(start.x, end.x) - coreRadius, rfminf(start.y, end.y) - coreRadius,
                                         rfmaxf(start.x, end.x) + coreRadius, rfmaxf(start.y, end.y) + coreRadius);
        // This collider's world segment of the static + sleeping tree.
        int lo = 0, hi = other.n;
        if (other.segStart) {
            const uint32_t wd = w.colWorld[c];
            lo = int(other.segStart[wd]);
            hi = int(other.segStart[wd + 1]);
        }
        float best = 1.0f;
        auto leaf = [&](int j) {
            const float4 b = other.leafAabb[j];
            if (!(sweep.x < b.z && sweep.z > b.x && sweep.y < b.w && sweep.w > b.y)) return;
            const uint32_t sc = other.vals[j];
            if (w.bstate[w.cbody[sc]] != STATE_STATIC) return;
            best = rfminf(best, ccd_cast_core(w, sc, start, d, dd, coreRadius, best));
        };
        if (hi - lo == 1) {
            leaf(lo);
        } else if (hi - lo > 1) {
            int stack[QUERY_STACK];
            int sp = 0;
            stack[sp++] = lo;
            while (sp > 0) {
                const int node = stack[--sp];
                const float4 nb = other.nodeAabb[node];
                if (nb.z < sweep.x || nb.x > sweep.z || nb.w < sweep.y || nb.y > sweep.w) continue;
                const int2 ch = other.child[node];
#pragma unroll
                for (int side = 0; side < 2; side++) {
                    const int x = side == 0 ? ch.x : ch.y;
                    if (x < 0) leaf(~x);
                    else if (sp < QUERY_STACK) stack[sp++] = x;
                    else atomicOr(status, STATUS_STACK_OVERFLOW);
                }
            }
        }
        if (best < 1.0f) atomicMin(hitTime + body, float_to_ordered(best));
    }
}

// Colliders of hit bodies move back with their body (worldPos += shift) and get their AABB rebuilt from the moved
// pose (resolve, ContinuousCollisionDetector.cpp:495-512, then buildColliderAABBs). Runs before the bodies move.
__global__ void k_ccd_shift_colliders(DeviceWorld w, const uint32_t* __restrict__ dynCol, uint32_t n,
                                      const float4* __restrict__ prevPos, const uint32_t* __restrict__ hitTime)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t c = dynCol[k];
        const uint32_t body = w.cbody[c];
        const float t = ordered_to_float(hitTime[body]);
        if (!(t < 1.0f)) continue;
        const float back = t - 1.0f;
        const float4 com = w.bpos[body], pcom = prevPos[body];
        const float shiftX = (com.x - pcom.x) * back, shiftY = (com.y - pcom.y) * back;
        float4 p = w.cpose[c];
        p.x += shiftX;
        p.y += shiftY;
        w.cpose[c] = p;
        w.caabb[c] = collider_aabb(w, c, p.x, p.y, p.z, p.w);
    }
}

// Hit bodies move back along their displacement to the time of impact; the hit time returns to 1.
__global__ void k_ccd_shift_bodies(DeviceWorld w, const uint32_t* __restrict__ dynBody, uint32_t n,
                                   const float4* __restrict__ prevPos, uint32_t* __restrict__ hitTime,
                                   StepCounters* counters)
{
    uint32_t moved = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t body = dynBody[k];
        const float t = ordered_to_float(hitTime[body]);
        if (!(t < 1.0f)) continue;
        const float back = t - 1.0f;
        float4 com = w.bpos[body];
        const float4 pcom = prevPos[body];
        const float shiftX = (com.x - pcom.x) * back, shiftY = (com.y - pcom.y) * back;
        com.x += shiftX;
        com.y += shiftY;
        w.bpos[body] = com;
        hitTime[body] = float_to_ordered(1.0f);
        moved++;
    }
    for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(0xffffffffu, moved, o);
    if ((threadIdx.x & 31) == 0 && moved) atomicAdd(&counters->ccdHits, moved);
}

// ---------------------------------------------------------------------------------------------------------------
// Exclusive scan of uint32 (reduce-then-scan, 2048 elements per block); used for pair offsets, compaction and
// work lists.
// ---------------------------------------------------------------------------------------------------------------
// ---------------------------------------------------------------------------------------------------------------
// Single-pass exclusive scan (decoupled look-back, scan_lookback). Tiles of SCAN_TILE elements are taken in ticket
// order by a grid of persistent blocks. tileState and the ticket counter are zeroed before the launch.
// ---------------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(SCAN_THREADS) k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       uint32_t n, const uint32_t* __restrict__ nDev,
                                                       uint32_t* __restrict__ total, uint32_t* __restrict__ tileState,
                                                       uint32_t* __restrict__ tileCounter, uint32_t* __restrict__ status)
{
    __shared__ uint32_t warpSums[SCAN_THREADS / 32];
    __shared__ uint32_t tileSlot, tilePrefix;
    if (nDev) n = min(n, *nDev);
    const uint32_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (n == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0 && total) *total = 0u;
        return;
    }
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    while (true) {
        if (threadIdx.x == 0) tileSlot = atomicAdd(tileCounter, 1u);
        __syncthreads();
        const uint32_t tile = tileSlot;
        if (tile >= tiles) return;
        const uint32_t base = tile * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
        uint32_t v[SCAN_ITEMS];
        uint32_t sum = 0;
#pragma unroll
        for (uint32_t j = 0; j < SCAN_ITEMS; j++) { v[j] = base + j < n ? in[base + j] : 0u; sum += v[j]; }
        uint32_t incl = sum;
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warpSums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t ws = lane < SCAN_THREADS / 32 ? warpSums[lane] : 0u;
            uint32_t wi = ws;
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            const uint32_t aggregate = __shfl_sync(0xffffffffu, wi, SCAN_THREADS / 32 - 1);
            if (lane < SCAN_THREADS / 32) warpSums[lane] = wi - ws;
            volatile uint32_t* state = tileState;
            uint32_t prefix = 0;
            if (tile == 0) {
                if (lane == 0) state[0] = (2u << 30) | aggregate;
            } else {
                if (lane == 0) state[tile] = (1u << 30) | aggregate;
                prefix = scan_lookback(tile, tileState, status);
                if (lane == 0) state[tile] = (2u << 30) | (prefix + aggregate);
            }
            if (lane == 0) {
                tilePrefix = prefix;
                if (total && tile == tiles - 1) *total = prefix + aggregate;
            }
        }
        __syncthreads();
        uint32_t run = tilePrefix + warpSums[warp] + incl - sum;
#pragma unroll
        for (uint32_t j = 0; j < SCAN_ITEMS; j++) {
            if (base + j < n) out[base + j] = run;
            run += v[j];
        }
        __syncthreads();   // tileSlot and warpSums are reused by the next tile
    }
}

}  // namespace ag2d
