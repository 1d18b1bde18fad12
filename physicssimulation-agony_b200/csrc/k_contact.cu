// Contact phase kernels: narrow phase, manifold compaction, warm-start hash, sleeping-island wake, solver graph
// colouring, the sequential-impulse solver, islands and sleep flags, and work-list rebuilds. Reference routines are
// cited per kernel (paths relative to PhysicsSimulation-Agony/PS_AGONY2D/).
#include "ag2d_solver.cuh"

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
    } else if (v.type == SHAPE_CAPSULE) {
        const float2 h = w.boxHalf[si];   // capsules share the table: (half length, radius)
        v.hw = h.x; v.r = h.y;
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
__device__ __forceinline__ void write_slot(const Contact& ct, uint32_t a, uint32_t b, Manifold* slot)
{
    Manifold m;
    m.a = a; m.b = b; m.nx = ct.n.x; m.ny = ct.n.y; m.depth = ct.depth; m.count = ct.count;
    m.id0 = ct.id[0]; m.px0 = ct.p[0].x; m.py0 = ct.p[0].y;
    if (ct.count > 1) { m.id1 = ct.id[1]; m.px1 = ct.p[1].x; m.py1 = ct.p[1].y; }
    else { m.id1 = 0; m.px1 = 0.0f; m.py1 = 0.0f; }
    m.jn0 = 0.0f; m.jt0 = 0.0f; m.jn1 = 0.0f; m.jt1 = 0.0f;
    *slot = m;
}

// Narrow phase with the manifold compaction fused in. Blocks take tiles of blockDim.x consecutive pairs in ticket
// order (tileState and the ticket counter zeroed before the launch); in a tile each warp takes 32 pairs, one per
// lane. Pairs of other shape types run one per lane; then the warp's polygon-polygon pairs run four at a time, one
// per group of NARROW_GROUP lanes (collide_polygon_polygon_group). Each pair's manifold goes to its slot in shared
// memory; the tile's hits are then counted (warp ballots, then a scan of the warps' counts), its output offset
// comes from the decoupled look-back over the preceding tiles, and the hit pairs' manifolds are copied straight to
// their places: manifolds come out in pair order. The last tile writes the manifold count. Launched with a
// multiple of 32 threads (at most 1024) and NARROW_SMEM_PER_THREAD bytes of dynamic shared memory per thread.
__global__ void k_narrow(DeviceWorld w, const uint2* __restrict__ pairs, const uint32_t* __restrict__ nPairs,
                         uint32_t pairCap, Manifold* __restrict__ out, uint32_t manifoldCap,
                         uint32_t* __restrict__ nOut, StepCounters* counters, uint32_t* __restrict__ tileState,
                         uint32_t* __restrict__ tileCounter)
{
    extern __shared__ __align__(16) unsigned char narrowSmem[];
    // [blockDim] manifold slots, [blockDim] hit flags, then per group A's vertices and B's (in A's frame).
    Manifold* const slot = reinterpret_cast<Manifold*>(narrowSmem);
    uint32_t* const hitS = reinterpret_cast<uint32_t*>(narrowSmem + blockDim.x * sizeof(Manifold));
    V2* const tiles = reinterpret_cast<V2*>(narrowSmem + blockDim.x * (sizeof(Manifold) + sizeof(uint32_t)));
    __shared__ uint32_t warpBase[32];
    __shared__ uint32_t tileSlot, tileBase;
    const uint32_t n = min(*nPairs, pairCap);
    if (n == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { *nOut = 0u; counters->manifolds = 0u; }
        return;
    }
    const uint32_t tiles_n = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    const uint32_t group = lane / NARROW_GROUP, gl = lane % NARROW_GROUP;
    const uint32_t gmask = ((1u << NARROW_GROUP) - 1u) << (group * NARROW_GROUP);
    V2* const sA = tiles + (threadIdx.x / NARROW_GROUP) * 2 * MAX_POLYGON_VERTICES;
    V2* const sB = sA + MAX_POLYGON_VERTICES;
    const uint32_t warpFirst = warp * 32;
    while (true) {
        if (threadIdx.x == 0) tileSlot = atomicAdd(tileCounter, 1u);
        __syncthreads();
        const uint32_t tile = tileSlot;
        if (tile >= tiles_n) return;
        const uint32_t p = tile * blockDim.x + threadIdx.x;
        const bool valid = p < n;
        uint32_t a = 0, b = 0;
        bool pp = false;
        hitS[threadIdx.x] = 0u;
        if (valid) {
            a = pairs[p].x;
            b = pairs[p].y;
            const uint32_t ta = shape_type(w.cshape[a]), tb = shape_type(w.cshape[b]);
            if (ta > tb || (ta == tb && b > a)) { const uint32_t t = a; a = b; b = t; }
            pp = ta == SHAPE_POLYGON && tb == SHAPE_POLYGON;
            if (!pp) {
                const ColliderView A = collider_view(w, a), B = collider_view(w, b);
                Contact ct;
                if (collide(A, B, ct)) {
                    hitS[threadIdx.x] = 1u;
                    write_slot(ct, a, b, slot + threadIdx.x);
                }
            }
        }
        uint32_t todo = __ballot_sync(0xffffffffu, pp);
        while (todo) {
            // Group g takes the g-th remaining polygon-polygon lane; its leader writes that pair's slot and flag.
            uint32_t pick = todo;
            for (uint32_t k = 0; k < group && pick; k++) pick &= pick - 1;
            const bool has = pick != 0;
            const uint32_t src = has ? uint32_t(__ffs(pick) - 1) : 0u;
            const uint32_t ga = __shfl_sync(0xffffffffu, a, src), gb = __shfl_sync(0xffffffffu, b, src);
            for (uint32_t k = 0; k < 32 / NARROW_GROUP && todo; k++) todo &= todo - 1;
            if (has) {
                const ColliderView A = collider_view(w, ga), B = collider_view(w, gb);
                Contact ct;
                const bool h = collide_polygon_polygon_group(A, B, ct, gl, gmask, sA, sB);
                if (gl == 0 && h) {
                    hitS[warpFirst + src] = 1u;
                    write_slot(ct, ga, gb, slot + warpFirst + src);
                }
                __syncwarp(gmask);   // the group's tiles are reused by its next pair
            }
        }
        __syncwarp();
        const bool h = hitS[threadIdx.x] != 0u;
        // Output offsets: the tile's hits in pair order after those of the preceding tiles.
        const uint32_t hits = __ballot_sync(0xffffffffu, h);
        if (lane == 0) warpBase[warp] = __popc(hits);
        __syncthreads();
        if (warp == 0) {
            const uint32_t c = lane < nWarps ? warpBase[lane] : 0u;
            uint32_t incl = c;
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const uint32_t aggregate = __shfl_sync(0xffffffffu, incl, 31);
            if (lane < nWarps) warpBase[lane] = incl - c;
            volatile uint32_t* state = tileState;
            uint32_t prefix = 0;
            if (tile == 0) {
                if (lane == 0) state[0] = (2u << 30) | aggregate;
            } else {
                if (lane == 0) state[tile] = (1u << 30) | aggregate;
                prefix = scan_lookback(tile, tileState, &counters->status);
                if (lane == 0) state[tile] = (2u << 30) | (prefix + aggregate);
            }
            if (lane == 0) {
                tileBase = prefix;
                if (tile == tiles_n - 1) {
                    const uint32_t total = prefix + aggregate;
                    counters->manifolds = total;
                    *nOut = min(total, manifoldCap);
                    if (total > manifoldCap) atomicOr(&counters->status, STATUS_MANIFOLD_OVERFLOW);
                }
            }
        }
        __syncthreads();
        if (h) {
            const uint32_t o = tileBase + warpBase[warp] + __popc(hits & ((1u << lane) - 1u));
            if (o < manifoldCap) out[o] = slot[threadIdx.x];
        }
        __syncthreads();   // tileSlot, tileBase, warpBase, the slots and the vertex tiles are reused by the next tile
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Warm start: the previous step's manifolds go into an open-addressing table keyed by the unordered collider pair,
// those with a non-zero impulse on an active contact flagged (bit 31 of the value: the reference caches only these,
// rebuildContactCache, NarrowPhaseCollisionDetector.cpp:272-297; makePairKey .h:216-219); each new manifold of the
// same ordered pair takes the flagged manifold's impulses of the contacts with equal ids (finalizeResults,
// :749-766). Every new manifold whose pair was there also takes that manifold's colour as its colouring hint.
// ---------------------------------------------------------------------------------------------------------------

// The table: one open-addressing region per world of a batch, [2 seg[w], 2 seg[w + 1]) for the world's
// seg[w + 1] - seg[w] previous manifolds (seg: the previous list's world starts), so a warm-start probe stays in its
// world's few kilobytes and hits in cache; a single world (seg null) uses the whole power-of-two table. Which
// region holds a pair changes nothing but where it is found.
struct WarmRegion {
    uint32_t base, size;   // size 0: the world had no manifolds
    __device__ __forceinline__ uint32_t home(unsigned long long key) const
    {
        return base + uint32_t(((key * 0x9E3779B97F4A7C15ull) >> 32) % size);
    }
    __device__ __forceinline__ uint32_t next(uint32_t s) const { return s + 1 == base + size ? base : s + 1; }
};
__device__ __forceinline__ WarmRegion warm_region(const uint32_t* seg, const uint32_t* colWorld, uint32_t a,
                                                  uint32_t capacity)
{
    if (!seg) return WarmRegion{0u, capacity};
    const uint32_t wd = colWorld[a];
    const uint32_t lo = seg[wd], hi = seg[wd + 1];
    if (hi < lo || 2ull * hi > capacity) return WarmRegion{0u, 0u};   // not a valid segmentation: no region
    return WarmRegion{2u * lo, 2u * (hi - lo)};
}

__global__ void k_warm_insert(const Manifold* __restrict__ prev, const uint32_t* __restrict__ nPrev,
                              unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t capacity,
                              const uint32_t* __restrict__ seg, const uint32_t* __restrict__ colWorld,
                              uint32_t* __restrict__ status)
{
    const uint32_t n = *nPrev;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Manifold m = prev[i];
        uint32_t mask = uint32_t(m.jn0 != 0.0f) | uint32_t(m.jt0 != 0.0f) << 1 | uint32_t(m.jn1 != 0.0f) << 2 |
                        uint32_t(m.jt1 != 0.0f) << 3;
        mask &= (1u << (2u * m.count)) - 1u;
        const unsigned long long key = pair_key(m.a, m.b);
        const WarmRegion r = warm_region(seg, colWorld, m.a, capacity);
        if (r.size == 0) { atomicOr(status, STATUS_HASH_FULL); continue; }   // cannot happen: m is in its world
        uint32_t s = r.home(key);
        uint32_t probes = 0;
        for (;;) {
            const unsigned long long old = atomicCAS(keys + s, ~0ull, key);
            if (old == ~0ull || old == key) { vals[s] = i | (mask ? WARM_CACHED : 0u); break; }
            s = r.next(s);
            if (++probes >= r.size) { atomicOr(status, STATUS_HASH_FULL); break; }
        }
    }
}

__global__ void k_warm_lookup(const Manifold* __restrict__ prev, Manifold* __restrict__ cur,
                              const uint32_t* __restrict__ nCur, const unsigned long long* __restrict__ keys,
                              const uint32_t* __restrict__ vals, uint32_t capacity, const uint32_t* __restrict__ seg,
                              const uint32_t* __restrict__ colWorld, StepCounters* counters,
                              const uint32_t* __restrict__ prevColor, uint32_t* __restrict__ hint)
{
    const uint32_t n = *nCur;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Manifold& c = cur[i];
        const unsigned long long key = pair_key(c.a, c.b);
        const WarmRegion r = warm_region(seg, colWorld, c.a, capacity);
        uint32_t idx = NO_COLOR;
        if (r.size) {
            uint32_t s = r.home(key);
            for (uint32_t probes = 0; probes < r.size; probes++) {
                const unsigned long long k = keys[s];
                if (k == key) { idx = vals[s]; break; }
                if (k == ~0ull) break;
                s = r.next(s);
            }
        }
        if (hint) hint[i] = (idx != NO_COLOR && prevColor) ? prevColor[idx & ~WARM_CACHED] : NO_COLOR;
        if (idx == NO_COLOR || !(idx & WARM_CACHED)) continue;
        idx &= ~WARM_CACHED;
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
            if (w.worldDirty) w.worldDirty[w.bodyWorld[b]] = 1u;
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
// Colouring + solve entry points (ag2d_solver.cuh). Two manifolds conflict when they share a body with non-zero
// inverse mass (static bodies are never written; the reference's planner makes the same exception:
// Solving/SolvingPlanner.cpp:85-88). Colours are independent sets, so solving colour after colour equals a
// sequential Gauss-Seidel sweep in colour-major order.
// ---------------------------------------------------------------------------------------------------------------

// One thread-block cluster runs the whole colouring and solve with hardware cluster barriers between colours.
__global__ void __launch_bounds__(SOLVE_CLUSTER_THREADS, 1)
k_color_solve_cluster(DeviceWorld w, Manifold* m, const uint32_t* nM, SolveScratch s, uint32_t velIters,
                      uint32_t posIters, StepCounters* counters)
{
    const cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank() * blockDim.x + threadIdx.x;
    const uint32_t size = cluster.num_blocks() * blockDim.x;
    color_and_solve(w, GlobalBodies{w.bvel, w.bpos, s.bodyMax, s.bodyMask}, m, *nM, s, velIters, posIters, rank, size,
                    ClusterSync{},
                    &counters->colors,
                    &counters->status);
}

// Cooperative grid variant (bounded software grid barrier) for manifold counts beyond one cluster's reach.
__global__ void k_color_solve_grid(DeviceWorld w, Manifold* m, const uint32_t* nM, SolveScratch s, uint32_t velIters,
                                   uint32_t posIters, uint32_t* bar, StepCounters* counters)
{
    const uint32_t rank = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t size = gridDim.x * blockDim.x;
    color_and_solve(w, GlobalBodies{w.bvel, w.bpos, s.bodyMax, s.bodyMask}, m, *nM, s, velIters, posIters, rank,
                    size, GridSync{bar, &counters->status},
                    &counters->colors, &counters->status);
}

// Batched worlds: each CTA takes the next team of consecutive worlds, whose manifolds are one contiguous range of
// the world-grouped list, and colours + solves that range as one problem (the worlds share no body, so their
// colour classes simply merge). Priorities are world-local indices: every world gets the colouring, hence the
// solving order, it has when stepped on its own, whichever team it is in. A team whose bodies fit the dynamic
// shared memory (bodyCap bodies) keeps their velocities, poses and colouring words there. The solver is bound by
// load latency and barriers, so what counts is how many teams an SM holds at once: the colouring words share the
// body cache when the records stay in global memory (32 B of shared memory a body), and the unpipelined variant is
// held to 64 registers a thread (1024 threads an SM).
// Union-find over a parent array in shared or global memory (generic addressing; volatile reads see other SMs'
// links), linking the larger root under the smaller, so every island's root is its smallest body index whatever
// the order of the links (IslandManager's islands, the same roots k_island_union gives).
__device__ __forceinline__ uint32_t team_find(uint32_t* par, uint32_t x)
{
    volatile uint32_t* p = par;
    uint32_t px = p[x];
    for (uint32_t guard = 0; px != x && guard < (1u << 20); guard++) {
        const uint32_t gp = p[px];
        if (gp != px) atomicCAS(par + x, px, gp);   // path halving, benign races
        x = px;
        px = gp;
    }
    return x;
}
__device__ __forceinline__ void team_union(uint32_t* par, uint32_t a, uint32_t b)
{
    for (uint32_t tries = 0; tries < (1u << 20); tries++) {
        uint32_t ra = team_find(par, a), rb = team_find(par, b);
        if (ra == rb) return;
        if (ra < rb) { const uint32_t t = ra; ra = rb; rb = t; }
        if (atomicCAS(par + ra, ra, rb) == ra) return;
    }
}

template <uint32_t THREADS, bool PIPELINED>
__global__ void __launch_bounds__(THREADS, PIPELINED ? 1 : 1024 / THREADS) k_color_solve_teams(TeamLaunch a)
{
    // [bodyCap] velocities, [bodyCap] poses, then 2 x [bodyCap] u64 colouring words, overwritten after colouring by
    // the constraint records (team_smem_bytes).
    extern __shared__ float4 teamCache[];
    __shared__ uint32_t colorCount[COLOR_SLOTS];
    __shared__ uint32_t colorStart[MAX_COLORS + 1];
    __shared__ uint32_t item;
    const DeviceWorld& w = a.w;
    Manifold* m = a.m;
    uint32_t* prio = const_cast<uint32_t*>(a.s.prio);
    while (true) {
        if (threadIdx.x == 0) item = atomicAdd(a.nextTeam, 1u);
        __syncthreads();
        const uint32_t k = item;
        __syncthreads();
        if (k >= a.teams) return;
        const uint32_t t = a.teamOrder[k];
        const uint32_t w0 = a.teamWorld[t], w1 = a.teamWorld[t + 1];
        const uint32_t lo = a.manSeg[w0], hi = a.manSeg[w1];
        if (hi <= lo) continue;
        for (uint32_t i = lo + threadIdx.x; i < hi; i += THREADS)
            prio[i] = priority_hash(i - a.manSeg[w.bodyWorld[w.cbody[m[i].a]]]);
        const SolveScratch ls{a.s.color + lo, a.s.order + lo, a.s.bodyMax, a.s.bodyMask, colorCount, colorStart,
                              a.s.cons + lo, prio + lo, a.s.listA + lo, a.s.listB + lo, a.s.pairBodies + lo,
                              a.s.hint ? a.s.hint + lo : nullptr};
        const uint32_t b0 = w.worldBodyStart[w0], nb = w.worldBodyStart[w1] - b0;
        if (nb <= a.bodyCap) {
            float4* vel = teamCache;
            float4* pos = teamCache + a.bodyCap;
            // No records on chip: the colouring words sit where the body cache goes and the bodies are loaded after
            // colouring (SharedBodies, lazy). Otherwise the bodies are loaded now and the words follow them.
            const bool lazy = a.consCap == 0;
            auto* maxW = reinterpret_cast<unsigned long long*>(lazy ? teamCache : teamCache + 2 * a.bodyCap);
            unsigned long long* maskW = maxW + a.bodyCap;
            for (uint32_t i = threadIdx.x; i < nb; i += THREADS) {
                if (!lazy) {
                    vel[i] = w.bvel[b0 + i];
                    pos[i] = w.bpos[b0 + i];
                }
                maxW[i] = 0ull;
                maskW[i] = 0ull;
            }
            __syncthreads();
            ConsSmem cs;
            cs.q = teamCache + 2 * a.bodyCap;
            cs.cap = a.consCap;
            cs.base = b0;
            SharedBodies sb{vel, pos, maxW, maskW, b0};
            if (lazy) { sb.count = nb; sb.gvel = w.bvel; sb.gpos = w.bpos; }
            const bool solved = color_and_solve<BlockSync, SharedBodies, PIPELINED>(
                w, sb, m + lo, hi - lo, ls, a.velIters, a.posIters, threadIdx.x, THREADS, BlockSync{},
                &a.counters->colors, &a.counters->status, cs);
            __syncthreads();
            // A team that gave up (its status bit is set and the step is redone or fails) leaves the bodies alone:
            // a lazy cache may still hold colouring words.
            if (solved) {
                for (uint32_t i = threadIdx.x; i < nb; i += THREADS) {
                    w.bvel[b0 + i] = vel[i];
                    w.bpos[b0 + i] = pos[i];
                }
            }
            if (solved && a.ufParent) {
                // The team's islands, in the shared memory the body cache used: links between two dynamic bodies.
                __syncthreads();
                uint32_t* par = reinterpret_cast<uint32_t*>(teamCache);
                for (uint32_t i = threadIdx.x; i < nb; i += THREADS) par[i] = i;
                __syncthreads();
                const uint2* pb = a.s.pairBodies + lo;
                for (uint32_t j = threadIdx.x; j < hi - lo; j += THREADS) {
                    const uint2 q = pb[j];
                    if ((q.x & PAIR_DYNAMIC) && (q.y & PAIR_DYNAMIC))
                        team_union(par, (q.x & PAIR_BODY) - b0, (q.y & PAIR_BODY) - b0);
                }
                __syncthreads();
                for (uint32_t i = threadIdx.x; i < nb; i += THREADS) a.ufParent[b0 + i] = b0 + team_find(par, i);
            }
        } else {
            __syncthreads();
            const bool solved = color_and_solve<BlockSync, GlobalBodies, PIPELINED>(
                w, GlobalBodies{w.bvel, w.bpos, a.s.bodyMax, a.s.bodyMask}, m + lo, hi - lo, ls, a.velIters,
                a.posIters, threadIdx.x, THREADS, BlockSync{}, &a.counters->colors, &a.counters->status);
            if (solved && a.ufParent) {
                __syncthreads();
                const uint2* pb = a.s.pairBodies + lo;
                for (uint32_t j = threadIdx.x; j < hi - lo; j += THREADS) {
                    const uint2 q = pb[j];
                    if ((q.x & PAIR_DYNAMIC) && (q.y & PAIR_DYNAMIC))
                        team_union(a.ufParent, q.x & PAIR_BODY, q.y & PAIR_BODY);
                }
            }
        }
        __syncthreads();
    }
}

template <uint32_t THREADS, bool PIPELINED>
static cudaError_t team_occupancy(uint32_t bodyCap, uint32_t consCap, int* out)
{
    cudaError_t e = cudaFuncSetAttribute(k_color_solve_teams<THREADS, PIPELINED>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(TEAM_SMEM_MAX));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, k_color_solve_teams<THREADS, PIPELINED>, THREADS,
                                                         team_smem_bytes(bodyCap, consCap));
}

cudaError_t team_solver_blocks_per_sm(uint32_t threads, bool pipelined, uint32_t bodyCap, uint32_t consCap, int* out)
{
    switch (threads) {
    case 64: return pipelined ? team_occupancy<64, true>(bodyCap, consCap, out) : team_occupancy<64, false>(bodyCap, consCap, out);
    case 128: return pipelined ? team_occupancy<128, true>(bodyCap, consCap, out) : team_occupancy<128, false>(bodyCap, consCap, out);
    case 256: return pipelined ? team_occupancy<256, true>(bodyCap, consCap, out) : team_occupancy<256, false>(bodyCap, consCap, out);
    case 512: return pipelined ? team_occupancy<512, true>(bodyCap, consCap, out) : team_occupancy<512, false>(bodyCap, consCap, out);
    default: return cudaErrorInvalidValue;
    }
}

template <uint32_t THREADS>
static void launch_teams(bool pipelined, uint32_t grid, size_t smem, cudaStream_t stream, const TeamLaunch& a)
{
    if (pipelined) k_color_solve_teams<THREADS, true><<<grid, THREADS, smem, stream>>>(a);
    else k_color_solve_teams<THREADS, false><<<grid, THREADS, smem, stream>>>(a);
}

cudaError_t launch_color_solve_teams(uint32_t threads, bool pipelined, uint32_t grid, cudaStream_t stream,
                                     const TeamLaunch& a)
{
    const size_t smem = team_smem_bytes(a.bodyCap, a.consCap);
    if (smem > TEAM_SMEM_MAX) return cudaErrorInvalidValue;
    switch (threads) {
    case 64: launch_teams<64>(pipelined, grid, smem, stream, a); break;
    case 128: launch_teams<128>(pipelined, grid, smem, stream, a); break;
    case 256: launch_teams<256>(pipelined, grid, smem, stream, a); break;
    case 512: launch_teams<512>(pipelined, grid, smem, stream, a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
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

// The active body constraints' links (Simulation.cpp:338-341: islandManager.step over each system's active edges).
__global__ void k_island_union_edges(DeviceWorld w, const uint2* __restrict__ edges, uint32_t n,
                                     uint32_t* __restrict__ parent)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t a = edges[i].x, b = edges[i].y;
        if (w.bstate[a] != STATE_DYNAMIC || w.bstate[b] != STATE_DYNAMIC) continue;
        for (uint32_t tries = 0; tries < 1u << 20; tries++) {
            uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
            if (ra == rb) break;
            if (ra < rb) { const uint32_t t = ra; ra = rb; rb = t; }
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
            if (w.worldDirty) w.worldDirty[w.bodyWorld[b]] = 1u;
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
        const uint8_t st = bstate[cbody[c]];
        colDyn[c] = st == STATE_DYNAMIC;
        colOther[c] = st == STATE_STATIC || st == STATE_SLEEPING;   // destroyed bodies' colliders: neither
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Spatial query (BroadPhaseCollisionDetector::queryCollidersInShape, BroadPhaseCollisionDetector.h:189-203;
// BvhTree::queryCollidersInShape, BvhTree.h:110-192): a collider is found when its body's tree (dynamic, static
// or sleeping) is selected and its AABB passes the query shape's leaf test (QueryShapes.h): strict overlap for an
// AABB (AABBQuery::simdOverlap), closest-point squared distance within the squared radius for a circle
// (CircleQuery::simdOverlap, radius clamped at 0). One flag per collider, compacted afterwards in index order.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_query_shape(const float4* __restrict__ caabb, const uint32_t* __restrict__ cbody,
                              const uint8_t* __restrict__ bstate, uint32_t n, uint32_t shape, float4 q,
                              uint32_t trees, uint32_t* __restrict__ flag)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint8_t st = bstate[cbody[c]];
        const uint32_t tree = st == STATE_DYNAMIC ? 1u : (st == STATE_STATIC ? 2u : (st == STATE_SLEEPING ? 4u : 0u));
        bool hit = false;
        if (trees & tree) {
            const float4 b = caabb[c];
            if (shape == 0) {
                hit = b.x < q.z && b.z > q.x && b.y < q.w && b.w > q.y;
            } else {
                const float r = rfmaxf(0.0f, q.z);
                const float rr = r * r;
                const float dx = rfmaxf(b.x - q.x, rfmaxf(0.0f, q.x - b.z));
                const float dy = rfmaxf(b.y - q.y, rfmaxf(0.0f, q.y - b.w));
                hit = (dx * dx + dy * dy) <= rr;
            }
        }
        flag[c] = hit ? 1u : 0u;
    }
}

// Signed distance from a query circle's centre to one collider, as NarrowPhaseCollisionDetector::
// findCollisionsInCircle (NarrowPhaseCollisionDetector.cpp:153-270) computes it: circle - centre distance minus the
// radius; box - the exact box distance field in the box frame; polygon - distance to the support edge's closest
// point (findSupportEdge / closestPointOnSegment, HelperMethods.h:73-109), or the (negative) separation inside.
// False where the reference skips the collider or the distance is not below the query radius.
__device__ __forceinline__ bool circle_contact(const ColliderView& B, V2 pos, float radius, float& sdf)
{
    if (B.type == SHAPE_CIRCLE) {
        const V2 delta = B.pos - pos;
        const float distSq = dot(delta, delta);
        const float radiusSum = B.r + radius;
        if (radiusSum <= 0.0f || distSq >= radiusSum * radiusSum) return false;
        sdf = sqrtf(distSq) - B.r;
    } else {
        const V2 right = V2{B.c, B.s}, up = V2{-B.s, B.c};
        const V2 d = pos - B.pos;
        const V2 loc = V2{dot(d, right), dot(d, up)};
        if (B.type == SHAPE_CAPSULE) {
            // Closest point of the core to the query centre (NarrowPhaseCollisionDetector.cpp:245-262).
            const V2 axis = V2{B.c, B.s};
            const float t = clamp_value(dot(d, axis), -B.hw, B.hw);
            const V2 delta = d - axis * t;
            const float distSquared = dot(delta, delta);
            const float radiusSum = B.r + radius;
            if (radiusSum <= 0.0f || distSquared >= radiusSum * radiusSum) return false;
            sdf = sqrtf(distSquared) - B.r;
        } else if (B.type == SHAPE_BOX) {
            const float dx = fabsf(loc.x) - B.hw, dy = fabsf(loc.y) - B.hh;
            const float maxD = rfmaxf(dx, dy);
            if (maxD > 0.0f && maxD >= radius) return false;
            const float ex = rfmaxf(0.0f, dx), ey = rfmaxf(0.0f, dy);
            const float outside = sqrtf(ex * ex + ey * ey);
            const float inside = rfminf(0.0f, maxD);
            sdf = inside + outside;
        } else {
            float maxSep = -FLT_MAX;
            uint32_t edge = 0;
            for (uint32_t i = 0; i < B.nv; i++) {
                const float sep = dot(ld2(B.normals, i), loc - ld2(B.verts, i));
                if (sep > radius) return false;
                if (sep > maxSep) { maxSep = sep; edge = i; }
            }
            if (maxSep >= ZERO_DIVISION_BOUNDARY) {
                const V2 a = ld2(B.verts, edge), b = ld2(B.verts, next_index(edge, B.nv));
                const V2 ab = b - a;
                const float denom = dot(ab, ab);
                V2 q = a;
                if (denom >= ZERO_DIVISION_BOUNDARY_SQUARED) {
                    const float t = dot(loc - a, ab) / denom;
                    q = a + ab * rfminf(rfmaxf(t, 0.0f), 1.0f);
                }
                const V2 e = loc - q;
                sdf = sqrtf(dot(e, e));
            } else {
                sdf = maxSep;
            }
        }
    }
    return sdf < radius;
}

// Circle contacts: the circle query's colliders (k_query_shape's circle test, radius clamped at 0) that the circle
// itself touches (circle_contact, the radius as given), with their signed distances.
__global__ void k_circle_contacts(DeviceWorld w, float x, float y, float radius, uint32_t trees,
                                  uint32_t* __restrict__ flag, float* __restrict__ dist)
{
    const float r = rfmaxf(0.0f, radius);
    const float rr = r * r;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < w.nColliders; c += gridDim.x * blockDim.x) {
        const uint8_t st = w.bstate[w.cbody[c]];
        const uint32_t tree = st == STATE_DYNAMIC ? 1u : (st == STATE_STATIC ? 2u : (st == STATE_SLEEPING ? 4u : 0u));
        bool hit = false;
        float sdf = 0.0f;
        if (trees & tree) {
            const float4 b = w.caabb[c];
            const float dx = rfmaxf(b.x - x, rfmaxf(0.0f, x - b.z));
            const float dy = rfmaxf(b.y - y, rfmaxf(0.0f, y - b.w));
            if ((dx * dx + dy * dy) <= rr) hit = circle_contact(collider_view(w, c), V2{x, y}, radius, sdf);
        }
        flag[c] = hit ? 1u : 0u;
        dist[c] = sdf;
    }
}

__global__ void k_scatter_contacts(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ offset,
                                   const float* __restrict__ dist, uint32_t n, uint32_t* __restrict__ list,
                                   float* __restrict__ listDist)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) { list[offset[i]] = i; listDist[offset[i]] = dist[i]; }
}

__global__ void k_scatter_list(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ offset, uint32_t n,
                               uint32_t* __restrict__ list)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) list[offset[i]] = i;
}

}  // namespace ag2d
