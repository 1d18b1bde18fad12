// Manifolds of sleeping islands kept on the device (NarrowPhaseCollisionDetector::sleepContactData /
// wakeContactData, CollisionDetection/Narrow/NarrowPhaseCollisionDetector.cpp:299-414; called from
// Simulation.cpp:350, 460, 578-585).
//
// The store is one array of manifold records with the island (its root body index) of each, grouped by world in a
// batch and, within a world, in the order the records went to sleep. Two operations per step:
//
//  - restore, after the wake pass and before the solver: the records of the islands that woke this step (and whose
//    colliders still exist) join the step's manifold list whole, in store order, at the end of their world's
//    segment, so the solver and the islands see them this step. The reference first lets a manifold generated this
//    frame for the same pair take the stored impulses (wakeContactData, :371-395); that never happens here: a
//    stored record's two bodies are in its sleeping island or static until the island wakes, and the pairs of a
//    frame are found from colliders that were awake when the broad phase ran, before the wake pass. Each pair is
//    stored at most once (it leaves the warm-start list when it is stored and the store when its island wakes), so
//    the reference's first-record-of-a-pair rule has nothing to choose either.
//  - sleep, after a step in which islands woke or fell asleep: the store drops the records of the woken islands and
//    of destroyed colliders; the step's manifolds with a body that is now asleep move to the store (tagged with that
//    body's island: body A's when A sleeps, else body B's), the rest stay as the next step's warm-start source.
//
// All compactions are stable (flag, exclusive scan, scatter), so the orders are deterministic and a world in a
// batch keeps exactly the records, in the same order, it has when stepped alone.
#include "ag2d_kernels.cuh"

namespace ag2d {

__device__ __forceinline__ bool collider_alive(const DeviceWorld& w, uint32_t c)
{
    return w.bstate[w.cbody[c]] != STATE_DESTROYED;
}

__device__ __forceinline__ uint32_t record_world(const DeviceWorld& w, const Manifold& m)
{
    return w.bodyWorld ? w.bodyWorld[w.cbody[m.a]] : 0u;
}

// First index in sorted[0, n) whose value is >= v (strictly greater when 'upper').
__device__ __forceinline__ uint32_t bound_search(const uint32_t* sorted, uint32_t n, uint32_t v, bool upper)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t x = sorted[mid];
        if (x < v || (upper && x == v)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Restore, step 1: flag[r] = 1 for the store records of woken islands with live colliders.
__global__ void k_isle_stage_flags(DeviceWorld w, const Manifold* __restrict__ isle,
                                   const uint32_t* __restrict__ isleId, const uint32_t* __restrict__ nIsle,
                                   const uint32_t* __restrict__ wakeIsland, uint32_t* __restrict__ flag)
{
    const uint32_t n = *nIsle;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t id = isleId[r];
        const Manifold& m = isle[r];
        flag[r] = (id < w.nBodies && wakeIsland[id] && collider_alive(w, m.a) && collider_alive(w, m.b)) ? 1u : 0u;
    }
}

// Restore, step 2: the staged records (store indices) in store order, with their worlds.
__global__ void k_isle_stage_list(DeviceWorld w, const Manifold* __restrict__ isle, const uint32_t* __restrict__ nIsle,
                                  const uint32_t* __restrict__ flag, const uint32_t* __restrict__ off,
                                  uint32_t* __restrict__ list, uint32_t* __restrict__ listWorld)
{
    const uint32_t n = *nIsle;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        if (!flag[r]) continue;
        list[off[r]] = r;
        listWorld[off[r]] = record_world(w, isle[r]);
    }
}

// Restore, step 3 (a single world): the staged records go after the fresh manifolds, with no colouring hint. A
// list that would pass 'cap' records the overflow instead (the step is retried with larger buffers).
__global__ void k_isle_append(Manifold* __restrict__ cur, const uint32_t* __restrict__ nCur, uint32_t cap,
                              uint32_t* __restrict__ hint, const Manifold* __restrict__ isle,
                              const uint32_t* __restrict__ list, const uint32_t* __restrict__ nList,
                              uint32_t* __restrict__ status)
{
    const uint32_t base = *nCur, n = *nList;
    if (uint64_t(base) + n > cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicOr(status, STATUS_MANIFOLD_OVERFLOW);
        return;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        cur[base + j] = isle[list[j]];
        if (hint) hint[base + j] = NO_COLOR;
    }
}

// Restore, step 3 (a batch): fresh manifolds and staged records merged by world into out (the fresh ones of a
// world first, in their order, then its staged ones in store order). seg: the fresh list's world starts. The
// caller makes out the step's list whatever happens, so every record of out[0, nCur) is written.
__global__ void k_isle_merge(DeviceWorld w, const Manifold* __restrict__ cur, const uint32_t* __restrict__ hint,
                             const uint32_t* __restrict__ nCur, const uint32_t* __restrict__ seg,
                             const Manifold* __restrict__ isle, const uint32_t* __restrict__ list,
                             const uint32_t* __restrict__ listWorld, const uint32_t* __restrict__ nList, uint32_t cap,
                             Manifold* __restrict__ out, uint32_t* __restrict__ outHint, uint32_t* __restrict__ status)
{
    const uint32_t nf = *nCur;
    uint32_t nu = *nList;
    if (uint64_t(nf) + nu > cap) {
        // Overflow: the fresh list is copied as it is (the step is retried with larger buffers), so that the
        // kernels after this one still read valid records.
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, STATUS_MANIFOLD_OVERFLOW);
        nu = 0;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf + nu; i += gridDim.x * blockDim.x) {
        if (i < nf) {
            const Manifold m = cur[i];
            const uint32_t pos = i + (nu ? bound_search(listWorld, nu, record_world(w, m), false) : 0u);
            out[pos] = m;
            if (outHint) outHint[pos] = hint ? hint[i] : NO_COLOR;
        } else {
            const uint32_t j = i - nf;
            const uint32_t pos = seg[listWorld[j] + 1] + j;
            out[pos] = isle[list[j]];
            if (outHint) outHint[pos] = NO_COLOR;
        }
    }
}

// Restore, step 4: the list's count takes the appended records (unless the append overflowed).
__global__ void k_isle_count(uint32_t* __restrict__ nCur, const uint32_t* __restrict__ nStage,
                             const uint32_t* __restrict__ nList, uint32_t cap, StepCounters* counters)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const uint32_t n = *nList;
    if (n && uint64_t(*nCur) + n <= cap) {
        *nCur += n;
        counters->manifolds += n;
    }
    counters->restored = n;
    counters->staged = *nStage;
}

// Sleep, step 1: the store records that stay (island still asleep, and, when 'checkAlive', colliders alive).
__global__ void k_isle_keep_flags(DeviceWorld w, const Manifold* __restrict__ isle,
                                  const uint32_t* __restrict__ isleId, const uint32_t* __restrict__ nIsle,
                                  const uint32_t* __restrict__ wakeIsland, uint32_t checkAlive,
                                  uint32_t* __restrict__ keep)
{
    const uint32_t n = *nIsle;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t id = isleId[r];
        const bool woke = id < w.nBodies && wakeIsland[id];
        bool k = !woke;
        if (k && checkAlive) k = collider_alive(w, isle[r].a) && collider_alive(w, isle[r].b);
        keep[r] = k ? 1u : 0u;
    }
}

// Sleep, step 2: each manifold of the step either stays (both bodies awake or static), moves to the store (a body
// asleep: the island of body A when A sleeps, else of body B) or is dropped (a destroyed collider).
__global__ void k_isle_move_flags(DeviceWorld w, const Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                                  uint32_t* __restrict__ stay, uint32_t* __restrict__ move,
                                  uint32_t* __restrict__ moveIsland)
{
    const uint32_t n = *nM;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Manifold& r = m[i];
        const uint32_t bA = w.cbody[r.a], bB = w.cbody[r.b];
        const uint8_t sA = w.bstate[bA], sB = w.bstate[bB];
        uint32_t s = 0, mv = 0, island = 0xFFFFFFFFu;
        if (sA != STATE_DESTROYED && sB != STATE_DESTROYED) {
            if (sA == STATE_SLEEPING) island = w.sleepIsland[bA];
            else if (sB == STATE_SLEEPING) island = w.sleepIsland[bB];
            mv = island != 0xFFFFFFFFu ? 1u : 0u;
            s = 1u - mv;
        }
        stay[i] = s;
        move[i] = mv;
        moveIsland[i] = island;
    }
}

// Sleep, step 3 (a batch): the worlds of the kept store records and of the moving manifolds (move null: none),
// compacted.
__global__ void k_isle_sleep_worlds(DeviceWorld w, const Manifold* __restrict__ isle,
                                    const uint32_t* __restrict__ nIsle, const uint32_t* __restrict__ keep,
                                    const uint32_t* __restrict__ keepOff, const Manifold* __restrict__ m,
                                    const uint32_t* __restrict__ nM, const uint32_t* __restrict__ move,
                                    const uint32_t* __restrict__ moveOff, uint32_t* __restrict__ keepWorld,
                                    uint32_t* __restrict__ moveWorld)
{
    const uint32_t ni = *nIsle, nm = move ? *nM : 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ni + nm; i += gridDim.x * blockDim.x) {
        if (i < ni) {
            if (keep[i]) keepWorld[keepOff[i]] = record_world(w, isle[i]);
        } else {
            const uint32_t k = i - ni;
            if (move[k]) moveWorld[moveOff[k]] = record_world(w, m[k]);
        }
    }
}

// Sleep, step 4: the new store (per world: kept records in store order, then the moving manifolds in list order).
// keepWorld / moveWorld are null for a single world (one segment: kept, then moved); move null: nothing moves.
__global__ void k_isle_store_scatter(DeviceWorld w, const Manifold* __restrict__ isle,
                                     const uint32_t* __restrict__ isleId, const uint32_t* __restrict__ nIsle,
                                     const uint32_t* __restrict__ keep, const uint32_t* __restrict__ keepOff,
                                     const uint32_t* __restrict__ nKeep, const Manifold* __restrict__ m,
                                     const uint32_t* __restrict__ nM, const uint32_t* __restrict__ move,
                                     const uint32_t* __restrict__ moveOff, const uint32_t* __restrict__ nMove,
                                     const uint32_t* __restrict__ moveIsland, const uint32_t* __restrict__ keepWorld,
                                     const uint32_t* __restrict__ moveWorld, Manifold* __restrict__ isleOut,
                                     uint32_t* __restrict__ isleIdOut)
{
    const uint32_t ni = *nIsle, nm = move ? *nM : 0u, nk = *nKeep, nmv = move ? *nMove : 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ni + nm; i += gridDim.x * blockDim.x) {
        if (i < ni) {
            if (!keep[i]) continue;
            const uint32_t k = keepOff[i];
            const uint32_t pos = k + (moveWorld && nmv ? bound_search(moveWorld, nmv, keepWorld[k], false) : 0u);
            isleOut[pos] = isle[i];
            isleIdOut[pos] = isleId[i];
        } else {
            const uint32_t q = i - ni;
            if (!move[q]) continue;
            const uint32_t k = moveOff[q];
            const uint32_t pos = k + (keepWorld ? bound_search(keepWorld, nk, moveWorld[k], true) : nk);
            isleOut[pos] = m[q];
            isleIdOut[pos] = moveIsland[q];
        }
    }
}

// Sleep, step 5: the store's new count.
__global__ void k_isle_store_count(const uint32_t* __restrict__ nKeep, const uint32_t* __restrict__ nMove,
                                   uint32_t* __restrict__ nIsle)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *nIsle = *nKeep + *nMove;
}

// Sleep, a single world that only gains records: the moving manifolds after the current store, in list order.
__global__ void k_isle_append_moved(const Manifold* __restrict__ m, const uint32_t* __restrict__ nM,
                                    const uint32_t* __restrict__ move, const uint32_t* __restrict__ moveOff,
                                    const uint32_t* __restrict__ moveIsland, const uint32_t* __restrict__ nIsle,
                                    Manifold* __restrict__ isle, uint32_t* __restrict__ isleId)
{
    const uint32_t n = *nM, base = *nIsle;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!move[i]) continue;
        isle[base + moveOff[i]] = m[i];
        isleId[base + moveOff[i]] = moveIsland[i];
    }
}

__global__ void k_isle_add_count(uint32_t* __restrict__ nIsle, const uint32_t* __restrict__ nMove)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *nIsle += *nMove;
}

// The warm-start list without the records moved to the store (and those of destroyed colliders), with colours.
__global__ void k_isle_list_scatter(const Manifold* __restrict__ m, const uint32_t* __restrict__ color,
                                    const uint32_t* __restrict__ nM, const uint32_t* __restrict__ stay,
                                    const uint32_t* __restrict__ stayOff, Manifold* __restrict__ out,
                                    uint32_t* __restrict__ colorOut)
{
    const uint32_t n = *nM;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!stay[i]) continue;
        out[stayOff[i]] = m[i];
        colorOut[stayOff[i]] = color[i];
    }
}

}  // namespace ag2d
