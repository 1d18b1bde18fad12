// Kernel declarations and launch constants for the collision/contact pipeline.
#pragma once

#include "ag2d_math.cuh"
#include "ag2d_world.cuh"

namespace ag2d {

constexpr uint32_t SORT_THREADS = 256;
constexpr uint32_t SORT_ITEMS = 16;
constexpr uint32_t SORT_TILE = SORT_THREADS * SORT_ITEMS;   // keys per onesweep tile
constexpr uint32_t SCAN_THREADS = 256;
constexpr uint32_t SCAN_ITEMS = 8;
constexpr uint32_t SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr int QUERY_STACK = 64;
constexpr uint32_t QUERY_STASH = 8;   // pairs a query keeps from its counting traversal
constexpr uint32_t MAX_COLORS = 256;
constexpr uint32_t NO_COLOR = 0xFFFFFFFFu;

// Traversal record of an internal node: both children's AABBs, their child codes (internal node index, or ~leaf)
// and the last leaf of each child's range, so that a traversal step is one 48-byte load.
struct alignas(16) NodeRec {
    float4 box[2];
    int2 child;
    int2 last;
};
static_assert(sizeof(NodeRec) == 48, "NodeRec is 48 bytes");

// Read-only view of one LBVH over n leaves in sorted order. A single tree has n - 1 internal nodes and root 0; a
// world-segmented tree (sortedWorld non-null) holds one tree per world segment [segStart[w], segStart[w + 1]),
// rooted at internal node segStart[w].
struct TreeView {
    int n;
    const int2* child;
    const int2* range;
    const float4* nodeAabb;
    const float4* leafAabb;       // AABBs in sorted (leaf) order
    const uint32_t* vals;         // collider index of each leaf
    const uint32_t* sortedWorld;  // world of each leaf, or null (one world)
    const uint32_t* segStart;     // [worlds + 1] segment starts, or null (one world)
    const NodeRec* rec;           // traversal records of the internal nodes
};

// Spatial kernels (k_spatial.cu).
__global__ void k_integrate(DeviceWorld w, const uint32_t* dynBody, const uint8_t* dynSimd, uint32_t nDyn, float dt,
                            float gx, float gy, float dampHalf, uint32_t phase);
__global__ void k_collider_pose(DeviceWorld w, const uint32_t* list, const uint8_t* listSimd, uint32_t n,
                                const uint32_t* worldMask);
__global__ void k_bounds_init(uint32_t* bounds, uint32_t worlds);
__global__ void k_bounds(const float4* aabb, const uint32_t* list, uint32_t n, const uint32_t* colWorld,
                         uint32_t* bounds);
__global__ void k_count_world(const uint32_t* list, uint32_t n, const uint32_t* elemWorld, uint32_t* counts);
__global__ void k_simd_flags(const uint32_t* list, uint32_t n, const uint32_t* offsets, uint32_t nElems,
                             const uint32_t* elemWorld, const uint32_t* worldStart, uint32_t worlds, uint8_t* simd);
__global__ void k_morton(const float4* aabb, const uint32_t* list, uint32_t n, const uint32_t* colWorld,
                         const uint32_t* bounds, uint32_t* keys, uint32_t* vals, uint32_t* keyOf);
__global__ void k_world_keys(const uint32_t* vals, uint32_t n, const uint32_t* colWorld, uint32_t* keys);
__global__ void k_seg_starts(const uint32_t* offsets, const uint32_t* worldStart, uint32_t worlds, uint32_t nElems,
                             const uint32_t* total, uint32_t* segStart);
__global__ void k_manifold_segments(const Manifold* m, const uint32_t* nM, const uint32_t* cbody,
                                    const uint32_t* bodyWorld, uint32_t worlds, uint32_t* segStart);
__global__ void k_tree_gather(const uint32_t* vals, uint32_t n, const uint32_t* keyOf, const uint32_t* colWorld,
                              const float4* caabb, uint32_t* sortedKey, uint32_t* sortedWorld, float4* leafAabb);
__global__ void k_sort_histogram(const uint32_t* keys, uint32_t n, uint32_t* hist);
__global__ void k_sort_digit_scan(uint32_t* hist);
__global__ void k_sort_pass(const uint32_t* keysIn, const uint32_t* valsIn, uint32_t* keysOut, uint32_t* valsOut,
                            uint32_t n, uint32_t shift, const uint32_t* digitBase, uint32_t* tileState,
                            uint32_t* tileCounter, uint32_t* status);
// Segments up to SEGMENT_SORT_MAX keys are sorted in shared memory (k_segment_sort), in two size classes.
constexpr uint32_t SEGMENT_SORT_SMALL = 2048;
constexpr uint32_t SEGMENT_SORT_MAX = 16384;
__global__ void k_segment_sort(const uint32_t* keysIn, const uint32_t* valsIn, uint32_t* keysOut, uint32_t* valsOut,
                               const uint32_t* segStart, uint32_t worlds, uint32_t minSize, uint32_t maxSize);
__global__ void k_lbvh_build(const uint32_t* keys, const uint32_t* sortedWorld, const uint32_t* segStart, int n,
                             int2* child, int2* range, int* parent, int* leafParent, float4* meet, NodeRec* rec);
__global__ void k_lbvh_refit(int n, const int2* child, const int* parent, const int* leafParent,
                             const float4* leafAabb, float4* nodeAabb, float4* meet, NodeRec* rec);
// Empty marker of a refit meeting slot (min x bits): a NaN no arithmetic produces.
constexpr uint32_t MEET_EMPTY = 0xFFFFFFFFu;
// Pair query: every candidate pair of the dynamic colliders, in query-rank order, into pairs; *total = the count.
// tileState [tiles + 1] and tileCounter zeroed before the launch (tiles: blockDim.x queries each).
constexpr uint32_t QUERY_MAX_THREADS = 256;
__global__ void k_query(TreeView dyn, TreeView other, const uint32_t* cbody, uint2* pairs, uint32_t pairCap,
                        uint32_t* total, uint32_t* status, uint32_t* tileState, uint32_t* tileCounter);
__global__ void k_ccd_sweep(DeviceWorld w, const uint32_t* dynCol, uint32_t n, TreeView other, const float4* prevPos,
                            const float4* prevPose, const float* minExtent, uint32_t* hitTime, uint32_t* status);
__global__ void k_ccd_shift_colliders(DeviceWorld w, const uint32_t* dynCol, uint32_t n, const float4* prevPos,
                                      const uint32_t* hitTime);
__global__ void k_ccd_shift_bodies(DeviceWorld w, const uint32_t* dynBody, uint32_t n, const float4* prevPos,
                                   uint32_t* hitTime, StepCounters* counters);
// Decoupled look-back over tiles taken in ticket order: tile t publishes flag << 30 | value in tileState[t] (flag 1:
// its aggregate, 2: its inclusive prefix) and sums its predecessors' values, read by the calling warp 32 at a time,
// nearest first, up to the nearest inclusive prefix. A tile only waits on tiles with smaller tickets, all held by
// running blocks, so the waits end; each is still bounded by SPIN_LIMIT (then STATUS_LOOKBACK_TIMEOUT is set and the
// partial sum returned). Called by one full warp; returns the exclusive prefix of tile 'tile' (> 0).
__device__ __forceinline__ uint32_t scan_lookback(uint32_t tile, uint32_t* tileState, uint32_t* status)
{
    const uint32_t lane = threadIdx.x & 31;
    volatile uint32_t* state = tileState;
    uint32_t prefix = 0, spins = 0;
    int32_t t = int32_t(tile) - 1;
    while (t >= 0) {
        const int32_t idx = t - int32_t(lane);
        const uint32_t sv = idx >= 0 ? state[idx] : (2u << 30);
        const uint32_t flag = sv >> 30;
        const uint32_t inc = __ballot_sync(0xffffffffu, flag == 2u);
        const uint32_t window = inc ? (((inc & (0u - inc)) << 1) - 1u) : 0xffffffffu;   // lanes up to the nearest
        if (__ballot_sync(0xffffffffu, flag == 0u) & window) {                             // inclusive prefix
            if (++spins > SPIN_LIMIT) {
                if (lane == 0) atomicOr(status, STATUS_LOOKBACK_TIMEOUT);
                break;
            }
            continue;
        }
        uint32_t v = ((window >> lane) & 1u) ? (sv & 0x3FFFFFFFu) : 0u;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        prefix += v;
        if (inc) break;
        t -= 32;
    }
    return prefix;
}

// Contact-cache key of an unordered collider pair, and its home slot in a power-of-two open-addressing table.
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

// Exclusive scan of in[0, min(n, *nDev)) into out (nDev may be null), total = the sum (may be null).
__global__ void k_scan(const uint32_t* in, uint32_t* out, uint32_t n, const uint32_t* nDev, uint32_t* total,
                       uint32_t* tileState, uint32_t* tileCounter, uint32_t* status);

// Contact kernels (k_contact.cu).
// Per thread: a 64-byte manifold slot, a hit flag and its share of its group's vertex tiles (100 bytes).
constexpr uint32_t NARROW_SMEM_PER_THREAD =
    uint32_t(sizeof(Manifold) + sizeof(uint32_t) + 2 * MAX_POLYGON_VERTICES * sizeof(V2) / NARROW_GROUP);
// Narrow phase + manifold compaction: manifolds of the hit pairs, in pair order, into out; tileState [tiles + 1] and
// tileCounter zeroed before the launch (tiles: blockDim.x pairs each).
__global__ void k_narrow(DeviceWorld w, const uint2* pairs, const uint32_t* nPairs, uint32_t pairCap, Manifold* out,
                         uint32_t manifoldCap, uint32_t* nOut, StepCounters* counters, uint32_t* tileState,
                         uint32_t* tileCounter);
__global__ void k_warm_insert(const Manifold* prev, const uint32_t* nPrev, unsigned long long* keys,
                              uint32_t* vals, uint32_t capacity, const uint32_t* seg, const uint32_t* colWorld,
                              uint32_t* status);
constexpr uint32_t WARM_CACHED = 0x80000000u;   // contact-cache value flag: the manifold had a non-zero impulse
__global__ void k_warm_lookup(const Manifold* prev, Manifold* cur, const uint32_t* nCur,
                              const unsigned long long* keys, const uint32_t* vals, uint32_t capacity,
                              const uint32_t* seg, const uint32_t* colWorld, StepCounters* counters,
                              const uint32_t* prevColor, uint32_t* hint);
__global__ void k_wake(DeviceWorld w, const Manifold* m, const uint32_t* nM, uint32_t* wakeIsland,
                       StepCounters* counters);
__global__ void k_wake_apply(DeviceWorld w, const uint32_t* wakeIsland, StepCounters* counters);
__global__ void k_island_init(DeviceWorld w, uint32_t* parent, uint32_t* flag);
__global__ void k_island_union(DeviceWorld w, const Manifold* m, const uint32_t* nM, uint32_t* parent);
__global__ void k_island_quiet(DeviceWorld w, uint32_t* parent, uint32_t* flag, float dt, float speedThreshold,
                               float timeThreshold);
__global__ void k_island_sleep(DeviceWorld w, uint32_t* parent, const uint32_t* flag, StepCounters* counters);
__global__ void k_state_flags(const uint8_t* bstate, const uint32_t* cbody, uint32_t nBodies, uint32_t nColliders,
                              uint32_t* bodyDyn, uint32_t* colDyn, uint32_t* colOther);
__global__ void k_scatter_list(const uint32_t* flag, const uint32_t* offset, uint32_t n, uint32_t* list);

// Sleeping-island manifold store (k_islands.cu): restore at wake, move at sleep.
__global__ void k_isle_stage_flags(DeviceWorld w, const Manifold* isle, const uint32_t* isleId, const uint32_t* nIsle,
                                   const uint32_t* wakeIsland, uint32_t* flag);
__global__ void k_isle_stage_list(DeviceWorld w, const Manifold* isle, const uint32_t* nIsle, const uint32_t* flag,
                                  const uint32_t* off, uint32_t* list, uint32_t* listWorld);
__global__ void k_isle_append(Manifold* cur, const uint32_t* nCur, uint32_t cap, uint32_t* hint, const Manifold* isle,
                              const uint32_t* list, const uint32_t* nList, uint32_t* status);
__global__ void k_isle_merge(DeviceWorld w, const Manifold* cur, const uint32_t* hint, const uint32_t* nCur,
                             const uint32_t* seg, const Manifold* isle, const uint32_t* list,
                             const uint32_t* listWorld, const uint32_t* nList, uint32_t cap, Manifold* out,
                             uint32_t* outHint, uint32_t* status);
__global__ void k_isle_count(uint32_t* nCur, const uint32_t* nStage, const uint32_t* nList, uint32_t cap,
                             StepCounters* counters);
__global__ void k_isle_keep_flags(DeviceWorld w, const Manifold* isle, const uint32_t* isleId, const uint32_t* nIsle,
                                  const uint32_t* wakeIsland, uint32_t checkAlive, uint32_t* keep);
__global__ void k_isle_move_flags(DeviceWorld w, const Manifold* m, const uint32_t* nM, uint32_t* stay,
                                  uint32_t* move, uint32_t* moveIsland);
__global__ void k_isle_sleep_worlds(DeviceWorld w, const Manifold* isle, const uint32_t* nIsle, const uint32_t* keep,
                                    const uint32_t* keepOff, const Manifold* m, const uint32_t* nM,
                                    const uint32_t* move, const uint32_t* moveOff, uint32_t* keepWorld,
                                    uint32_t* moveWorld);
__global__ void k_isle_store_scatter(DeviceWorld w, const Manifold* isle, const uint32_t* isleId,
                                     const uint32_t* nIsle, const uint32_t* keep, const uint32_t* keepOff,
                                     const uint32_t* nKeep, const Manifold* m, const uint32_t* nM,
                                     const uint32_t* move, const uint32_t* moveOff, const uint32_t* nMove,
                                     const uint32_t* moveIsland, const uint32_t* keepWorld, const uint32_t* moveWorld,
                                     Manifold* isleOut, uint32_t* isleIdOut);
__global__ void k_isle_store_count(const uint32_t* nKeep, const uint32_t* nMove, uint32_t* nIsle);
__global__ void k_isle_append_moved(const Manifold* m, const uint32_t* nM, const uint32_t* move,
                                    const uint32_t* moveOff, const uint32_t* moveIsland, const uint32_t* nIsle,
                                    Manifold* isle, uint32_t* isleId);
__global__ void k_isle_add_count(uint32_t* nIsle, const uint32_t* nMove);
__global__ void k_isle_list_scatter(const Manifold* m, const uint32_t* color, const uint32_t* nM,
                                    const uint32_t* stay, const uint32_t* stayOff, Manifold* out,
                                    uint32_t* colorOut);
__global__ void k_query_shape(const float4* caabb, const uint32_t* cbody, const uint8_t* bstate, uint32_t n,
                              uint32_t shape, float4 q, uint32_t trees, uint32_t* flag);
__global__ void k_circle_contacts(DeviceWorld w, float x, float y, float radius, uint32_t trees, uint32_t* flag,
                                  float* dist);
__global__ void k_scatter_contacts(const uint32_t* flag, const uint32_t* offset, const float* dist, uint32_t n,
                                   uint32_t* list, float* listDist);

// Body constraints (k_joints.cu): springs (kind 0), revolute (1), prismatic (2) and slider (3) joints and motors
// (4), the reference's ConstraintType order, each kind's active
// constraints in rec[k] grouped by level (level l: [levelStart[k][l], levelStart[k][l + 1])), solver data in
// data[k], the motors' accumulated impulses by dense index in motorImpulse. One CTA of JOINT_THREADS threads.
constexpr uint32_t JOINT_KINDS_DEVICE = 5;
constexpr uint32_t JOINT_THREADS = 1024;
struct JointLaunch {
    const JointRec* rec[JOINT_KINDS_DEVICE];
    JointData* data[JOINT_KINDS_DEVICE];
    const uint32_t* levelStart[JOINT_KINDS_DEVICE];
    uint32_t count[JOINT_KINDS_DEVICE];
    uint32_t levels[JOINT_KINDS_DEVICE];
    uint32_t iterations[JOINT_KINDS_DEVICE];
    uint32_t maxIterations;
    float dt;
    float* motorImpulse;
};
__global__ void k_joints(DeviceWorld w, JointLaunch L);
// Island links of the active constraints' body pairs (edges[i] = {a, b}), as k_island_union links manifolds.
__global__ void k_island_union_edges(DeviceWorld w, const uint2* edges, uint32_t n, uint32_t* parent);

// Collision events (k_events.cu): the events of the manifolds in man[0, min(*nMan, manCap)) whose colliders opted
// in (cev), appended to ring (counters->events counts them all; STATUS_EVENT_OVERFLOW when more than ringCap).
// Launched with a multiple of 32 threads a block, before the solver changes the velocities.
__global__ void k_collision_events(DeviceWorld w, const ColliderEvent* cev, const Manifold* man,
                                   const uint32_t* nMan, uint32_t manCap, EventRecord* ring, uint32_t ringCap,
                                   StepCounters* counters);

// Batch repacking (k_repack.cu). A segment copies 'count' elements from [src, ...) of the current array (fromNew
// 0), or from the staged section of joining world 'src' (fromNew 1), to [dst, ...) of the new array; the deltas
// shift the indices stored in the elements (new start - source start of that kind of element in the segment's
// world; a staged world's indices start at 0).
struct GatherSeg {
    uint32_t dst, src, count, fromNew;
    int32_t dBody, dCol, dCircle, dBox, dPoly, dVert, dMat, pad;
};
enum GatherMode : uint32_t {
    GATHER_PLAIN = 0, GATHER_ISLAND, GATHER_BODY, GATHER_SHAPE, GATHER_MATERIAL, GATHER_VERTEX
};
template <class T>
cudaError_t launch_gather(T* dst, const T* srcOld, const T* srcNew, const GatherSeg* segs, uint32_t nsegs,
                          uint32_t total, uint32_t mode, uint32_t grid, cudaStream_t stream,
                          const unsigned long long* sections, uint32_t nsec, uint32_t section);
__global__ void k_world_of(const uint32_t* starts, uint32_t worlds, uint32_t n, uint32_t* out);
__global__ void k_fill_u32(uint32_t* out, uint32_t n, uint32_t value);
// Host reads: how k_extract packs a field (EXTRACT_DIRECT fields are copied as they lie).
enum ExtractKind : uint32_t {
    EXTRACT_DIRECT = 0, EXTRACT_F4_COMP, EXTRACT_F4_XYZ, EXTRACT_F2_COMP, EXTRACT_U8_U32, EXTRACT_ISLAND
};
__global__ void k_extract(const void* src, uint32_t lo, uint32_t n, uint32_t kind, uint32_t comp, uint32_t bias,
                          void* out);

}  // namespace ag2d
