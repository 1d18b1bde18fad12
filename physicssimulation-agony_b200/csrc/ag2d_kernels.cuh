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
constexpr uint32_t MAX_COLORS = 256;
constexpr uint32_t NO_COLOR = 0xFFFFFFFFu;

// Read-only view of one LBVH (n leaves; n - 1 internal nodes, root 0).
struct TreeView {
    int n;
    const int2* child;
    const int2* range;
    const float4* nodeAabb;
    const float4* leafAabb;   // AABBs in sorted (leaf) order
    const uint32_t* vals;     // collider index of each leaf
};

// Spatial kernels (k_spatial.cu).
__global__ void k_integrate(DeviceWorld w, const uint32_t* dynBody, uint32_t nDyn, float dt, float gx, float gy,
                            float dampHalf);
__global__ void k_collider_pose(DeviceWorld w, const uint32_t* list, uint32_t n);
__global__ void k_bounds_init(uint32_t* bounds);
__global__ void k_bounds(const float4* aabb, const uint32_t* list, uint32_t n, uint32_t* bounds);
__global__ void k_morton(const float4* aabb, const uint32_t* list, uint32_t n, const uint32_t* bounds,
                         uint32_t* keys, uint32_t* vals);
__global__ void k_sort_histogram(const uint32_t* keys, uint32_t n, uint32_t* hist);
__global__ void k_sort_digit_scan(uint32_t* hist);
__global__ void k_sort_pass(const uint32_t* keysIn, const uint32_t* valsIn, uint32_t* keysOut, uint32_t* valsOut,
                            uint32_t n, uint32_t shift, const uint32_t* digitBase, uint32_t* tileState,
                            uint32_t* tileCounter, uint32_t* status);
__global__ void k_lbvh_build(const uint32_t* keys, const uint32_t* vals, int n, const float4* caabb, int2* child,
                             int2* range, int* parent, int* leafParent, float4* leafAabb, uint32_t* visit);
__global__ void k_lbvh_refit(int n, const int2* child, const int* parent, const int* leafParent,
                             const float4* leafAabb, float4* nodeAabb, uint32_t* visit);
__global__ void k_query_count(TreeView dyn, TreeView other, const uint32_t* cbody, uint32_t* counts,
                              uint32_t* status);
__global__ void k_query_write(TreeView dyn, TreeView other, const uint32_t* cbody, const uint32_t* offsets,
                              uint2* pairs, uint32_t pairCap, uint32_t* status);
__global__ void k_scan_blocks(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* blockSums);
__global__ void k_scan_add(uint32_t* out, uint32_t n, const uint32_t* blockOffsets);
__global__ void k_scan_total(const uint32_t* in, const uint32_t* out, uint32_t n, uint32_t* total);

// Contact kernels (k_contact.cu).
__global__ void k_narrow(DeviceWorld w, const uint2* pairs, const uint32_t* nPairs, uint32_t pairCap,
                         Manifold* slots, uint32_t* hit);
__global__ void k_compact_manifolds(const Manifold* slots, const uint32_t* hit, const uint32_t* offsets,
                                    const uint32_t* nPairs, uint32_t pairCap, Manifold* out, uint32_t manifoldCap,
                                    uint32_t* nOut, StepCounters* counters);
__global__ void k_warm_insert(const Manifold* prev, const uint32_t* nPrev, unsigned long long* keys,
                              uint32_t* vals, uint32_t capacity, uint32_t* status);
__global__ void k_warm_lookup(const Manifold* prev, Manifold* cur, const uint32_t* nCur,
                              const unsigned long long* keys, const uint32_t* vals, uint32_t capacity,
                              StepCounters* counters);
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

}  // namespace ag2d
