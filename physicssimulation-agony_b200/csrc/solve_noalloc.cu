// Allocation-free colour + solve over caller-owned device arrays (ag2d_solve_noalloc, include/ag2d.h).
//
// The scratch the solver needs (constraint records, colours, solving order, uncoloured lists, per-body colouring
// words) lives in one file-scope __device__ array of fixed size, so a call makes no device allocation. The array's
// address is looked up once per device with cudaGetSymbolAddress, on the first call made with that device current;
// later calls only launch. The kernel clears the per-body colouring words it relies on at the start of every call,
// so nothing in the array has to start at zero. Two calls that overlap on one device share the array and race:
// callers serialise them (one stream, or an event between streams).
#include "ag2d.h"
#include "ag2d_solver.cuh"

#include <cstdint>
#include <mutex>
#include <string>

namespace ag2d {

constexpr uint32_t NOALLOC_MAX_MANIFOLDS = AG2D_SOLVE_NOALLOC_MAX_MANIFOLDS;
constexpr uint32_t NOALLOC_MAX_BODIES = AG2D_SOLVE_NOALLOC_MAX_BODIES;
constexpr uint32_t NOALLOC_THREADS = 512;

// Scratch layout (byte offsets; every part 256-byte aligned).
constexpr size_t NA_CONS = 0;                                                         // Constraint[M]
constexpr size_t NA_COLOR = NA_CONS + size_t(NOALLOC_MAX_MANIFOLDS) * sizeof(Constraint);   // u32[M]
constexpr size_t NA_ORDER = NA_COLOR + size_t(NOALLOC_MAX_MANIFOLDS) * 4;            // u32[M]
constexpr size_t NA_LIST_A = NA_ORDER + size_t(NOALLOC_MAX_MANIFOLDS) * 4;           // uint4[M]
constexpr size_t NA_LIST_B = NA_LIST_A + size_t(NOALLOC_MAX_MANIFOLDS) * 16;         // uint4[M]
constexpr size_t NA_BODY_MAX = NA_LIST_B + size_t(NOALLOC_MAX_MANIFOLDS) * 16;       // u64[B]
constexpr size_t NA_BODY_MASK = NA_BODY_MAX + size_t(NOALLOC_MAX_BODIES) * 8;        // u64[B]
constexpr size_t NA_PAIRS = NA_BODY_MASK + size_t(NOALLOC_MAX_BODIES) * 8;           // uint2[M]
constexpr size_t NA_BYTES = NA_PAIRS + size_t(NOALLOC_MAX_MANIFOLDS) * 8;             // 3.1 MiB
static_assert(NA_COLOR % 256 == 0 && NA_BODY_MAX % 256 == 0 && NA_BODY_MASK % 256 == 0 && NA_PAIRS % 256 == 0,
              "256-byte parts");
static_assert(sizeof(ag2d_manifold) == sizeof(Manifold), "ag2d_manifold is the device Manifold record");

static __device__ __align__(256) unsigned char g_solveScratch[NA_BYTES];

// One CTA colours and solves the n manifolds with the routine every solver variant shares (color_and_solve), on
// global body state. Writes {status bits, colours} to statusOut when given.
__global__ void __launch_bounds__(NOALLOC_THREADS, 1)
k_color_solve_static(DeviceWorld w, Manifold* m, uint32_t n, unsigned char* scratch, uint32_t velIters,
                     uint32_t posIters, uint32_t* statusOut)
{
    __shared__ uint32_t colorCount[COLOR_SLOTS];
    __shared__ uint32_t colorStart[MAX_COLORS + 1];
    __shared__ uint32_t colors, status;
    auto* bodyMax = reinterpret_cast<unsigned long long*>(scratch + NA_BODY_MAX);
    auto* bodyMask = reinterpret_cast<unsigned long long*>(scratch + NA_BODY_MASK);
    for (uint32_t i = threadIdx.x; i < w.nBodies; i += blockDim.x) {
        bodyMax[i] = 0ull;
        bodyMask[i] = 0ull;
    }
    if (threadIdx.x == 0) {
        colors = 0;
        status = 0;
    }
    __syncthreads();
    const SolveScratch s{reinterpret_cast<uint32_t*>(scratch + NA_COLOR), reinterpret_cast<uint32_t*>(scratch + NA_ORDER),
                         bodyMax, bodyMask, colorCount, colorStart, reinterpret_cast<Constraint*>(scratch + NA_CONS),
                         nullptr, reinterpret_cast<uint4*>(scratch + NA_LIST_A),
                         reinterpret_cast<uint4*>(scratch + NA_LIST_B), reinterpret_cast<uint2*>(scratch + NA_PAIRS)};
    color_and_solve(w, GlobalBodies{w.bvel, w.bpos, bodyMax, bodyMask}, m, n, s, velIters, posIters, threadIdx.x,
                    blockDim.x, BlockSync{}, &colors, &status);
    __syncthreads();
    if (threadIdx.x == 0 && statusOut) {
        statusOut[0] = status;
        statusOut[1] = colors;
    }
}

}  // namespace ag2d

namespace ag2d {
void set_last_error(const std::string& message);   // the thread's ag2d_last_error_string (capi.cu)
}

namespace {

// Scratch address per device ordinal, filled on the first call with that device current.
constexpr int MAX_DEVICES = 64;
std::mutex g_scratchMutex;
unsigned char* g_scratchPtr[MAX_DEVICES] = {};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int32_t fail(int32_t code, const std::string& msg)
{
    ag2d::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" {

int32_t ag2d_solve_noalloc(const ag2d_solve_view* view, ag2d_manifold* manifolds, uint32_t n_manifolds,
                           uint32_t velocity_iterations, uint32_t position_iterations, void* stream,
                           uint32_t* device_status)
{
    using namespace ag2d;
    if (!view) return fail(AG2D_ERR_INVALID_ARG, "null view");
    if (n_manifolds > NOALLOC_MAX_MANIFOLDS)
        return fail(AG2D_ERR_CAPACITY, "n_manifolds " + std::to_string(n_manifolds) + " exceeds the static scratch limit " +
                                           std::to_string(NOALLOC_MAX_MANIFOLDS));
    if (view->n_bodies > NOALLOC_MAX_BODIES)
        return fail(AG2D_ERR_CAPACITY, "n_bodies " + std::to_string(view->n_bodies) + " exceeds the static scratch limit " +
                                           std::to_string(NOALLOC_MAX_BODIES));
    if (n_manifolds > 0 && (!manifolds || !view->body_velocity || !view->body_pose || !view->collider_body ||
                            !view->collider_material || !view->materials))
        return fail(AG2D_ERR_INVALID_ARG, "null device array");
    if (!aligned16(manifolds) || !aligned16(view->body_velocity) || !aligned16(view->body_pose) ||
        !aligned16(view->materials))
        return fail(AG2D_ERR_INVALID_ARG, "manifold, body and material arrays must be 16-byte aligned");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail(AG2D_ERR_NO_DEVICE, "no current CUDA device");
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratchMutex);
        if (!g_scratchPtr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_solveScratch);
            if (e != cudaSuccess)
                return fail(AG2D_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratchPtr[dev] = static_cast<unsigned char*>(p);
        }
        scratch = g_scratchPtr[dev];
    }
    DeviceWorld w{};
    w.nBodies = view->n_bodies;
    w.nColliders = view->n_colliders;
    w.nMaterials = view->n_materials;
    w.bvel = reinterpret_cast<float4*>(view->body_velocity);
    w.bpos = reinterpret_cast<float4*>(view->body_pose);
    w.cbody = const_cast<uint32_t*>(view->collider_body);
    w.cmat = const_cast<uint32_t*>(view->collider_material);
    w.materials = reinterpret_cast<float4*>(const_cast<float*>(view->materials));
    w.nWorlds = 1;
    k_color_solve_static<<<1, NOALLOC_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        w, reinterpret_cast<Manifold*>(manifolds), n_manifolds, scratch, velocity_iterations, position_iterations,
        device_status);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(AG2D_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return AG2D_OK;
}

}  // extern "C"
