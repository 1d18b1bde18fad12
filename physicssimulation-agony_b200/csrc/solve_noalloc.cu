// Allocation-free colour + solve over caller-owned device arrays (ag2d_solve_noalloc, include/ag2d.h).
//
// The scratch the solver needs (constraint records, colours, solving order, uncoloured lists, per-body colouring
// words) lives in one file-scope __device__ array of fixed size, so a call makes no device allocation. The array's
// address belongs to a CUDA context, not to a device ordinal: it is looked up with cudaGetSymbolAddress on the first
// call made in each context (the first call on a device, and again after a cudaDeviceReset or under another context
// made current on that device) and cached under the context's process-unique id; later calls in that context only
// launch. The kernel clears the per-body colouring words it relies on at the start of every call, so nothing in the
// array has to start at zero. Two calls that overlap on one device share the array and race: callers serialise them
// (one stream, or an event between streams).
#include "ag2d.h"
#include "ag2d_solver.cuh"

#include <cuda.h>   // driver API types only; the two context queries are reached through cudaGetDriverEntryPoint

#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>

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

// Scratch address per CUDA context, keyed by the context's id (cuCtxGetId: unique for the life of the process, so a
// context created after a reset never finds the address of the one it replaced, even at the same CUcontext value).
std::mutex g_scratchMutex;
std::unordered_map<unsigned long long, unsigned char*> g_scratchByContext;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context; 0 when no context is current or the driver cannot say (the caller
// then looks the address up without caching it).
unsigned long long current_context_id()
{
    static CtxGetCurrentFn getCurrent = nullptr;
    static CtxGetIdFn getId = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getCurrent = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getId = reinterpret_cast<CtxGetIdFn>(p);
    });
    if (!getCurrent || !getId) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (getCurrent(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (getId(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

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
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return fail(AG2D_ERR_NO_DEVICE, "no current CUDA device");
    // An error left by the caller's earlier work is reported as such and left in place for the caller, so that the
    // launch check below only ever sees this call's own launch.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        return fail(AG2D_ERR_CUDA, std::string("a CUDA error from earlier work is pending (not cleared): ") +
                                       cudaGetErrorString(pending));
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratchMutex);
        const unsigned long long ctx = current_context_id();
        const auto hit = ctx ? g_scratchByContext.find(ctx) : g_scratchByContext.end();
        if (hit != g_scratchByContext.end()) {
            scratch = hit->second;
        } else {
            // Set-up for this context: the device address of the static array as this context maps it.
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_solveScratch);
            if (e != cudaSuccess)
                return fail(AG2D_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            scratch = static_cast<unsigned char*>(p);
            // The lookup may have made the device's primary context current: key by the context now current.
            const unsigned long long now = current_context_id();
            if (now) g_scratchByContext[now] = scratch;
        }
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
