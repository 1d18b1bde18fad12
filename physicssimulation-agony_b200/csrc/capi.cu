// C ABI of libag2d.so (include/ag2d.h): world lifecycle, object creation, the per-step launch sequence, field
// access and phase-level taps. Host code; every kernel it launches is in k_spatial.cu / k_contact.cu.
#include "ag2d.h"
#include "ag2d_solver.cuh"
#include "host_objects.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <stdexcept>
#include <string>
#include <vector>

using namespace ag2d;

namespace {

thread_local std::string g_error;

struct ApiError : std::runtime_error {
    int32_t code;
    ApiError(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(expr)                                                                                              \
    do {                                                                                                      \
        const cudaError_t e_ = (expr);                                                                        \
        if (e_ != cudaSuccess)                                                                                \
            throw ApiError(e_ == cudaErrorMemoryAllocation ? AG2D_ERR_OOM : AG2D_ERR_CUDA,                     \
                           std::string(#expr) + ": " + cudaGetErrorString(e_));                               \
    } while (0)

}  // namespace

namespace ag2d {
// Sets the calling thread's ag2d_last_error_string (for entry points defined in other translation units).
void set_last_error(const std::string& message) { g_error = message; }
}  // namespace ag2d

namespace {

template <class F>
int32_t guarded(F&& f)
{
    try {
        f();
        return AG2D_OK;
    } catch (const ApiError& e) {
        g_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_error = "host allocation failed";
        return AG2D_ERR_OOM;
    } catch (const std::exception& e) {
        g_error = e.what();
        return AG2D_ERR_INVALID_ARG;
    }
}

// Device buffer (re)allocations in this process: a reallocation synchronises the device and fresh memory is slow
// to map, so a steady step should make none (reported by ag2d_world_counters).
static std::atomic<uint64_t> g_deviceAllocs{0};

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // Grows to at least 'count' elements; contents are not preserved. A buffer that grows again takes half as much
    // again on top, so a steadily growing size (a server batch filling up) reallocates a logarithmic number of
    // times: fresh device memory is slow to map.
    void reserve(size_t count)
    {
        if (count <= n && p) return;
        const size_t c = std::max<size_t>(p ? std::max(count, n + n / 2) : count, 1);
        release();
        CK(cudaMalloc(reinterpret_cast<void**>(&p), c * sizeof(T)));
        g_deviceAllocs.fetch_add(1, std::memory_order_relaxed);
        n = c;
    }
    void upload(const T* src, size_t count, cudaStream_t s)
    {
        reserve(count);
        if (count) CK(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

// Page-locked host buffer (grow only): host<->device copies through it are one DMA each, without the driver's
// staging of pageable memory. Freeing synchronises the device, so it only happens when the buffer grows.
struct PinnedBuf {
    uint8_t* p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { if (p) cudaFreeHost(p); }
    void reserve(size_t bytes)
    {
        if (bytes <= n && p) return;
        const size_t c = std::max<size_t>(p ? std::max(bytes, n + n / 2) : bytes, 4096);
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        CK(cudaHostAlloc(reinterpret_cast<void**>(&p), c, cudaHostAllocDefault));
        n = c;
    }
};

template <class T>
void swap_bufs(DBuf<T>& a, DBuf<T>& b)
{
    std::swap(a.p, b.p);
    std::swap(a.n, b.n);
}

inline uint32_t div_up(uint64_t a, uint64_t b) { return uint32_t((a + b - 1) / b); }

// A device array copied into host memory (synchronised on return).
template <class T>
static std::vector<T> download(const T* p, size_t n, cudaStream_t s)
{
    std::vector<T> v(n);
    if (n) CK(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return v;
}

// Single-pass exclusive scans (k_scan): the tile states and the ticket counter, zeroed before each scan, and the
// grid of persistent blocks (set from the SM count when the device is first used).
struct Scanner {
    DBuf<uint32_t> state;          // [tiles + 1]: tile states, then the ticket counter
    uint32_t blocks = 1;
    uint32_t* status = nullptr;    // where a look-back that gave up is recorded
    void reserve(uint32_t n) { state.reserve(size_t(div_up(std::max<uint32_t>(n, 1), SCAN_TILE)) + 1); }
    // Exclusive scan of in[0, n) (n the capacity; nDev, if given, the device-side count within it: elements past it
    // are neither read nor written); total, if given, receives the sum.
    void run(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total, cudaStream_t s,
             const uint32_t* nDev = nullptr)
    {
        const uint32_t tiles = std::max<uint32_t>(div_up(n, SCAN_TILE), 1);
        reserve(n);
        CK(cudaMemsetAsync(state.p, 0, (size_t(tiles) + 1) * sizeof(uint32_t), s));
        k_scan<<<std::min(tiles, blocks), SCAN_THREADS, 0, s>>>(in, out, n, nDev, total, state.p, state.p + tiles,
                                                               status);
        CK(cudaGetLastError());
    }
};

struct Tree {
    DBuf<uint32_t> keys, vals, keys2, vals2;
    DBuf<int2> child, range;
    DBuf<int> parent, leafParent;
    DBuf<float4> leafAabb, nodeAabb;
    DBuf<NodeRec> rec;
    DBuf<float4> meet;   // refit meeting slots, one per internal node
    DBuf<uint32_t> bounds, hist, tileState, tileCounter;
    // World-segmented trees: Morton key per collider, sorted keys / worlds, segment starts (filled with the lists).
    DBuf<uint32_t> keyOf, sortedKey, sortedWorld, segStart;
    uint32_t worlds = 1;
    int n = 0;
    void reserve(uint32_t cap, uint32_t nWorlds)
    {
        worlds = nWorlds;
        keys.reserve(cap); vals.reserve(cap); keys2.reserve(cap); vals2.reserve(cap);
        child.reserve(cap); range.reserve(cap); parent.reserve(cap); leafParent.reserve(cap);
        leafAabb.reserve(cap); nodeAabb.reserve(cap); meet.reserve(cap); rec.reserve(cap);
        bounds.reserve(4 * size_t(nWorlds)); hist.reserve(4 * 256); tileCounter.reserve(4);
        tileState.reserve(size_t(div_up(std::max<uint32_t>(cap, 1), SORT_TILE)) * 256 * 4);
        if (nWorlds > 1) {
            keyOf.reserve(cap); sortedKey.reserve(cap); sortedWorld.reserve(cap); segStart.reserve(nWorlds + 1);
        }
    }
    TreeView view() const
    {
        const bool seg = worlds > 1;
        return TreeView{n, child.p, range.p, nodeAabb.p, leafAabb.p, vals.p, seg ? sortedWorld.p : nullptr,
                        seg ? segStart.p : nullptr, rec.p};
    }
};

struct DeviceInfo {
    int sms = 0;
    int coopSolveBlocks = 0;   // co-resident CTAs of the grid solver
    int solveCluster = 0;      // CTAs per cluster of the cluster solver (16 when the device allows it)
};

// glibc fmin / fmax (the reference's std::fmin / std::fmax on x86-64): the first argument unless the comparison
// fails or the second is NaN.
inline float host_fmin(float a, float b) { return (a < b || b != b) ? a : b; }
inline float host_fmax(float a, float b) { return (a > b || b != b) ? a : b; }
constexpr uint32_t ORDERED_ONE = 0xBF800000u;   // 1.0f in the order-preserving map of float_to_ordered

// Min extent of every collider about its origin (ObjectManager.cpp setColliderExtents calls: circle radius, min box
// half extent, polygon in-radius PhysicsGeometry::calculatePolygonInnerRadius), for continuous collision detection.
inline std::vector<float> min_extents(const std::vector<uint32_t>& cs, const std::vector<float>& cr,
                                      const std::vector<float2>& bh, const std::vector<uint32_t>& po,
                                      const std::vector<uint32_t>& pc, const std::vector<float2>& pv,
                                      const std::vector<float2>& pn)
{
    std::vector<float> me(cs.size());
    for (size_t i = 0; i < cs.size(); i++) {
        const uint32_t type = cs[i] >> 30, si = cs[i] & 0x3FFFFFFFu;
        if (type == SHAPE_CIRCLE) {
            me[i] = cr[si];
        } else if (type == SHAPE_BOX) {
            me[i] = host_fmin(bh[si].x, bh[si].y);
        } else if (type == SHAPE_CAPSULE) {
            me[i] = bh[si].y;   // setColliderExtents(radius, ...) (ObjectManager.cpp:228)
        } else {
            float r = FLT_MAX;
            for (uint32_t k = 0; k < pc[si]; k++) {
                const float2 n = pn[po[si] + k], v = pv[po[si] + k];
                r = host_fmin(r, n.x * v.x + n.y * v.y);
            }
            me[i] = host_fmax(r, 0.0f);
        }
    }
    return me;
}

// Element counts of one resident world, per kind of array (a server engine's worlds are consecutive ranges).
struct WorldExtent {
    uint32_t body = 0, col = 0, circle = 0, box = 0, poly = 0, vert = 0, mat = 0, man = 0, statics = 0;
    uint32_t isle = 0;   // manifolds of sleeping islands
};

// A world waiting to join a server batch: all its arrays in one host blob (sections at 64-byte aligned offsets,
// indices local to the world), copied to the device with one transfer and gathered into place there.
enum StagedSection : uint32_t {
    SEC_VEL, SEC_POS, SEC_ROT, SEC_WRAP, SEC_BOUND, SEC_TIMER, SEC_STATE, SEC_ISLAND,
    SEC_CBODY, SEC_CSHAPE, SEC_CMAT, SEC_COFF, SEC_CPOSE, SEC_CAABB, SEC_CROT, SEC_MINEXT,
    SEC_CIRCLE, SEC_BOXHALF, SEC_POLYOFF, SEC_POLYCOUNT, SEC_POLYVERTS, SEC_POLYNORMALS, SEC_MATS, SEC_PREV,
    SEC_PREVCOLOR, SEC_ISLE, SEC_ISLEID, NSEC
};
struct StagedWorld {
    WorldExtent ext;
    std::vector<uint8_t> blob;
    uint64_t sec[NSEC] = {};
};

// Checkpoint of an engine (ag2d_batch_save / ag2d_batch_restore): a header, then one section per resident array at
// 256-byte aligned offsets, in device layout with batch-global indices. It holds everything a step reads from the
// previous one (body and collider state, collider poses and AABBs, the warm-start manifolds with their colours, the
// world partition), so that a restored engine steps on exactly as the saved one would.
enum CkptSection : uint32_t {
    CK_VEL, CK_POS, CK_ROT, CK_WRAP, CK_BOUND, CK_TIMER, CK_STATE, CK_ISLAND,
    CK_CBODY, CK_CSHAPE, CK_CMAT, CK_COFF, CK_CPOSE, CK_CAABB, CK_CROT, CK_MINEXT,
    CK_CIRCLE, CK_BOXHALF, CK_POLYOFF, CK_POLYCOUNT, CK_POLYVERTS, CK_POLYNORMALS, CK_MATS, CK_PREV,
    CK_PREVCOLOR, CK_WBODY, CK_WCOL, CK_ISLE, CK_ISLEID, NCK
};
constexpr char CKPT_MAGIC[8] = {'A', 'G', '2', 'D', 'C', 'K', 'P', 'T'};
constexpr uint32_t CKPT_VERSION = 3;
struct CkptHeader {
    char magic[8];
    uint32_t version, headerBytes;
    ag2d_world_settings settings;
    uint32_t nWorlds, nBodies, nColliders, nCircles, nBoxes, nPolygons, nPolyVerts, nMaterialRows;
    uint32_t nPrev, nStatic, lastManifolds, nIsle;
    uint32_t lastPairs, pad;   // the saved engine's last step: candidate pairs (sizes the restored buffers)
    uint64_t totalBytes;
    uint64_t off[NCK], len[NCK];
};

// One world's state in the upload format (host arrays), and the warm-start manifolds.
struct PackedArrays {
    std::vector<float4> vel, pos, co, mats;
    std::vector<float2> rot, bh, pv, pn;
    std::vector<float> wc, br, st, cr;
    std::vector<uint8_t> state;
    std::vector<uint32_t> isl, cb, cs, cm, po, pc;
    std::vector<Manifold> prev;
    std::vector<uint32_t> pcol;   // colour of each warm-start manifold (empty: none known)
    std::vector<Manifold> isle;   // manifolds of sleeping islands, and the island (root body) of each
    std::vector<uint32_t> isleId;
    std::vector<float4> cp;   // collider world poses at the end of the last step (empty: never stepped, zeros)

    // Appends another world, shifting its body, collider, shape, vertex and material indices past this one's.
    void append(const PackedArrays& o)
    {
        const uint32_t bo = uint32_t(vel.size()), cof = uint32_t(cb.size()), circ = uint32_t(cr.size());
        const uint32_t box = uint32_t(bh.size()), poly = uint32_t(po.size()), vert = uint32_t(pv.size());
        const uint32_t mat = uint32_t(mats.size());
        auto cat = [](auto& d, const auto& s) { d.insert(d.end(), s.begin(), s.end()); };
        cat(vel, o.vel); cat(pos, o.pos); cat(rot, o.rot); cat(wc, o.wc); cat(br, o.br); cat(st, o.st);
        cat(state, o.state);
        for (uint32_t v : o.isl) isl.push_back(v == 0xFFFFFFFFu ? v : v + bo);
        for (uint32_t v : o.cb) cb.push_back(v + bo);
        for (uint32_t v : o.cs) {
            const uint32_t type = shape_type(v), idx = shape_index(v);
            const uint32_t base = type == SHAPE_CIRCLE ? circ : (type == SHAPE_POLYGON ? poly : box);   // box table:
                                                                                                       // boxes, capsules
            cs.push_back((type << 30) | (idx + base));
        }
        for (uint32_t v : o.cm) cm.push_back(v + mat);
        cat(co, o.co); cat(cr, o.cr); cat(bh, o.bh);
        for (uint32_t v : o.po) po.push_back(v + vert);
        cat(pc, o.pc); cat(pv, o.pv); cat(pn, o.pn); cat(mats, o.mats);
        for (Manifold m : o.prev) { m.a += cof; m.b += cof; prev.push_back(m); }
        if (o.pcol.size() == o.prev.size()) cat(pcol, o.pcol);
        else pcol.insert(pcol.end(), o.prev.size(), NO_COLOR);
        for (Manifold m : o.isle) { m.a += cof; m.b += cof; isle.push_back(m); }
        for (uint32_t v : o.isleId) isleId.push_back(v == 0xFFFFFFFFu ? v : v + bo);
        if (!o.cp.empty() || !cp.empty()) {
            cp.resize(cof, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            if (o.cp.empty()) cp.resize(cof + o.cb.size(), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            else cat(cp, o.cp);
        }
    }
};

// Packs one world's arrays into its staging blob. Collider poses come from the world's last step (zeros for a
// never-stepped world, as when uploaded alone); AABBs and wrapped rotations are recomputed by the joining world's
// first full pose pass.
StagedWorld stage_world(const PackedArrays& a)
{
    StagedWorld w;
    WorldExtent& e = w.ext;
    e.body = uint32_t(a.vel.size());
    e.col = uint32_t(a.cb.size());
    e.circle = uint32_t(a.cr.size());
    e.box = uint32_t(a.bh.size());
    e.poly = uint32_t(a.po.size());
    e.vert = uint32_t(a.pv.size());
    e.mat = uint32_t(a.mats.size());
    e.man = uint32_t(a.prev.size());
    e.isle = uint32_t(a.isle.size());
    e.statics = uint32_t(std::count(a.state.begin(), a.state.end(), uint8_t(STATE_STATIC)));
    const std::vector<float> me = min_extents(a.cs, a.cr, a.bh, a.po, a.pc, a.pv, a.pn);
    const size_t sizes[NSEC] = {
        e.body * sizeof(float4), e.body * sizeof(float4), e.body * sizeof(float2), e.body * 4, e.body * 4,
        e.body * 4, e.body, e.body * 4,
        e.col * 4, e.col * 4, e.col * 4, e.col * sizeof(float4), e.col * sizeof(float4), e.col * sizeof(float4),
        e.col * 4, e.col * 4,
        e.circle * 4, e.box * sizeof(float2), e.poly * 4, e.poly * 4, e.vert * sizeof(float2), e.vert * sizeof(float2),
        e.mat * sizeof(float4), e.man * sizeof(Manifold), e.man * 4, e.isle * sizeof(Manifold), e.isle * 4};
    uint64_t off = 0;
    for (uint32_t k = 0; k < NSEC; k++) {
        w.sec[k] = off;
        off += (sizes[k] + 63) & ~uint64_t(63);
    }
    w.blob.assign(off, 0);   // zero sections: collider AABBs and wrapped rotations, poses of a never-stepped world
    auto put = [&](uint32_t k, const void* src) {
        if (sizes[k]) std::memcpy(w.blob.data() + w.sec[k], src, sizes[k]);
    };
    put(SEC_VEL, a.vel.data()); put(SEC_POS, a.pos.data()); put(SEC_ROT, a.rot.data()); put(SEC_WRAP, a.wc.data());
    put(SEC_BOUND, a.br.data()); put(SEC_TIMER, a.st.data()); put(SEC_STATE, a.state.data());
    put(SEC_ISLAND, a.isl.data());
    put(SEC_CBODY, a.cb.data()); put(SEC_CSHAPE, a.cs.data()); put(SEC_CMAT, a.cm.data()); put(SEC_COFF, a.co.data());
    if (a.cp.size() == e.col) put(SEC_CPOSE, a.cp.data());
    put(SEC_MINEXT, me.data());
    put(SEC_CIRCLE, a.cr.data()); put(SEC_BOXHALF, a.bh.data()); put(SEC_POLYOFF, a.po.data());
    put(SEC_POLYCOUNT, a.pc.data()); put(SEC_POLYVERTS, a.pv.data()); put(SEC_POLYNORMALS, a.pn.data());
    put(SEC_MATS, a.mats.data()); put(SEC_PREV, a.prev.data());
    if (a.pcol.size() == e.man) put(SEC_PREVCOLOR, a.pcol.data());
    else if (e.man) std::memset(w.blob.data() + w.sec[SEC_PREVCOLOR], 0xFF, sizes[SEC_PREVCOLOR]);   // NO_COLOR
    put(SEC_ISLE, a.isle.data());
    put(SEC_ISLEID, a.isleId.data());
    return w;
}

// Candidate pairs (and manifolds) reserved per collider up front. A settled pile of convex bodies has about two
// candidate pairs per collider; growing later synchronises the device and can take long on first touch of memory.
constexpr uint32_t INITIAL_PAIRS_PER_COLLIDER = 8;

// Manifold count above which the solver runs on the whole grid instead of one cluster.
constexpr uint32_t GRID_SOLVE_THRESHOLD = 600000;

}  // namespace

// Launch limits of the solver kernels on a device (queried once per device and process).
static DeviceInfo probe_device(int device)
{
    static std::mutex mu;
    static std::map<int, DeviceInfo> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(device);
    if (it != cache.end()) return it->second;
    DeviceInfo dev;
    CK(cudaDeviceGetAttribute(&dev.sms, cudaDevAttrMultiProcessorCount, device));
    int perSm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_color_solve_grid, 256, 0));
    dev.coopSolveBlocks = std::max(1, perSm) * dev.sms;
    // Largest cluster (16 non-portable, else 8, 4, 2) that can be resident.
    dev.solveCluster = 1;
    if (cudaFuncSetAttribute(k_color_solve_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
        cudaSuccess) {
        for (int cl : {16, 8, 4, 2}) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cl);
            cfg.blockDim = dim3(SOLVE_CLUSTER_THREADS);
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cl;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, k_color_solve_cluster, &cfg) == cudaSuccess &&
                clusters >= 1) {
                dev.solveCluster = cl;
                break;
            }
        }
    }
    cudaGetLastError();
    // The narrow phase stages polygons in dynamic shared memory: up to 512 threads x NARROW_SMEM_PER_THREAD.
    CK(cudaFuncSetAttribute(k_narrow, cudaFuncAttributeMaxDynamicSharedMemorySize, int(512 * NARROW_SMEM_PER_THREAD)));
    // AG2D_SOLVER=grid forces the whole-grid solver (test hook for that variant).
    if (const char* v = std::getenv("AG2D_SOLVER")) {
        if (std::string(v) == "grid") dev.solveCluster = 1;
    }
    cache[device] = dev;
    return dev;
}

// ConstraintSystemBase::normalizeAxis (ConstraintSystemBase.h:144-152): false for a (near) zero-length axis.
static bool normalize_axis(float& x, float& y)
{
    const float lenSq = x * x + y * y;
    if (!(lenSq > 1e-12f)) return false;
    const float len = std::sqrt(lenSq);
    x = x / len;
    y = y / len;
    return true;
}

// PrismaticJointConstraintSystem::computeReferenceAngle (PrismaticJointConstraintSystem.h:118-125).
static float reference_angle(float rotA, float rotB)
{
    const float pi = 3.14159265358979323846f, twoPi = 2.0f * pi;
    float a = rotB - rotA;
    a -= twoPi * std::floor((a + pi) / twoPi);
    return a;
}

// A deferred body command (ObjectManager::ObjectCommand, SimulationImpl/ObjectManager.h:45): queued by destroy and the
// setters in call order, applied at the start of the next step (Simulation::update -> flushCommands,
// Simulation.cpp:39; ObjectManager::applyCommand, ObjectManager.cpp:662-790). Stale handles are dropped.
struct BodyCommand {
    int32_t kind;   // AG2D_COMMAND_*
    uint64_t handle;
    float a, b;
    uint32_t slot = 0;   // AG2D_COMMAND_POLYGON_SHAPE: the outline's index in pendingPolygons
};

struct ag2d_world {
    ag2d_world_settings settings{};
    cudaStream_t stream = nullptr;
    DeviceInfo dev;
    HostObjects objects;
    bool hostDirty = true;          // host objects changed since the last upload
    bool listsDirty = true;         // work lists need a rebuild (state changes)
    bool fullPose = true;           // next pose pass covers every collider (first step after an upload)
    bool aabbValid = false;         // caabb holds the broad phase's AABBs (a step ran, or a state brought them)
    bool otherDirty = true;         // static + sleeping tree must be rebuilt
    uint64_t stepsTaken = 0;
    std::vector<BodyCommand> commands;   // queued body commands, applied by flushCommands
    std::vector<std::vector<float>> pendingPolygons;   // prepared outlines the queued polygon commands name

    // Collision callbacks (SimulationImpl/CollisionCallbackManager.h): slot 0 is the permanent "no callback",
    // destroyed slots are reused last-in first-out.
    struct CallbackEntry {
        ag2d_collision_callback fn = nullptr;
        void* user = nullptr;
    };
    std::vector<CallbackEntry> callbacks = std::vector<CallbackEntry>(1);
    std::vector<uint8_t> callbackAlive = std::vector<uint8_t>(1, 1);
    std::vector<uint16_t> callbackFree;
    uint32_t callbacksAlive = 0;          // excluding slot 0
    bool eventsEnabled = true;            // SimulationSettings::collisionEventsEnabled
    std::vector<ColliderEvent> loadedOptIn;   // colliders' opt-ins of a world made by load_state (no host colliders)
    bool optInDirty = true;               // cevent needs an upload
    uint32_t optInColliders = 0;          // colliders with a callback, as last uploaded
    bool recording = false;               // this step records events
    bool dispatching = false;             // callbacks are running (a callback may not step the world)
    uint32_t eventCap = 0;
    std::vector<ag2d_collision_event> lastEvents;   // the last step's events, in dispatch order

    // Body constraints: device lists rebuilt from the host tables (objects.jointSystems) when these change or
    // bodies change state; deferred destroys and setters (ConstraintSystemBase::flushImpl) applied with the body
    // commands.
    struct JointCommand {
        int32_t kind, field;   // field < 0: destroy
        uint64_t handle;
        float a, b;
    };
    std::vector<JointCommand> jointCommands;
    uint32_t jointActive[JOINT_KINDS] = {}, jointLevels[JOINT_KINDS] = {};
    std::vector<uint32_t> jointLevelHost[JOINT_KINDS];
    uint32_t nJointEdges = 0, motorsOnDevice = 0;
    bool jointsDirty = false;   // the device lists need a rebuild before the next step

    uint32_t nBodies = 0, nColliders = 0, nDynBody = 0, nDynCol = 0, nOther = 0, nStatic = 0;
    uint32_t nDestroyed = 0;   // bodies removed by destroy commands (still in the arrays, in no list)
    uint32_t pairCap = 0, manifoldCap = 0, hashCap = 0;
    uint32_t lastManifolds = 0;
    uint32_t lastPairs = 0;   // candidate pairs of the last step
    uint32_t prevCount = 0;   // manifolds in prevManifolds (the warm-start source), as the host knows them

    // Bodies.
    DBuf<float4> bvel, bpos;
    DBuf<float2> brot;
    DBuf<float> wrapCount, boundRadius, sleepTimer;
    DBuf<uint8_t> bstate;
    DBuf<uint32_t> sleepIsland;
    // Body constraints on the device: each kind's active constraints in level order, their solver data and level
    // starts, the motors' accumulated impulses by dense index, the active pairs' bodies for the islands.
    DBuf<JointRec> jointRec[JOINT_KINDS];
    DBuf<JointData> jointData[JOINT_KINDS];
    DBuf<uint32_t> jointLevel[JOINT_KINDS];
    DBuf<float> motorImpulse, snapMotorImpulse;
    DBuf<uint2> jointEdges;
    // Collision events: per-collider opt-in and the step's event ring.
    DBuf<ColliderEvent> cevent;
    DBuf<EventRecord> eventRing;
    // Snapshot of the mutable body state (restored when a step overflows a buffer).
    DBuf<float4> snapVel, snapPos;
    DBuf<float2> snapRot;
    DBuf<float> snapWrap, snapTimer;
    DBuf<uint8_t> snapState;
    DBuf<uint32_t> snapIsland;
    // Colliders and shapes.
    DBuf<uint32_t> cbody, cshape, cmat;
    DBuf<float4> coff, cpose, caabb;
    DBuf<float> cworldRot;
    DBuf<float> minExtent;      // continuous collision: min extent per collider
    DBuf<float4> prevPose;      // continuous collision: collider world poses before integration
    DBuf<uint32_t> ccdHit;      // continuous collision: earliest time of impact per body (ordered float, 1 = none)
    DBuf<float> circleRadius;
    DBuf<float2> boxHalf, polyVerts, polyNormals;
    DBuf<uint32_t> polyOffset, polyCount;
    DBuf<float4> materials;
    // Work lists.
    DBuf<uint32_t> dynBody, dynCol, otherCol, flagA, flagB, flagC, offA, offB, offC, listCounts;
    // Trees and pairs.
    Tree dynTree, otherTree;
    DBuf<uint32_t> queryState;   // pair-query tile states ([dynamic colliders / 64 + 1]) and ticket counter
    DBuf<uint2> pairs;
    // Manifolds.
    DBuf<Manifold> manifolds, prevManifolds;
    DBuf<uint32_t> nManifolds, nPrev;
    DBuf<uint32_t> narrowState;   // narrow-phase tile states ([pairCap / 64 + 1]) and ticket counter
    DBuf<unsigned long long> hashKeys;
    DBuf<uint32_t> hashVals;
    // Colouring and solver.
    DBuf<uint32_t> color, colorCount, colorStart, order, bar, prio;
    // Colour of each warm-start manifold (NO_COLOR: unknown), swapped with 'color' after each step; the warm-start
    // lookup turns it into this step's colouring hints (written into 'color').
    DBuf<uint32_t> prevColor;
    bool hintsReady = false;   // this step's lookup wrote the hints
    DBuf<uint4> listA, listB;
    DBuf<unsigned long long> bodyMax, bodyMask;
    // Manifolds of sleeping islands (k_islands.cu): world-grouped records and the island (root body) of each, with
    // the back buffers the sleep pass scatters into. isleUpper bounds the count as the host knows it (0: empty).
    DBuf<Manifold> isle, bk_isle;
    DBuf<uint32_t> isleId, bk_isleId, nIsle;
    uint32_t isleUpper = 0;
    // Restore scratch: staging flags and offsets, the staged records and their worlds, and counts [staged, -, kept,
    // moved, staying].
    DBuf<uint32_t> isleFlag, isleOff, isleList, isleListWorld, isleCounts;
    // Batches: the step's list with the restored records merged in by world (swapped in as 'manifolds' / 'color').
    DBuf<Manifold> mergeMan;
    DBuf<uint32_t> mergeHint;
    // Sleep pass scratch over the step's list: stay / move flags and offsets, the island of each moving manifold, the
    // worlds of the kept and moving records, and the compacted list with its colours.
    DBuf<uint32_t> sleepStay, sleepMove, sleepStayOff, sleepMoveOff, sleepMoveIsland, sleepKeepWorld,
        sleepMoveWorld, sleepColor;
    DBuf<Manifold> sleepList;
    bool prevHoldsSleepers = false;   // the warm-start list still holds records moved to the store (compactPrev)
    bool islandsLinked = false;       // this step's team solver already linked the islands (phaseIslands skips it)
    DBuf<Constraint> cons;
    DBuf<uint2> pairBodies;
    // Islands.
    DBuf<uint32_t> ufParent, ufFlag, wakeIsland;
    // World partition of a batch (nWorlds == 1: a single world, none of these is used).
    uint32_t nWorlds = 1;
    uint32_t teamColliders = 1024;         // solver team size: consecutive worlds packed up to this many colliders
    uint32_t teamThreads = 256;            // CTA size of the team solver
    uint32_t teamBodyCap = 2048;           // bodies of a team staged in shared memory (larger teams use global)
    uint32_t teamConsCap = 0;              // constraint records a team keeps in shared memory (more: global)
    uint32_t maxWorldCols = 0;             // colliders of the largest world of a batch (segmented-sort class)
    bool segSortReady = false;
    uint32_t bigConsCap = 0;
    bool consOnChip = false;               // team constraint records in shared memory when they fit (tunable)
    uint32_t nTeams = 0;
    uint32_t teamBlocks = 1;               // co-resident CTAs of the team solver at this shared-memory size
    uint32_t nBigTeams = 0, bigBodyCap = 0, bigBlocks = 1;   // worlds larger than a team, one CTA each
    uint32_t bigThreads = BIG_TEAM_THREADS;                   // their CTA size (tunable: 256 or 512)
    bool bigPipelined = false;                                 // their passes pipelined (tunable)
    cudaStream_t sideStream = nullptr;     // the big-world solver runs here, beside the small-team solver
    cudaEvent_t forkEvent = nullptr, joinEvent = nullptr;
    uint32_t queryThreads = 256;           // block sizes of the pair query and the narrow phase (tunable)
    uint32_t narrowThreads = 256;
    std::vector<uint32_t> hBodyStart, hColStart;     // [nWorlds + 1]
    DBuf<uint32_t> bodyWorld, colWorld, worldBodyStart, worldColStart, manSeg, nextWorld, worldDirty;
    DBuf<uint32_t> isleSeg;                  // world starts of the sleeping islands' manifolds (server repacks)
    DBuf<uint32_t> prevSeg;                  // world starts of the warm-start list (warm-start table regions)
    bool prevSegValid = false;               // prevSeg describes prevManifolds as it is
    DBuf<uint32_t> teamWorld, teamOrder;     // solver teams: first world of each team; small then big, largest first
    DBuf<uint8_t> dynSimd, dynColSimd;               // SIMD-path flag of each work-list entry
    // Request-server engines: extents of the resident worlds, back buffers the repack gathers into, and the
    // staging upload of joining worlds.
    std::vector<WorldExtent> worldExt;
    bool manSegFresh = false;   // a batched step ran since the last repack (per-world manifold extents changed)
    DBuf<float4> bk_bvel, bk_bpos, bk_coff, bk_cpose, bk_caabb, bk_mats, out_vel, out_pos;
    DBuf<float2> bk_brot, bk_boxHalf, bk_polyVerts, bk_polyNormals;
    DBuf<float> bk_wrap, bk_bound, bk_timer, bk_cworldRot, bk_minExt, bk_circle;
    DBuf<uint8_t> bk_bstate, staging, out_state;
    DBuf<uint32_t> bk_island, bk_cbody, bk_cshape, bk_cmat, bk_polyOff, bk_polyCount, newWorldMask;
    DBuf<Manifold> bk_prev;
    DBuf<uint32_t> bk_prevColor;
    DBuf<unsigned long long> stagedSections;   // [joining world][section] byte offsets into 'staging'
    PinnedBuf hostStage, hostOut;              // page-locked copies of the staged blobs and the leaving bodies
    // Host reads: fields packed on the device (k_extract) into readStage, then copied straight into a page-locked
    // destination, or through two page-locked halves of readBounce (the copy of one chunk overlaps the host copy
    // of the previous one) into pageable memory.
    DBuf<uint8_t> readStage;
    PinnedBuf readBounce;
    cudaEvent_t readEv[2] = {nullptr, nullptr};
    // Asynchronous reads: a ring of device staging buffers; each read packs on the engine stream and copies on
    // copyStream, so the copy overlaps the steps launched after it.
    static constexpr int NASYNC = 4;
    struct AsyncSlot {
        DBuf<uint8_t> buf;
        cudaEvent_t packed = nullptr, done = nullptr;
        bool used = false;
    };
    AsyncSlot asyncSlot[NASYNC];
    uint32_t asyncNext = 0;
    cudaStream_t copyStream = nullptr;
    DBuf<uint32_t> queryFlag, queryOffset, queryList, queryCount;   // spatial query scratch
    DBuf<float> queryDist, queryListDist;
    DBuf<GatherSeg> gatherSegs;
    bool newWorldsPending = false;   // joined worlds take a full pose pass in their first step
    // Shape table sizes of the last upload.
    uint32_t nCircles = 0, nBoxes = 0, nPolygons = 0, nPolyVerts = 0, nMaterialRows = 0;
    // Counters.
    DBuf<StepCounters> dCounters;
    StepCounters* hCounters = nullptr;
    Scanner scanner;

    // Per-phase device timers (CUDA events on the world's stream) and the count of kernel launches.
    static constexpr int NPHASE = 15;
    bool profiling = false;
    // The collision-detection pass (AG2D_PHASE_COLLIDE) as a captured CUDA graph, replayed while its launch shapes
    // hold (list sizes, capacities, block sizes, whether the static tree is rebuilt).
    cudaGraphExec_t collideExec = nullptr;
    uint64_t collideKey[9] = {};
    uint64_t collideSeen[9] = {};   // the shape of the last pass run without a graph
    uint64_t collideLaunches = 0;
    cudaEvent_t ev[NPHASE][2] = {};
    bool evPending[NPHASE] = {};
    double phaseMs[NPHASE] = {};
    uint64_t phaseCalls[NPHASE] = {};
    uint64_t launches = 0;
    uint64_t listRebuilds = 0, retries = 0, regrows = 0;
    double hostMs = 0.0, syncMs = 0.0;

    void pbegin(int p)
    {
        if (!profiling) return;
        if (!ev[p][0]) { CK(cudaEventCreate(&ev[p][0])); CK(cudaEventCreate(&ev[p][1])); }
        CK(cudaEventRecord(ev[p][0], stream));
    }
    void pend(int p)
    {
        if (!profiling) return;
        CK(cudaEventRecord(ev[p][1], stream));
        evPending[p] = true;
    }
    void pcollect()
    {
        for (int p = 0; p < NPHASE; p++) {
            if (!evPending[p]) continue;
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, ev[p][0], ev[p][1]));
            phaseMs[p] += ms;
            phaseCalls[p]++;
            evPending[p] = false;
        }
    }

    DeviceWorld view() const
    {
        DeviceWorld w;
        w.nBodies = nBodies; w.nColliders = nColliders; w.nMaterials = objects.materialCount();
        w.bvel = bvel.p; w.bpos = bpos.p; w.brot = brot.p; w.wrapCount = wrapCount.p; w.boundRadius = boundRadius.p;
        w.sleepTimer = sleepTimer.p; w.bstate = bstate.p; w.sleepIsland = sleepIsland.p;
        w.cbody = cbody.p; w.cshape = cshape.p; w.cmat = cmat.p; w.coff = coff.p; w.cpose = cpose.p;
        w.cworldRot = cworldRot.p; w.caabb = caabb.p;
        w.circleRadius = circleRadius.p; w.boxHalf = boxHalf.p; w.polyOffset = polyOffset.p; w.polyCount = polyCount.p;
        w.polyVerts = polyVerts.p; w.polyNormals = polyNormals.p; w.materials = materials.p;
        const bool seg = nWorlds > 1;
        w.nWorlds = nWorlds;
        w.bodyWorld = seg ? bodyWorld.p : nullptr;
        w.colWorld = seg ? colWorld.p : nullptr;
        w.worldBodyStart = seg ? worldBodyStart.p : nullptr;
        w.worldColStart = seg ? worldColStart.p : nullptr;
        w.worldDirty = seg ? worldDirty.p : nullptr;
        return w;
    }

    // Per-body and per-collider work buffers for the current sizes (grow only).
    // capsKnown: the pair and manifold capacities were already set (a checkpoint's counts), so the first-upload
    // guess of INITIAL_PAIRS_PER_COLLIDER a collider is not applied.
    void sizeFor(bool capsKnown = false)
    {
        snapVel.reserve(nBodies); snapPos.reserve(nBodies); snapRot.reserve(nBodies); snapWrap.reserve(nBodies);
        snapTimer.reserve(nBodies); snapState.reserve(nBodies); snapIsland.reserve(nBodies);
        prevPose.reserve(nColliders);
        ccdHit.reserve(nBodies);
        const uint32_t nmax = std::max(nBodies, nColliders);
        for (auto* b : {&dynBody, &dynCol, &otherCol, &flagA, &flagB, &flagC, &offA, &offB, &offC}) b->reserve(nmax);
        dynSimd.reserve(nmax);
        dynColSimd.reserve(nmax);
        dynTree.reserve(nColliders, nWorlds);
        otherTree.reserve(nColliders, nWorlds);
        queryState.reserve(size_t(div_up(std::max<uint32_t>(nColliders, 1), 64)) + 1);
        bodyMax.reserve(nBodies);
        bodyMask.reserve(nBodies);
        ufParent.reserve(nBodies); ufFlag.reserve(nBodies); wakeIsland.reserve(nBodies);
        const uint32_t cap = std::max<uint32_t>(INITIAL_PAIRS_PER_COLLIDER * nColliders, 4096);
        if (!capsKnown && (cap > pairCap || cap > manifoldCap))
            reserveCapacities(std::max(pairCap + pairCap / 2, cap), std::max(manifoldCap + manifoldCap / 2, cap));
        scanner.reserve(std::max({pairCap, nColliders, nBodies}));
    }

    // Rebuilds the resident batch on the device: the worlds 'keep' (indices into worldExt, in order) followed by the
    // joining worlds 'add' (host blobs, indices local to each world). Every world's state is carried over element
    // for element, so the worlds step on exactly as they would alone; joining worlds get their first-step full
    // pose pass. One transfer per joining world; the gathers shift the stored indices. Returns synchronised.
    void repack(const std::vector<uint32_t>& keep, const std::vector<const StagedWorld*>& add)
    {
        ensureDevice();
        const cudaStream_t s = stream;
        // AG2D_SERVER_LOG: per-part times of each repack on stderr (synchronising between the parts).
        const bool log = std::getenv("AG2D_SERVER_LOG") != nullptr;
        auto tPrev = std::chrono::steady_clock::now();
        std::string parts;
        auto mark = [&](const char* name) {
            if (!log) return;
            CK(cudaStreamSynchronize(s));
            const auto now = std::chrono::steady_clock::now();
            parts += std::string(" ") + name + "=" +
                     std::to_string(std::chrono::duration<double, std::milli>(now - tPrev).count());
            tPrev = now;
        };
        const uint32_t W0 = uint32_t(worldExt.size());
        compactPrev();
        prevSegValid = false;
        // Current extents of the warm-start manifolds and of the sleeping islands' manifolds (both world-grouped).
        if (W0 == 1) {
            uint32_t n[2] = {0, 0};
            CK(cudaMemcpyAsync(n, nPrev.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(n + 1, nIsle.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            worldExt[0].man = n[0];
            worldExt[0].isle = n[1];
        } else if (W0 > 1 && manSegFresh) {
            isleSeg.reserve(W0 + 1);
            const uint32_t g = gridFor(std::max<uint32_t>(manifoldCap, isleUpper));
            k_manifold_segments<<<g, 256, 0, s>>>(prevManifolds.p, nPrev.p, cbody.p, bodyWorld.p, W0, manSeg.p);
            k_manifold_segments<<<g, 256, 0, s>>>(isle.p, nIsle.p, cbody.p, bodyWorld.p, W0, isleSeg.p);
            CK(cudaGetLastError());
            std::vector<uint32_t> seg(W0 + 1), iseg(W0 + 1);
            CK(cudaMemcpyAsync(seg.data(), manSeg.p, (W0 + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(iseg.data(), isleSeg.p, (W0 + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            for (uint32_t k = 0; k < W0; k++) {
                worldExt[k].man = seg[k + 1] - seg[k];
                worldExt[k].isle = iseg[k + 1] - iseg[k];
            }
        }
        auto prefix = [](const std::vector<WorldExtent>& ex, uint32_t WorldExtent::*f) {
            std::vector<uint32_t> st(ex.size() + 1, 0);
            for (size_t i = 0; i < ex.size(); i++) st[i + 1] = st[i] + ex[i].*f;
            return st;
        };
        constexpr int NK = 9;
        static constexpr uint32_t WorldExtent::*kinds[NK] = {&WorldExtent::body, &WorldExtent::col,
                                                             &WorldExtent::circle, &WorldExtent::box,
                                                             &WorldExtent::poly, &WorldExtent::vert,
                                                             &WorldExtent::mat, &WorldExtent::man,
                                                             &WorldExtent::isle};
        std::vector<uint32_t> oldStart[NK], newStart[NK];
        std::vector<WorldExtent> next;
        for (uint32_t k : keep) next.push_back(worldExt[k]);
        for (const StagedWorld* w : add) next.push_back(w->ext);
        for (int c = 0; c < NK; c++) {
            oldStart[c] = prefix(worldExt, kinds[c]);
            newStart[c] = prefix(next, kinds[c]);
        }
        // Segments per kind (empty ones left out). A kept world's segment reads the current arrays from its old
        // start; a joining world's reads its staged sections (src = its index among the joining worlds). The
        // deltas shift the indices stored inside the elements to the new starts.
        std::vector<GatherSeg> segs[NK];
        for (size_t j = 0; j < next.size(); j++) {
            const bool fresh = j >= keep.size();
            GatherSeg g{};
            g.fromNew = fresh ? 1u : 0u;
            int32_t d[NK];
            for (int c = 0; c < NK; c++)
                d[c] = int32_t(newStart[c][j]) - (fresh ? 0 : int32_t(oldStart[c][keep[j]]));
            g.dBody = d[0]; g.dCol = d[1]; g.dCircle = d[2]; g.dBox = d[3]; g.dPoly = d[4]; g.dVert = d[5];
            g.dMat = d[6];
            for (int c = 0; c < NK; c++) {
                g.dst = newStart[c][j];
                g.src = fresh ? uint32_t(j - keep.size()) : oldStart[c][keep[j]];
                g.count = next[j].*kinds[c];
                if (g.count) segs[c].push_back(g);
            }
        }
        std::vector<GatherSeg> allSegs;
        uint32_t segOff[NK + 1] = {0};
        for (int c = 0; c < NK; c++) {
            segOff[c] = uint32_t(allSegs.size());
            allSegs.insert(allSegs.end(), segs[c].begin(), segs[c].end());
        }
        segOff[NK] = uint32_t(allSegs.size());
        mark("plan");
        gatherSegs.upload(allSegs.data(), allSegs.size(), s);   // empty when every world leaves
        // Staging: each joining world's blob at a 256-byte aligned offset, one transfer each.
        std::vector<unsigned long long> secOff(std::max<size_t>(add.size(), 1) * NSEC, 0);
        uint64_t stagedBytes = 0;
        for (size_t f = 0; f < add.size(); f++) {
            for (uint32_t k = 0; k < NSEC; k++) secOff[f * NSEC + k] = stagedBytes + add[f]->sec[k];
            stagedBytes += (add[f]->blob.size() + 255) & ~uint64_t(255);
        }
        staging.reserve(std::max<uint64_t>(stagedBytes, 1));
        // The blobs are packed into a page-locked buffer and go over in one transfer.
        hostStage.reserve(std::max<uint64_t>(stagedBytes, 1));
        uint64_t at = 0;
        for (const StagedWorld* w : add) {
            if (!w->blob.empty()) std::memcpy(hostStage.p + at, w->blob.data(), w->blob.size());
            at += (w->blob.size() + 255) & ~uint64_t(255);
        }
        if (stagedBytes) CK(cudaMemcpyAsync(staging.p, hostStage.p, stagedBytes, cudaMemcpyHostToDevice, s));
        stagedSections.upload(secOff.data(), secOff.size(), s);
        mark("stage");
        // Gathers into the back buffers, then swap them in front.
        const uint32_t grid = gridFor(std::max(newStart[0].back(), newStart[1].back()) + 1);
        auto run = [&](auto& front, auto& back, uint32_t section, int kind, uint32_t mode) {
            using T = std::remove_reference_t<decltype(*front.p)>;
            const uint32_t total = newStart[kind].back();
            // Warm-start manifolds trade places with the current-step buffer every step: keep the full capacity.
            back.reserve(std::max<uint32_t>(kind == 7 ? std::max(total, manifoldCap) : total, 1));
            CK(launch_gather(back.p, front.p, reinterpret_cast<const T*>(staging.p), gatherSegs.p + segOff[kind],
                             segOff[kind + 1] - segOff[kind], total, mode, grid, s, stagedSections.p, NSEC, section));
            swap_bufs(front, back);
        };
        run(bvel, bk_bvel, SEC_VEL, 0, GATHER_PLAIN);
        run(bpos, bk_bpos, SEC_POS, 0, GATHER_PLAIN);
        run(brot, bk_brot, SEC_ROT, 0, GATHER_PLAIN);
        run(wrapCount, bk_wrap, SEC_WRAP, 0, GATHER_PLAIN);
        run(boundRadius, bk_bound, SEC_BOUND, 0, GATHER_PLAIN);
        run(sleepTimer, bk_timer, SEC_TIMER, 0, GATHER_PLAIN);
        run(bstate, bk_bstate, SEC_STATE, 0, GATHER_PLAIN);
        run(sleepIsland, bk_island, SEC_ISLAND, 0, GATHER_ISLAND);
        run(cbody, bk_cbody, SEC_CBODY, 1, GATHER_BODY);
        run(cshape, bk_cshape, SEC_CSHAPE, 1, GATHER_SHAPE);
        run(cmat, bk_cmat, SEC_CMAT, 1, GATHER_MATERIAL);
        run(coff, bk_coff, SEC_COFF, 1, GATHER_PLAIN);
        run(cpose, bk_cpose, SEC_CPOSE, 1, GATHER_PLAIN);
        run(caabb, bk_caabb, SEC_CAABB, 1, GATHER_PLAIN);
        run(cworldRot, bk_cworldRot, SEC_CROT, 1, GATHER_PLAIN);
        run(minExtent, bk_minExt, SEC_MINEXT, 1, GATHER_PLAIN);
        run(circleRadius, bk_circle, SEC_CIRCLE, 2, GATHER_PLAIN);
        run(boxHalf, bk_boxHalf, SEC_BOXHALF, 3, GATHER_PLAIN);
        run(polyOffset, bk_polyOff, SEC_POLYOFF, 4, GATHER_VERTEX);
        run(polyCount, bk_polyCount, SEC_POLYCOUNT, 4, GATHER_PLAIN);
        run(polyVerts, bk_polyVerts, SEC_POLYVERTS, 5, GATHER_PLAIN);
        run(polyNormals, bk_polyNormals, SEC_POLYNORMALS, 5, GATHER_PLAIN);
        run(materials, bk_mats, SEC_MATS, 6, GATHER_PLAIN);
        run(prevManifolds, bk_prev, SEC_PREV, 7, GATHER_PLAIN);
        run(prevColor, bk_prevColor, SEC_PREVCOLOR, 7, GATHER_PLAIN);
        run(isle, bk_isle, SEC_ISLE, 8, GATHER_PLAIN);
        run(isleId, bk_isleId, SEC_ISLEID, 8, GATHER_ISLAND);
        mark("gather");
        // Sizes, partition and per-world state.
        worldExt = next;
        const uint32_t W = uint32_t(next.size());
        nBodies = newStart[0].back();
        nColliders = newStart[1].back();
        nCircles = newStart[2].back(); nBoxes = newStart[3].back(); nPolygons = newStart[4].back();
        nPolyVerts = newStart[5].back(); nMaterialRows = newStart[6].back();
        objects.materials.assign(size_t(nMaterialRows) * 3, 0.0f);   // the material count the device view reads
        nStatic = 0;
        for (const WorldExtent& e : next) nStatic += e.statics;
        prevCount = newStart[7].back();
        CK(cudaMemcpyAsync(nPrev.p, &prevCount, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        isleUpper = newStart[8].back();
        CK(cudaMemcpyAsync(nIsle.p, &isleUpper, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        nWorlds = std::max<uint32_t>(W, 1);
        hBodyStart = newStart[0];
        hColStart = newStart[1];
        if (W == 0) { hBodyStart = {0, 0}; hColStart = {0, 0}; }
        sizeFor();
        mark("size");
        const uint32_t ones = std::max<uint32_t>(nBodies, 1);
        k_fill_u32<<<gridFor(ones), 256, 0, s>>>(ccdHit.p, ones, ORDERED_ONE);
        if (nWorlds > 1) {
            bodyWorld.reserve(std::max<uint32_t>(nBodies, 1));
            colWorld.reserve(std::max<uint32_t>(nColliders, 1));
            worldBodyStart.upload(hBodyStart.data(), hBodyStart.size(), s);
            worldColStart.upload(hColStart.data(), hColStart.size(), s);
            k_world_of<<<gridFor(nBodies), 256, 0, s>>>(worldBodyStart.p, nWorlds, nBodies, bodyWorld.p);
            k_world_of<<<gridFor(nColliders), 256, 0, s>>>(worldColStart.p, nWorlds, nColliders, colWorld.p);
            manSeg.reserve(nWorlds + 1);
            nextWorld.reserve(2);
            worldDirty.reserve(nWorlds);
            CK(cudaMemsetAsync(worldDirty.p, 0, sizeof(uint32_t) * nWorlds, s));
            setTeams(teamColliders, teamThreads);
        }
        // Joining worlds: a full pose pass in their first step (as a freshly uploaded world has).
        newWorldMask.reserve(nWorlds);
        std::vector<uint32_t> mask(nWorlds, 0u);
        for (size_t j = keep.size(); j < next.size(); j++) mask[j] = 1u;
        newWorldMask.upload(mask.data(), mask.size(), s);
        newWorldsPending = next.size() > keep.size();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        mark("partition");
        if (log)
            std::fprintf(stderr, "ag2d repack worlds=%zu joined=%zu bodies=%u colliders=%u ms:%s\n", next.size(),
                         add.size(), nBodies, nColliders, parts.c_str());
        hostDirty = false;
        listsDirty = true;
        otherDirty = true;
        fullPose = false;
        manSegFresh = false;
        lastManifolds = prevCount;
    }

    // The final body state (velocity, pose, state) of the given resident worlds, concatenated in that order: one
    // device gather and one transfer per field.
    void exportBodies(const std::vector<uint32_t>& worlds, std::vector<float4>& vel, std::vector<float4>& pos,
                      std::vector<uint8_t>& state)
    {
        const cudaStream_t s = stream;
        std::vector<uint32_t> start(worldExt.size() + 1, 0);
        for (size_t k = 0; k < worldExt.size(); k++) start[k + 1] = start[k] + worldExt[k].body;
        std::vector<GatherSeg> segs;
        uint32_t total = 0;
        for (uint32_t k : worlds) {
            GatherSeg g{};
            g.dst = total;
            g.src = start[k];
            g.count = worldExt[k].body;
            total += g.count;
            if (g.count) segs.push_back(g);
        }
        vel.resize(total); pos.resize(total); state.resize(total);
        if (!total) return;
        gatherSegs.upload(segs.data(), segs.size(), s);
        out_vel.reserve(total); out_pos.reserve(total); out_state.reserve(total);
        const uint32_t grid = gridFor(total), n = uint32_t(segs.size());
        CK(launch_gather<float4>(out_vel.p, bvel.p, nullptr, gatherSegs.p, n, total, GATHER_PLAIN, grid, s, nullptr, 0, 0));
        CK(launch_gather<float4>(out_pos.p, bpos.p, nullptr, gatherSegs.p, n, total, GATHER_PLAIN, grid, s, nullptr, 0, 0));
        CK(launch_gather<uint8_t>(out_state.p, bstate.p, nullptr, gatherSegs.p, n, total, GATHER_PLAIN, grid, s, nullptr,
                                  0, 0));
        // Through a page-locked buffer: velocities, poses, states back to back.
        const size_t bv = size_t(total) * sizeof(float4);
        hostOut.reserve(2 * bv + total);
        CK(cudaMemcpyAsync(hostOut.p, out_vel.p, bv, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hostOut.p + bv, out_pos.p, bv, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hostOut.p + 2 * bv, out_state.p, total, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        std::memcpy(vel.data(), hostOut.p, bv);
        std::memcpy(pos.data(), hostOut.p + bv, bv);
        std::memcpy(state.data(), hostOut.p + 2 * bv, total);
    }

    // Sizes every per-element buffer of a batch for 'bodies' resident bodies (one collider each) up front, so
    // that a server filling up does not reallocate on the way. Only for an engine with no resident world.
    void reserveResident(uint32_t bodies)
    {
        ensureDevice();
        const uint32_t b = std::max<uint32_t>(bodies, 1), verts = 8 * b, worlds = std::max<uint32_t>(b / 16, 2);
        auto both = [](auto& x, auto& y, size_t n) { x.reserve(n); y.reserve(n); };
        both(bvel, bk_bvel, b); both(bpos, bk_bpos, b); both(brot, bk_brot, b); both(wrapCount, bk_wrap, b);
        both(boundRadius, bk_bound, b); both(sleepTimer, bk_timer, b); both(bstate, bk_bstate, b);
        both(sleepIsland, bk_island, b); both(cbody, bk_cbody, b); both(cshape, bk_cshape, b);
        both(cmat, bk_cmat, b); both(coff, bk_coff, b); both(cpose, bk_cpose, b); both(caabb, bk_caabb, b);
        both(cworldRot, bk_cworldRot, b); both(minExtent, bk_minExt, b); both(circleRadius, bk_circle, b);
        both(boxHalf, bk_boxHalf, b); both(polyOffset, bk_polyOff, b); both(polyCount, bk_polyCount, b);
        both(polyVerts, bk_polyVerts, verts); both(polyNormals, bk_polyNormals, verts); both(materials, bk_mats, worlds);
        bodyWorld.reserve(b); colWorld.reserve(b); worldBodyStart.reserve(worlds + 1); worldColStart.reserve(worlds + 1);
        manSeg.reserve(worlds + 1); worldDirty.reserve(worlds); newWorldMask.reserve(worlds);
        staging.reserve(size_t(b) * 64);
        hostStage.reserve(size_t(b) * 64);
        hostOut.reserve(size_t(b) * 8);
        const uint32_t saveB = nBodies, saveC = nColliders, saveW = nWorlds;
        nBodies = b; nColliders = b; nWorlds = worlds;
        sizeFor();
        bk_prev.reserve(manifoldCap);
        bk_prevColor.reserve(manifoldCap);
        nBodies = saveB; nColliders = saveC; nWorlds = saveW;
        CK(cudaStreamSynchronize(stream));
    }

    // Launch shape of the CTAs that solve worlds larger than a team: mode bit 0 = 256 threads (else 512), bit 1 =
    // pipelined global-record passes.
    uint32_t bigMode() const { return (bigThreads == 256 ? 1u : 0u) | (bigPipelined ? 2u : 0u); }
    void setBigMode(uint32_t mode)
    {
        bigThreads = (mode & 1u) ? 256u : 512u;
        bigPipelined = (mode & 2u) != 0;
        if (nWorlds > 1) setTeams(teamColliders, teamThreads);
    }

    // Solver teams: consecutive worlds packed while the team stays within 'colliders' colliders (a larger world is
    // a team of its own), scheduled largest first, each solved by one CTA of 'threads' threads.
    void setTeams(uint32_t colliders, uint32_t threads)
    {
        teamColliders = colliders;
        teamThreads = threads;
        maxWorldCols = 0;
        for (uint32_t k = 0; k < nWorlds; k++) maxWorldCols = std::max(maxWorldCols, hColStart[k + 1] - hColStart[k]);
        teamBodyCap = std::min<uint32_t>(MAX_TEAM_BODY_CAP, colliders);
        // Constraint records kept on chip: room for 3 manifolds per collider (a settled pile of convex bodies has
        // about 1.5 on average, with denser worlds well above), within the CTA's shared-memory limit; a team with
        // more solves from global memory.
        auto consFit = [&](uint32_t bodyCap, uint32_t want) -> uint32_t {
            if (!consOnChip) return 0;
            const size_t room = (TEAM_SMEM_MAX - size_t(bodyCap) * 2 * sizeof(float4)) / CONS_SMEM_BYTES;
            return uint32_t(std::min<size_t>(want, room));
        };
        teamConsCap = consFit(teamBodyCap, 3 * colliders);
        int perSm = 0;
        CK(team_solver_blocks_per_sm(teamThreads, false, teamBodyCap, teamConsCap, &perSm));
        teamBlocks = uint32_t(std::max(1, perSm) * dev.sms);
        // Worlds above the team size are teams of their own ("big", solved by bigThreads-thread CTAs);
        // the others are packed, in order, into teams of up to 'colliders' colliders.
        std::vector<uint32_t> start{0};
        std::vector<uint32_t> big, small;
        uint32_t acc = 0, bigMax = 0;
        auto close = [&](uint32_t k) {
            if (k > start.back()) { small.push_back(uint32_t(start.size() - 1)); start.push_back(k); }
            acc = 0;
        };
        for (uint32_t k = 0; k < nWorlds; k++) {
            const uint32_t c = hColStart[k + 1] - hColStart[k];
            if (c > colliders) {
                close(k);
                big.push_back(uint32_t(start.size() - 1));
                start.push_back(k + 1);
                bigMax = std::max(bigMax, c);
                continue;
            }
            if (acc > 0 && acc + c > colliders) close(k);
            acc += c;
        }
        close(nWorlds);
        auto size = [&](uint32_t t) { return hColStart[start[t + 1]] - hColStart[start[t]]; };
        auto bySize = [&](uint32_t x, uint32_t y) { return size(x) > size(y); };
        std::stable_sort(big.begin(), big.end(), bySize);
        std::stable_sort(small.begin(), small.end(), bySize);
        nTeams = uint32_t(small.size());
        nBigTeams = uint32_t(big.size());
        bigBodyCap = std::min<uint32_t>(MAX_TEAM_BODY_CAP, bigMax);
        bigConsCap = consFit(bigBodyCap, 3 * bigMax);
        bigBlocks = 1;
        if (nBigTeams) {
            CK(team_solver_blocks_per_sm(bigThreads, bigPipelined, bigBodyCap, bigConsCap, &perSm));
            bigBlocks = uint32_t(std::max(1, perSm) * dev.sms);
        }
        std::vector<uint32_t> order(small);
        order.insert(order.end(), big.begin(), big.end());   // small teams, then big teams
        teamWorld.upload(start.data(), start.size(), stream);
        teamOrder.upload(order.data(), std::max<size_t>(order.size(), 1), stream);
        CK(cudaStreamSynchronize(stream));
    }

    // Installs the world partition of a batch: world k owns bodies [bodyStart[k], bodyStart[k + 1]) and colliders
    // [colStart[k], colStart[k + 1]). Called after the arrays are uploaded.
    void setPartition(const std::vector<uint32_t>& bodyStart, const std::vector<uint32_t>& colStart)
    {
        const cudaStream_t s = stream;
        nWorlds = uint32_t(bodyStart.size() - 1);
        hBodyStart = bodyStart;
        hColStart = colStart;
        std::vector<uint32_t> bw(nBodies), cw(nColliders);
        for (uint32_t k = 0; k < nWorlds; k++) {
            for (uint32_t i = bodyStart[k]; i < bodyStart[k + 1]; i++) bw[i] = k;
            for (uint32_t i = colStart[k]; i < colStart[k + 1]; i++) cw[i] = k;
        }
        bodyWorld.upload(bw.data(), bw.size(), s);
        colWorld.upload(cw.data(), cw.size(), s);
        worldBodyStart.upload(bodyStart.data(), bodyStart.size(), s);
        worldColStart.upload(colStart.data(), colStart.size(), s);
        manSeg.reserve(nWorlds + 1);
        nextWorld.reserve(2);
        setTeams(teamColliders, teamThreads);
        worldDirty.reserve(nWorlds);
        CK(cudaMemsetAsync(worldDirty.p, 0, sizeof(uint32_t) * nWorlds, s));
        dynSimd.reserve(std::max(nBodies, nColliders));
        dynColSimd.reserve(std::max(nBodies, nColliders));
        dynTree.reserve(nColliders, nWorlds);
        otherTree.reserve(nColliders, nWorlds);
        CK(cudaStreamSynchronize(s));
        listsDirty = true;
        otherDirty = true;
        fullPose = true;
    }

    // Checkpoint layout of the current state (counts from the host's view of the engine; the warm-start count is
    // read from the device).
    CkptHeader checkpointLayout()
    {
        ensureUploaded();
        CkptHeader h{};
        std::memcpy(h.magic, CKPT_MAGIC, sizeof(h.magic));
        h.version = CKPT_VERSION;
        h.headerBytes = sizeof(CkptHeader);
        h.settings = settings;
        h.nWorlds = nWorlds;
        h.nBodies = nBodies; h.nColliders = nColliders; h.nCircles = nCircles; h.nBoxes = nBoxes;
        h.nPolygons = nPolygons; h.nPolyVerts = nPolyVerts; h.nMaterialRows = nMaterialRows;
        h.nStatic = nStatic;
        h.lastManifolds = lastManifolds;
        h.lastPairs = lastPairs;
        compactPrev();
        CK(cudaMemcpyAsync(&h.nPrev, nPrev.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(&h.nIsle, nIsle.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        const uint64_t b = nBodies, c = nColliders, m = h.nPrev, wp = uint64_t(nWorlds) + 1, si = h.nIsle;
        const uint64_t len[NCK] = {
            b * 16, b * 16, b * 8, b * 4, b * 4, b * 4, b, b * 4,
            c * 4, c * 4, c * 4, c * 16, c * 16, c * 16, c * 4, c * 4,
            uint64_t(nCircles) * 4, uint64_t(nBoxes) * 8, uint64_t(nPolygons) * 4, uint64_t(nPolygons) * 4,
            uint64_t(nPolyVerts) * 8, uint64_t(nPolyVerts) * 8, uint64_t(nMaterialRows) * 16, m * sizeof(Manifold),
            m * 4, wp * 4, wp * 4, si * sizeof(Manifold), si * 4};
        uint64_t at = (sizeof(CkptHeader) + 255) & ~uint64_t(255);
        for (uint32_t k = 0; k < NCK; k++) {
            h.off[k] = at;
            h.len[k] = len[k];
            at += (len[k] + 255) & ~uint64_t(255);
        }
        h.totalBytes = at;
        return h;
    }

    // Writes the checkpoint into host memory 'dst' (h.totalBytes bytes): one transfer per section, all on the engine
    // stream, then one wait.
    void saveCheckpoint(const CkptHeader& h, uint8_t* dst)
    {
        const cudaStream_t s = stream;
        std::memcpy(dst, &h, sizeof(h));
        const void* src[NCK] = {bvel.p, bpos.p, brot.p, wrapCount.p, boundRadius.p, sleepTimer.p, bstate.p,
                                sleepIsland.p, cbody.p, cshape.p, cmat.p, coff.p, cpose.p, caabb.p, cworldRot.p,
                                minExtent.p, circleRadius.p, boxHalf.p, polyOffset.p, polyCount.p, polyVerts.p,
                                polyNormals.p, materials.p, prevManifolds.p, prevColor.p, nullptr, nullptr};
        for (uint32_t k = 0; k < CK_WBODY; k++)
            if (h.len[k]) CK(cudaMemcpyAsync(dst + h.off[k], src[k], h.len[k], cudaMemcpyDeviceToHost, s));
        std::vector<uint32_t> bs = hBodyStart, cs = hColStart;
        if (nWorlds <= 1) { bs = {0, nBodies}; cs = {0, nColliders}; }
        std::memcpy(dst + h.off[CK_WBODY], bs.data(), h.len[CK_WBODY]);
        std::memcpy(dst + h.off[CK_WCOL], cs.data(), h.len[CK_WCOL]);
        if (h.len[CK_ISLE]) CK(cudaMemcpyAsync(dst + h.off[CK_ISLE], isle.p, h.len[CK_ISLE], cudaMemcpyDeviceToHost, s));
        if (h.len[CK_ISLEID])
            CK(cudaMemcpyAsync(dst + h.off[CK_ISLEID], isleId.p, h.len[CK_ISLEID], cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }

    // Makes this (fresh) engine the state a checkpoint holds: every section goes over as it lies in the blob (one
    // DMA each from page-locked memory), the world partition and the per-element world ids are rebuilt on the
    // device, and the next step starts exactly as the saved engine's next step would (work lists and the static
    // tree are rebuilt from the restored state, as after any change of state).
    void restoreCheckpoint(const CkptHeader& h, const uint8_t* src)
    {
        ensureDevice();
        const cudaStream_t s = stream;
        nBodies = h.nBodies; nColliders = h.nColliders; nCircles = h.nCircles; nBoxes = h.nBoxes;
        nPolygons = h.nPolygons; nPolyVerts = h.nPolyVerts; nMaterialRows = h.nMaterialRows; nStatic = h.nStatic;
        nWorlds = std::max<uint32_t>(h.nWorlds, 1);
        auto up = [&](auto& buf, uint32_t k, size_t count) {
            buf.reserve(std::max<size_t>(count, 1));
            if (h.len[k]) CK(cudaMemcpyAsync(buf.p, src + h.off[k], h.len[k], cudaMemcpyHostToDevice, s));
        };
        up(bvel, CK_VEL, nBodies); up(bpos, CK_POS, nBodies); up(brot, CK_ROT, nBodies);
        up(wrapCount, CK_WRAP, nBodies); up(boundRadius, CK_BOUND, nBodies); up(sleepTimer, CK_TIMER, nBodies);
        up(bstate, CK_STATE, nBodies); up(sleepIsland, CK_ISLAND, nBodies);
        up(cbody, CK_CBODY, nColliders); up(cshape, CK_CSHAPE, nColliders); up(cmat, CK_CMAT, nColliders);
        up(coff, CK_COFF, nColliders); up(cpose, CK_CPOSE, nColliders); up(caabb, CK_CAABB, nColliders);
        up(cworldRot, CK_CROT, nColliders); up(minExtent, CK_MINEXT, nColliders);
        up(circleRadius, CK_CIRCLE, nCircles); up(boxHalf, CK_BOXHALF, nBoxes); up(polyOffset, CK_POLYOFF, nPolygons);
        up(polyCount, CK_POLYCOUNT, nPolygons); up(polyVerts, CK_POLYVERTS, nPolyVerts);
        up(polyNormals, CK_POLYNORMALS, nPolyVerts); up(materials, CK_MATS, nMaterialRows);
        objects.materials.assign(size_t(nMaterialRows) * 3, 0.0f);   // the material count the device view reads
        const uint32_t* ws = reinterpret_cast<const uint32_t*>(src + h.off[CK_WBODY]);
        const uint32_t* wc = reinterpret_cast<const uint32_t*>(src + h.off[CK_WCOL]);
        hBodyStart.assign(ws, ws + nWorlds + 1);
        hColStart.assign(wc, wc + nWorlds + 1);
        // Buffers sized from the saved engine's last step (three times its pairs and manifolds: above the growth
        // threshold of twice the count), not from the first-upload guess of pairs a collider.
        const bool known = h.lastPairs > 0;
        if (known) {
            lastManifolds = h.lastManifolds;
            lastPairs = h.lastPairs;
            reserveCapacities(uint32_t(std::min<uint64_t>(std::max<uint64_t>(3ull * h.lastPairs, 4096), 1ull << 30)),
                              uint32_t(std::min<uint64_t>(std::max<uint64_t>({3ull * h.lastManifolds, h.nPrev, 4096}),
                                                          1ull << 30)));
        }
        sizeFor(known);
        if (h.nPrev > manifoldCap) reserveCapacities(std::max(h.nPrev, pairCap), h.nPrev);
        if (h.len[CK_PREV])
            CK(cudaMemcpyAsync(prevManifolds.p, src + h.off[CK_PREV], h.len[CK_PREV], cudaMemcpyHostToDevice, s));
        if (h.len[CK_PREVCOLOR])
            CK(cudaMemcpyAsync(prevColor.p, src + h.off[CK_PREVCOLOR], h.len[CK_PREVCOLOR], cudaMemcpyHostToDevice, s));
        prevCount = h.nPrev;
        prevSegValid = false;
        CK(cudaMemcpyAsync(nPrev.p, &prevCount, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        {
            // The store at the capacity the sleep pass would grow it to (half again on its size, at least the
            // manifold capacity), both buffers and the scratch, so the restored engine's steps allocate nothing.
            const size_t cap = std::max<size_t>({size_t(h.nIsle) + h.nIsle / 2, size_t(manifoldCap), size_t(1024)});
            for (auto* b : {&isle, &bk_isle}) b->reserve(cap);
            for (auto* b : {&isleId, &bk_isleId}) b->reserve(cap);
            reserveIsleScratch(uint32_t(std::min<size_t>(cap, 0xFFFFFFFFu)));
        }
        up(isle, CK_ISLE, h.nIsle);
        up(isleId, CK_ISLEID, h.nIsle);
        isleUpper = h.nIsle;
        CK(cudaMemcpyAsync(nIsle.p, &isleUpper, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        const uint32_t ones = std::max<uint32_t>(nBodies, 1);
        k_fill_u32<<<gridFor(ones), 256, 0, s>>>(ccdHit.p, ones, ORDERED_ONE);
        CK(cudaGetLastError());
        if (nWorlds > 1) {
            bodyWorld.reserve(std::max<uint32_t>(nBodies, 1));
            colWorld.reserve(std::max<uint32_t>(nColliders, 1));
            worldBodyStart.upload(hBodyStart.data(), hBodyStart.size(), s);
            worldColStart.upload(hColStart.data(), hColStart.size(), s);
            if (nBodies) k_world_of<<<gridFor(nBodies), 256, 0, s>>>(worldBodyStart.p, nWorlds, nBodies, bodyWorld.p);
            if (nColliders)
                k_world_of<<<gridFor(nColliders), 256, 0, s>>>(worldColStart.p, nWorlds, nColliders, colWorld.p);
            CK(cudaGetLastError());
            manSeg.reserve(nWorlds + 1);
            nextWorld.reserve(2);
            worldDirty.reserve(nWorlds);
            CK(cudaMemsetAsync(worldDirty.p, 0, sizeof(uint32_t) * nWorlds, s));
            setTeams(teamColliders, teamThreads);
        }
        CK(cudaStreamSynchronize(s));
        hostDirty = false;
        listsDirty = true;
        otherDirty = true;
        fullPose = false;
        aabbValid = true;
        newWorldsPending = false;
        manSegFresh = false;
        hintsReady = false;
        lastManifolds = h.lastManifolds;
    }

    ~ag2d_world()
    {
        if (collideExec) cudaGraphExecDestroy(collideExec);
        if (copyStream) cudaStreamSynchronize(copyStream);
        for (auto& a : asyncSlot) {
            if (a.packed) cudaEventDestroy(a.packed);
            if (a.done) cudaEventDestroy(a.done);
        }
        for (auto& e : readEv)
            if (e) cudaEventDestroy(e);
        if (copyStream) cudaStreamDestroy(copyStream);
        for (auto& e : ev) {
            if (e[0]) cudaEventDestroy(e[0]);
            if (e[1]) cudaEventDestroy(e[1]);
        }
        if (hCounters) cudaFreeHost(hCounters);
        if (forkEvent) cudaEventDestroy(forkEvent);
        if (joinEvent) cudaEventDestroy(joinEvent);
        if (sideStream) cudaStreamDestroy(sideStream);
        if (stream) cudaStreamDestroy(stream);
    }

    uint32_t gridFor(uint64_t n, uint32_t threads = 256) const
    {
        const uint64_t want = (n + threads - 1) / threads;
        const uint64_t cap = uint64_t(std::max(dev.sms, 1)) * std::max<uint32_t>(1, 2048 / threads);   // one full SM each
        return uint32_t(std::max<uint64_t>(1, std::min(want, cap)));
    }

    // Settings only: device resources are created on first device use (creating many worlds on the host, e.g. to
    // pack them into a batch, costs no CUDA calls per world).
    void init(const ag2d_world_settings& s)
    {
        settings = s;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw ApiError(AG2D_ERR_NO_DEVICE, "no CUDA device");
        if (s.device < 0 || s.device >= count) throw ApiError(AG2D_ERR_INVALID_ARG, "device ordinal out of range");
    }

    bool deviceReady() const { return stream != nullptr; }

    void ensureDevice()
    {
        if (deviceReady()) return;
        CK(cudaSetDevice(settings.device));
        dev = probe_device(settings.device);
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&sideStream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&forkEvent, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&joinEvent, cudaEventDisableTiming));
        CK(cudaMallocHost(reinterpret_cast<void**>(&hCounters), sizeof(StepCounters)));
        std::memset(hCounters, 0, sizeof(StepCounters));
        dCounters.reserve(1);
        scanner.status = &dCounters.p->status;
        scanner.blocks = uint32_t(std::max(dev.sms, 1)) * (2048 / SCAN_THREADS);
        bar.reserve(2);
        nManifolds.reserve(1);
        nPrev.reserve(1);
        nIsle.reserve(1);
        isleCounts.reserve(8);
        listCounts.reserve(3);
        colorCount.reserve(COLOR_SLOTS);
        colorStart.reserve(MAX_COLORS + 1);
        CK(cudaMemsetAsync(nPrev.p, 0, sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(nManifolds.p, 0, sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(nIsle.p, 0, sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(isleCounts.p, 0, 8 * sizeof(uint32_t), stream));
    }

    // Restore and sleep-pass scratch for a store of up to 'n' records.
    void reserveIsleScratch(uint32_t n)
    {
        n = std::max<uint32_t>(n, 1);
        for (auto* b : {&isleFlag, &isleOff, &isleList, &isleListWorld, &sleepKeepWorld}) b->reserve(n);
        scanner.reserve(n);
    }

    void reserveCapacities(uint32_t pairCapNew, uint32_t manCapNew)
    {
        regrows++;
        pairCap = pairCapNew;
        manifoldCap = manCapNew;
        pairs.reserve(pairCap);
        narrowState.reserve(size_t(div_up(pairCap, 64)) + 2);
        // Manifold arrays keep their contents (the previous step's manifolds are the warm-start source).
        auto grow_keep = [&](DBuf<Manifold>& b, uint32_t cap) {
            if (b.n >= cap && b.p) return;
            DBuf<Manifold> nb;
            nb.reserve(cap);
            if (b.p) CK(cudaMemcpyAsync(nb.p, b.p, b.n * sizeof(Manifold), cudaMemcpyDeviceToDevice, stream));
            CK(cudaStreamSynchronize(stream));
            swap_bufs(b, nb);
        };
        grow_keep(manifolds, manifoldCap);
        grow_keep(prevManifolds, manifoldCap);
        if (prevColor.n < manifoldCap || !prevColor.p) {   // colours of the warm-start manifolds are kept too
            DBuf<uint32_t> nb;
            nb.reserve(manifoldCap);
            if (prevColor.p) CK(cudaMemcpyAsync(nb.p, prevColor.p, prevColor.n * 4, cudaMemcpyDeviceToDevice, stream));
            CK(cudaStreamSynchronize(stream));
            swap_bufs(prevColor, nb);
        }
        color.reserve(manifoldCap);
        order.reserve(manifoldCap);
        prio.reserve(manifoldCap);
        listA.reserve(manifoldCap);
        listB.reserve(manifoldCap);
        pairBodies.reserve(manifoldCap);
        cons.reserve(manifoldCap);
        hashCap = 16;
        while (hashCap < 2 * manifoldCap) hashCap <<= 1;
        hashKeys.reserve(hashCap);
        hashVals.reserve(hashCap);
        scanner.reserve(std::max({pairCap, nColliders, nBodies}));
    }

    // The host objects (bodies, colliders, shapes, materials) in the upload format.
    void hostArrays(PackedArrays& a) const
    {
        const HostObjects& o = objects;
        const uint32_t nb = uint32_t(o.bodies.size()), nc = uint32_t(o.colliders.size());
        a.vel.resize(nb); a.pos.resize(nb); a.rot.resize(nb); a.wc.resize(nb); a.br.resize(nb); a.st.resize(nb);
        a.state.resize(nb); a.isl.resize(nb);
        for (uint32_t i = 0; i < nb; i++) {
            const HBody& b = o.bodies[i];
            a.vel[i] = make_float4(b.vx, b.vy, b.w, b.invMass);
            a.pos[i] = make_float4(b.comX, b.comY, b.rot, b.invInertia);
            a.rot[i] = make_float2(b.cos, b.sin);
            a.wc[i] = b.wrapCount; a.br[i] = b.boundRadius; a.st[i] = b.sleepTimer;
            a.state[i] = uint8_t(o.bodyGroups.groupOf(i) == 0 ? STATE_STATIC :
                                 (o.bodyGroups.groupOf(i) == 1 ? STATE_SLEEPING : STATE_DYNAMIC));
            a.isl[i] = b.sleepIsland;
        }
        a.cb.resize(nc); a.cs.resize(nc); a.cm.resize(nc); a.co.resize(nc);
        for (uint32_t i = 0; i < nc; i++) {
            const HCollider& c = o.colliders[i];
            a.cb[i] = c.body; a.cs[i] = (c.type << 30) | c.shape; a.cm[i] = c.material;
            a.co[i] = make_float4(c.comOffX, c.comOffY, c.localRot, 0.0f);
        }
        a.cr = o.circleRadius;
        a.bh.resize(o.boxHalfW.size());
        for (size_t i = 0; i < a.bh.size(); i++) a.bh[i] = make_float2(o.boxHalfW[i], o.boxHalfH[i]);
        a.po.clear(); a.pc.clear(); a.pv.clear(); a.pn.clear();
        for (const HPolygon& p : o.polygons) {
            a.po.push_back(uint32_t(a.pv.size()));
            a.pc.push_back(uint32_t(p.verts.size() / 2));
            for (size_t k = 0; k < p.verts.size() / 2; k++) {
                a.pv.push_back(make_float2(p.verts[2 * k], p.verts[2 * k + 1]));
                a.pn.push_back(make_float2(p.normals[2 * k], p.normals[2 * k + 1]));
            }
        }
        a.mats.resize(o.materialCount());
        for (size_t i = 0; i < a.mats.size(); i++)
            a.mats[i] = make_float4(o.materials[3 * i], o.materials[3 * i + 1], o.materials[3 * i + 2], 0.0f);
        a.prev.clear();
        a.isle.clear();
        a.isleId.clear();
    }

    // Uploads the host objects as the device state.
    void upload()
    {
        PackedArrays a;
        hostArrays(a);
        nBodies = uint32_t(a.vel.size());
        nColliders = uint32_t(a.cb.size());
        uploadArrays(a.vel, a.pos, a.rot, a.wc, a.br, a.st, a.state, a.isl, a.cb, a.cs, a.cm, a.co, a.cr, a.bh, a.po,
                     a.pc, a.pv, a.pn, a.mats);
    }

    void uploadArrays(const std::vector<float4>& vel, const std::vector<float4>& pos, const std::vector<float2>& rot,
                      const std::vector<float>& wc, const std::vector<float>& br, const std::vector<float>& st,
                      const std::vector<uint8_t>& state, const std::vector<uint32_t>& isl,
                      const std::vector<uint32_t>& cb, const std::vector<uint32_t>& cs,
                      const std::vector<uint32_t>& cm, const std::vector<float4>& co, const std::vector<float>& cr,
                      const std::vector<float2>& bh, const std::vector<uint32_t>& po,
                      const std::vector<uint32_t>& pc, const std::vector<float2>& pv,
                      const std::vector<float2>& pn, const std::vector<float4>& mats)
    {
        ensureDevice();
        const cudaStream_t s = stream;
        bvel.upload(vel.data(), nBodies, s); bpos.upload(pos.data(), nBodies, s); brot.upload(rot.data(), nBodies, s);
        wrapCount.upload(wc.data(), nBodies, s); boundRadius.upload(br.data(), nBodies, s);
        sleepTimer.upload(st.data(), nBodies, s); bstate.upload(state.data(), nBodies, s);
        sleepIsland.upload(isl.data(), nBodies, s);
        snapVel.reserve(nBodies); snapPos.reserve(nBodies); snapRot.reserve(nBodies); snapWrap.reserve(nBodies);
        snapTimer.reserve(nBodies); snapState.reserve(nBodies); snapIsland.reserve(nBodies);
        cbody.upload(cb.data(), nColliders, s); cshape.upload(cs.data(), nColliders, s);
        cmat.upload(cm.data(), nColliders, s); coff.upload(co.data(), nColliders, s);
        cpose.reserve(nColliders); caabb.reserve(nColliders); cworldRot.reserve(nColliders);
        CK(cudaMemsetAsync(cpose.p, 0, sizeof(float4) * std::max<uint32_t>(nColliders, 1), s));
        CK(cudaMemsetAsync(caabb.p, 0, sizeof(float4) * std::max<uint32_t>(nColliders, 1), s));
        CK(cudaMemsetAsync(cworldRot.p, 0, sizeof(float) * std::max<uint32_t>(nColliders, 1), s));
        circleRadius.upload(cr.data(), cr.size(), s); boxHalf.upload(bh.data(), bh.size(), s);
        polyOffset.upload(po.data(), po.size(), s); polyCount.upload(pc.data(), pc.size(), s);
        polyVerts.upload(pv.data(), pv.size(), s); polyNormals.upload(pn.data(), pn.size(), s);
        materials.upload(mats.data(), mats.size(), s);
        {
            const std::vector<float> me = min_extents(cs, cr, bh, po, pc, pv, pn);
            minExtent.upload(me.data(), me.size(), s);
            const std::vector<uint32_t> ones(std::max<uint32_t>(nBodies, 1), ORDERED_ONE);
            ccdHit.upload(ones.data(), ones.size(), s);
            prevPose.reserve(nColliders);
        }
        nStatic = uint32_t(std::count(state.begin(), state.end(), uint8_t(STATE_STATIC)));
        const uint32_t nmax = std::max(nBodies, nColliders);
        for (auto* b : {&dynBody, &dynCol, &otherCol, &flagA, &flagB, &flagC, &offA, &offB, &offC}) b->reserve(nmax);
        dynTree.reserve(nColliders, nWorlds);
        otherTree.reserve(nColliders, nWorlds);
        nCircles = uint32_t(cr.size()); nBoxes = uint32_t(bh.size()); nPolygons = uint32_t(po.size());
        nPolyVerts = uint32_t(pv.size()); nMaterialRows = uint32_t(mats.size());
        queryState.reserve(size_t(div_up(std::max<uint32_t>(nColliders, 1), 64)) + 1);
        bodyMax.reserve(nBodies);
        bodyMask.reserve(nBodies);
        ufParent.reserve(nBodies); ufFlag.reserve(nBodies); wakeIsland.reserve(nBodies);
        const uint32_t cap = std::max<uint32_t>(INITIAL_PAIRS_PER_COLLIDER * nColliders, 4096);
        reserveCapacities(std::max(pairCap, cap), std::max(manifoldCap, cap));
        CK(cudaMemsetAsync(nPrev.p, 0, sizeof(uint32_t), s));
        CK(cudaMemsetAsync(nManifolds.p, 0, sizeof(uint32_t), s));
        CK(cudaMemsetAsync(nIsle.p, 0, sizeof(uint32_t), s));
        isleUpper = 0;
        prevSegValid = false;
        optInDirty = true;
        motorsOnDevice = 0;
        jointsDirty = jointTotal() > 0;
        CK(cudaStreamSynchronize(s));
        hostDirty = false;
        listsDirty = true;
        fullPose = true;
        aabbValid = false;
        otherDirty = true;
        lastManifolds = 0;
        prevCount = 0;
    }

    void ensureUploaded()
    {
        ensureDevice();
        if (hostDirty) upload();
    }

    // The device state as upload-format host arrays plus the warm-start manifolds (for packing into a batch).
    void exportArrays(PackedArrays& a)
    {
        if (hostDirty) {   // never uploaded (or changed on the host since): no device round trip
            hostArrays(a);
            return;
        }
        ensureUploaded();
        compactPrev();
        const cudaStream_t s = stream;
        auto get = [&](auto& v, const auto* p, size_t n) {
            v.resize(n);
            if (n) CK(cudaMemcpyAsync(v.data(), p, n * sizeof(v[0]), cudaMemcpyDeviceToHost, s));
        };
        get(a.vel, bvel.p, nBodies); get(a.pos, bpos.p, nBodies); get(a.rot, brot.p, nBodies);
        get(a.wc, wrapCount.p, nBodies); get(a.br, boundRadius.p, nBodies); get(a.st, sleepTimer.p, nBodies);
        get(a.state, bstate.p, nBodies); get(a.isl, sleepIsland.p, nBodies);
        get(a.cb, cbody.p, nColliders); get(a.cs, cshape.p, nColliders); get(a.cm, cmat.p, nColliders);
        get(a.co, coff.p, nColliders); get(a.cp, cpose.p, nColliders);
        get(a.cr, circleRadius.p, nCircles); get(a.bh, boxHalf.p, nBoxes);
        get(a.po, polyOffset.p, nPolygons); get(a.pc, polyCount.p, nPolygons);
        get(a.pv, polyVerts.p, nPolyVerts); get(a.pn, polyNormals.p, nPolyVerts);
        get(a.mats, materials.p, nMaterialRows);
        uint32_t np = 0;
        CK(cudaMemcpyAsync(&np, nPrev.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        get(a.prev, prevManifolds.p, np);
        get(a.pcol, prevColor.p, np);
        uint32_t ni = 0;
        CK(cudaMemcpyAsync(&ni, nIsle.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        get(a.isle, isle.p, ni);
        get(a.isleId, isleId.p, ni);
        CK(cudaStreamSynchronize(s));
    }

    void rebuildLists()
    {
        listRebuilds++;
        const cudaStream_t s = stream;
        const uint32_t nmax = std::max(nBodies, nColliders);
        k_state_flags<<<gridFor(nmax), 256, 0, s>>>(bstate.p, cbody.p, nBodies, nColliders, flagA.p, flagB.p, flagC.p);
        CK(cudaGetLastError());
        scanner.run(flagA.p, offA.p, nBodies, listCounts.p + 0, s);
        scanner.run(flagB.p, offB.p, nColliders, listCounts.p + 1, s);
        scanner.run(flagC.p, offC.p, nColliders, listCounts.p + 2, s);
        k_scatter_list<<<gridFor(nBodies), 256, 0, s>>>(flagA.p, offA.p, nBodies, dynBody.p);
        k_scatter_list<<<gridFor(nColliders), 256, 0, s>>>(flagB.p, offB.p, nColliders, dynCol.p);
        k_scatter_list<<<gridFor(nColliders), 256, 0, s>>>(flagC.p, offC.p, nColliders, otherCol.p);
        CK(cudaGetLastError());
        if (nWorlds > 1) {
            // World segments of both trees (the lists are world-grouped).
            const uint32_t W = nWorlds;
            k_seg_starts<<<gridFor(W + 1), 256, 0, s>>>(offB.p, worldColStart.p, W, nColliders, listCounts.p + 1,
                                                        dynTree.segStart.p);
            k_seg_starts<<<gridFor(W + 1), 256, 0, s>>>(offC.p, worldColStart.p, W, nColliders, listCounts.p + 2,
                                                        otherTree.segStart.p);
            CK(cudaGetLastError());
            launches += 2;
        }
        uint32_t counts[3] = {0, 0, 0};
        CK(cudaMemcpyAsync(counts, listCounts.p, sizeof(counts), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        nDynBody = counts[0];
        nDynCol = counts[1];
        nOther = counts[2];
        if (nWorlds > 1) {
            // SIMD-path flag of each entry: its rank within its world's part of the list against (count & ~7).
            const uint32_t W = nWorlds;
            if (nDynBody)
                k_simd_flags<<<gridFor(nDynBody), 256, 0, s>>>(dynBody.p, nDynBody, offA.p, nBodies, bodyWorld.p,
                                                               worldBodyStart.p, W, dynSimd.p);
            if (nDynCol)
                k_simd_flags<<<gridFor(nDynCol), 256, 0, s>>>(dynCol.p, nDynCol, offB.p, nColliders, colWorld.p,
                                                              worldColStart.p, W, dynColSimd.p);
            CK(cudaGetLastError());
            launches += 2;
        }
        listsDirty = false;
    }

    void snapshot(bool restore)
    {
        const cudaStream_t s = stream;
        auto cp = [&](void* dst, const void* src, size_t bytes) {
            if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
        };
        const size_t n = nBodies;
        if (!restore) {
            cp(snapVel.p, bvel.p, n * sizeof(float4)); cp(snapPos.p, bpos.p, n * sizeof(float4));
            cp(snapRot.p, brot.p, n * sizeof(float2)); cp(snapWrap.p, wrapCount.p, n * sizeof(float));
            cp(snapTimer.p, sleepTimer.p, n * sizeof(float)); cp(snapState.p, bstate.p, n);
            cp(snapIsland.p, sleepIsland.p, n * sizeof(uint32_t));
            cp(snapMotorImpulse.p, motorImpulse.p, motorsOnDevice * sizeof(float));
        } else {
            cp(motorImpulse.p, snapMotorImpulse.p, motorsOnDevice * sizeof(float));
            cp(bvel.p, snapVel.p, n * sizeof(float4)); cp(bpos.p, snapPos.p, n * sizeof(float4));
            cp(brot.p, snapRot.p, n * sizeof(float2)); cp(wrapCount.p, snapWrap.p, n * sizeof(float));
            cp(sleepTimer.p, snapTimer.p, n * sizeof(float)); cp(bstate.p, snapState.p, n);
            cp(sleepIsland.p, snapIsland.p, n * sizeof(uint32_t));
        }
    }

    // ---- phases ----
    void phaseIntegrate()
    {
        const float damp = settings.angular_damping;
        const float dampHalf = (damp >= 0.0f && damp < 1.0f) ? std::pow(damp, settings.dt * 0.5f) : 2.0f;
        if (nDynBody) {
            pbegin(0);
            const uint8_t* simd = nWorlds > 1 ? dynSimd.p : nullptr;
            if (jointsActive()) {
                // The constraints between the halves (Simulation::integrateAndApplyConstraints, :392-407).
                k_integrate<<<gridFor(nDynBody), 256, 0, stream>>>(view(), dynBody.p, simd, nDynBody, settings.dt,
                                                                  settings.gravity_x, settings.gravity_y, dampHalf, 1u);
                launchJoints();
                k_integrate<<<gridFor(nDynBody), 256, 0, stream>>>(view(), dynBody.p, simd, nDynBody, settings.dt,
                                                                  settings.gravity_x, settings.gravity_y, dampHalf, 2u);
                launches += 2;
            } else {
                k_integrate<<<gridFor(nDynBody), 256, 0, stream>>>(view(), dynBody.p, simd, nDynBody, settings.dt,
                                                                  settings.gravity_x, settings.gravity_y, dampHalf, 3u);
                launches++;
            }
            CK(cudaGetLastError());
            pend(0);
        }
    }

    // full: every collider (or, with 'changedWorlds', those of the worlds whose bodies changed state this step).
    void phasePose(bool full, bool changedWorlds = false)
    {
        const uint32_t n = full ? nColliders : nDynCol;
        if (n == 0) return;
        pbegin(1);
        const uint32_t* mask = (full && changedWorlds && nWorlds > 1) ? worldDirty.p : nullptr;
        k_collider_pose<<<gridFor(n), 256, 0, stream>>>(view(), full ? nullptr : dynCol.p,
                                                         (full || nWorlds == 1) ? nullptr : dynColSimd.p, n, mask);
        CK(cudaGetLastError());
        pend(1);
        launches++;
    }

    // Radix passes over (keys, vals) for the digits [0, passes) with one histogram pass; the result ends in
    // t.keys / t.vals (buffers swap after an odd number of passes).
    void sortPasses(Tree& t, uint32_t n, uint32_t passes)
    {
        const cudaStream_t s = stream;
        CK(cudaMemsetAsync(t.hist.p, 0, 4 * 256 * sizeof(uint32_t), s));
        k_sort_histogram<<<gridFor(n), 256, 0, s>>>(t.keys.p, n, t.hist.p);
        k_sort_digit_scan<<<4, 256, 0, s>>>(t.hist.p);
        CK(cudaGetLastError());
        const uint32_t tiles = div_up(n, SORT_TILE);
        CK(cudaMemsetAsync(t.tileState.p, 0, size_t(tiles) * 256 * passes * sizeof(uint32_t), s));
        CK(cudaMemsetAsync(t.tileCounter.p, 0, 4 * sizeof(uint32_t), s));
        uint32_t *ki = t.keys.p, *vi = t.vals.p, *ko = t.keys2.p, *vo = t.vals2.p;
        for (uint32_t pass = 0; pass < passes; pass++) {
            k_sort_pass<<<tiles, SORT_THREADS, 0, s>>>(ki, vi, ko, vo, n, pass * 8, t.hist.p + pass * 256,
                                                        t.tileState.p + size_t(pass) * tiles * 256,
                                                        t.tileCounter.p + pass, &dCounters.p->status);
            CK(cudaGetLastError());
            std::swap(ki, ko);
            std::swap(vi, vo);
        }
        if (passes & 1) {
            swap_bufs(t.keys, t.keys2);
            swap_bufs(t.vals, t.vals2);
        }
        launches += 2 + passes;
    }

    // Tree over the colliders of 'list' (Morton keys from the world's bounds, sorted, Karras build, refit). With
    // several worlds the order is (world, Morton key) and every world gets its own tree over its segment.
    void buildTree(Tree& t, const uint32_t* list, uint32_t n)
    {
        const cudaStream_t s = stream;
        t.n = int(n);
        if (n == 0) return;
        const uint32_t W = nWorlds;
        const bool seg = W > 1;
        const uint32_t* cw = seg ? colWorld.p : nullptr;
        launches += 5 + (n > 1 ? 1 : 0);
        k_bounds_init<<<gridFor(W), 256, 0, s>>>(t.bounds.p, W);
        k_bounds<<<gridFor(n), 256, 0, s>>>(caabb.p, list, n, cw, t.bounds.p);
        k_morton<<<gridFor(n), 256, 0, s>>>(caabb.p, list, n, cw, t.bounds.p, t.keys.p, t.vals.p,
                                             seg ? t.keyOf.p : nullptr);
        CK(cudaGetLastError());
        const bool isDyn = &t == &dynTree;
        if (isDyn) pbegin(12);
        if (seg && maxWorldCols <= SEGMENT_SORT_MAX) {
            // Every world's segment sorted in shared memory, small and large segments by separate launches.
            if (!segSortReady) {
                CK(cudaFuncSetAttribute(k_segment_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(SEGMENT_SORT_MAX * sizeof(unsigned long long))));
                segSortReady = true;
            }
            const uint32_t grid = std::min<uint32_t>(W, uint32_t(dev.sms) * 8);
            k_segment_sort<<<grid, 256, SEGMENT_SORT_SMALL * sizeof(unsigned long long), s>>>(
                t.keys.p, t.vals.p, t.keys2.p, t.vals2.p, t.segStart.p, W, 0, SEGMENT_SORT_SMALL);
            launches++;
            if (maxWorldCols > SEGMENT_SORT_SMALL) {
                k_segment_sort<<<std::min<uint32_t>(W, uint32_t(dev.sms)), 1024,
                                 SEGMENT_SORT_MAX * sizeof(unsigned long long), s>>>(
                    t.keys.p, t.vals.p, t.keys2.p, t.vals2.p, t.segStart.p, W, SEGMENT_SORT_SMALL, SEGMENT_SORT_MAX);
                launches++;
            }
            CK(cudaGetLastError());
            swap_bufs(t.keys, t.keys2);
            swap_bufs(t.vals, t.vals2);
        } else {
            sortPasses(t, n, 4);
        }
        if (seg && maxWorldCols > SEGMENT_SORT_MAX) {
            // Stable passes on the world id: order (world, Morton key, collider).
            uint32_t passes = 1;
            while (passes < 4 && (W - 1) >> (8 * passes)) passes++;
            k_world_keys<<<gridFor(n), 256, 0, s>>>(t.vals.p, n, colWorld.p, t.keys.p);
            CK(cudaGetLastError());
            launches++;
            sortPasses(t, n, passes);
        }
        if (isDyn) pend(12);
        if (isDyn) pbegin(13);
        k_tree_gather<<<gridFor(n), 256, 0, s>>>(t.vals.p, n, seg ? t.keyOf.p : nullptr, cw, caabb.p,
                                                  seg ? t.sortedKey.p : nullptr, seg ? t.sortedWorld.p : nullptr,
                                                  t.leafAabb.p);
        k_lbvh_build<<<gridFor(n), 256, 0, s>>>(seg ? t.sortedKey.p : t.keys.p, seg ? t.sortedWorld.p : nullptr,
                                                 seg ? t.segStart.p : nullptr, int(n), t.child.p, t.range.p,
                                                 t.parent.p, t.leafParent.p, t.meet.p, t.rec.p);
        CK(cudaGetLastError());
        if (n > 1) {
            k_lbvh_refit<<<gridFor(n), 256, 0, s>>>(int(n), t.child.p, t.parent.p, t.leafParent.p, t.leafAabb.p,
                                                     t.nodeAabb.p, t.meet.p, t.rec.p);
            CK(cudaGetLastError());
        }
        if (isDyn) pend(13);
    }

    // Continuous collision detection after the dynamic poses (Simulation.cpp:299-316): sweep fast dynamic colliders
    // against the static colliders of their world, move hit bodies and their colliders back to the time of impact.
    void phaseCcd()
    {
        const cudaStream_t s = stream;
        if (nDynCol == 0 || nDynBody == 0) return;
        if (otherDirty) {
            pbegin(3);
            buildTree(otherTree, otherCol.p, nOther);
            pend(3);
            otherDirty = false;
        }
        otherTree.n = int(nOther);
        if (nOther == 0) return;
        pbegin(14);
        const DeviceWorld w = view();
        k_ccd_sweep<<<gridFor(nDynCol), 256, 0, s>>>(w, dynCol.p, nDynCol, otherTree.view(), snapPos.p, prevPose.p,
                                                     minExtent.p, ccdHit.p, &dCounters.p->status);
        k_ccd_shift_colliders<<<gridFor(nDynCol), 256, 0, s>>>(w, dynCol.p, nDynCol, snapPos.p, ccdHit.p);
        k_ccd_shift_bodies<<<gridFor(nDynBody), 256, 0, s>>>(w, dynBody.p, nDynBody, snapPos.p, ccdHit.p,
                                                             dCounters.p);
        CK(cudaGetLastError());
        pend(14);
        launches += 3;
    }

    void phaseBroad()
    {
        const cudaStream_t s = stream;
        pbegin(2);
        buildTree(dynTree, dynCol.p, nDynCol);
        pend(2);
        if (otherDirty) {
            pbegin(3);
            buildTree(otherTree, otherCol.p, nOther);
            pend(3);
            otherDirty = false;
        }
        otherTree.n = int(nOther);
        uint32_t* total = &dCounters.p->pairs;
        if (nDynCol == 0) {
            CK(cudaMemsetAsync(total, 0, sizeof(uint32_t), s));
            return;
        }
        pbegin(4);
        launches += 1;
        const uint32_t gq = gridFor(nDynCol, queryThreads);
        const uint32_t tiles = div_up(nDynCol, queryThreads);
        queryState.reserve(size_t(tiles) + 1);
        CK(cudaMemsetAsync(queryState.p, 0, (size_t(tiles) + 1) * sizeof(uint32_t), s));
        k_query<<<gq, queryThreads, 0, s>>>(dynTree.view(), otherTree.view(), cbody.p, pairs.p, pairCap, total,
                                            &dCounters.p->status, queryState.p, queryState.p + tiles);
        CK(cudaGetLastError());
        pend(4);
    }

    void phaseNarrow(bool warm = true)
    {
        const cudaStream_t s = stream;
        const uint32_t* nPairs = &dCounters.p->pairs;
        // Grid sized for the capacity, work bounded by the device-side pair count; the manifolds are compacted in
        // the same kernel.
        const uint32_t gn = gridFor(pairCap, narrowThreads);
        const uint32_t tilesCap = std::max<uint32_t>(div_up(pairCap, narrowThreads), 1);
        pbegin(5);
        CK(cudaMemsetAsync(narrowState.p, 0, (size_t(tilesCap) + 1) * sizeof(uint32_t), s));
        k_narrow<<<gn, narrowThreads, narrowThreads * NARROW_SMEM_PER_THREAD, s>>>(
            view(), pairs.p, nPairs, pairCap, manifolds.p, manifoldCap, nManifolds.p, dCounters.p, narrowState.p,
            narrowState.p + tilesCap);
        CK(cudaGetLastError());
        pend(5);
        launches += 1;
        if (!warm) return;
        pbegin(7);
        // Warm start from the previous step's manifolds.
        // Table sized for the manifolds actually stored (load <= 1/2), not the buffer capacity: a smaller table is
        // cheaper to clear and stays in L2.
        uint32_t slotsUsed = 1024;
        while (slotsUsed < 2 * prevCount && slotsUsed < hashCap) slotsUsed <<= 1;
        slotsUsed = std::min(slotsUsed, hashCap);
        CK(cudaMemsetAsync(hashKeys.p, 0xFF, size_t(slotsUsed) * sizeof(unsigned long long), s));
        // A batch keeps one table region per world (the previous list's world starts, kept from the last step's
        // solve or recomputed when the list changed since).
        const uint32_t* seg = nullptr;
        if (nWorlds > 1) {
            prevSeg.reserve(nWorlds + 1);
            if (!prevSegValid) {
                k_manifold_segments<<<gridFor(manifoldCap), 256, 0, s>>>(prevManifolds.p, nPrev.p, cbody.p,
                                                                         bodyWorld.p, nWorlds, prevSeg.p);
                launches++;
            }
            seg = prevSeg.p;
        }
        k_warm_insert<<<gridFor(manifoldCap), 256, 0, s>>>(prevManifolds.p, nPrev.p, hashKeys.p, hashVals.p, slotsUsed,
                                                           seg, colWorld.p, &dCounters.p->status);
        k_warm_lookup<<<gridFor(manifoldCap), 256, 0, s>>>(prevManifolds.p, manifolds.p, nManifolds.p, hashKeys.p,
                                                           hashVals.p, slotsUsed, seg, colWorld.p, dCounters.p,
                                                           prevColor.p, color.p);
        hintsReady = true;
        CK(cudaGetLastError());
        pend(7);
    }

    void phaseWake()
    {
        const cudaStream_t s = stream;
        pbegin(8);
        launches += 2;
        CK(cudaMemsetAsync(wakeIsland.p, 0, sizeof(uint32_t) * std::max<uint32_t>(nBodies, 1), s));
        k_wake<<<gridFor(manifoldCap), 256, 0, s>>>(view(), manifolds.p, nManifolds.p, wakeIsland.p, dCounters.p);
        k_wake_apply<<<gridFor(nBodies), 256, 0, s>>>(view(), wakeIsland.p, dCounters.p);
        CK(cudaGetLastError());
        pend(8);
    }

    // Manifolds of the islands that woke this step join the list (k_islands.cu, restore): fresh manifolds of their
    // pairs take the stored impulses; the rest are appended at the end of their world's segment (a batch's list is
    // merged into mergeMan / mergeHint, which then become 'manifolds' / 'color').
    void phaseRestore()
    {
        if (isleUpper == 0) return;
        const cudaStream_t s = stream;
        const DeviceWorld wv = view();
        reserveIsleScratch(isleUpper);
        uint32_t* cnt = isleCounts.p;
        uint32_t* st = &dCounters.p->status;
        const uint32_t gi = gridFor(isleUpper), gm = gridFor(manifoldCap);
        k_isle_stage_flags<<<gi, 256, 0, s>>>(wv, isle.p, isleId.p, nIsle.p, wakeIsland.p, isleFlag.p);
        scanner.run(isleFlag.p, isleOff.p, isleUpper, cnt + 0, s, nIsle.p);
        k_isle_stage_list<<<gi, 256, 0, s>>>(wv, isle.p, nIsle.p, isleFlag.p, isleOff.p, isleList.p, isleListWorld.p);
        uint32_t* hint = hintsReady ? color.p : nullptr;
        if (nWorlds > 1) {
            mergeMan.reserve(manifoldCap);
            mergeHint.reserve(manifoldCap);
            k_manifold_segments<<<gm, 256, 0, s>>>(manifolds.p, nManifolds.p, cbody.p, bodyWorld.p, nWorlds, manSeg.p);
            k_isle_merge<<<gm, 256, 0, s>>>(wv, manifolds.p, hint, nManifolds.p, manSeg.p, isle.p, isleList.p,
                                            isleListWorld.p, cnt + 0, manifoldCap, mergeMan.p,
                                            hint ? mergeHint.p : nullptr, st);
            swap_bufs(manifolds, mergeMan);
            if (hint) swap_bufs(color, mergeHint);
            launches += 2;
        } else {
            k_isle_append<<<gi, 256, 0, s>>>(manifolds.p, nManifolds.p, manifoldCap, hint, isle.p, isleList.p, cnt + 0,
                                             st);
            launches += 1;
        }
        k_isle_count<<<1, 32, 0, s>>>(nManifolds.p, cnt + 0, cnt + 0, manifoldCap, dCounters.p);
        CK(cudaGetLastError());
        launches += 4;
    }

    // After a step in which islands woke or fell asleep (k_islands.cu, sleep): the store drops the woken islands'
    // records and takes the manifolds of the bodies now asleep from the warm-start list ('prevManifolds'). The list
    // itself keeps those records until it is read (compactPrev): the next step cannot regenerate their pairs (both
    // bodies asleep, or one asleep and one static), so they warm-start nothing and give no colour hint, and the
    // next step replaces the list anyway.
    void phaseSleepStore(uint32_t storedBefore, bool slept, bool removals)
    {
        const cudaStream_t s = stream;
        const DeviceWorld wv = view();
        const uint32_t listN = std::max<uint32_t>(prevCount, 1), stored = std::max<uint32_t>(storedBefore, 1);
        const uint64_t need = uint64_t(storedBefore) + (slept ? prevCount : 0);
        if (need > 0xFFFFFFFFull) throw ApiError(AG2D_ERR_CAPACITY, "sleeping-island store would exceed 2^32 records");
        // Both store buffers keep one capacity (they trade places), grown together by half again when short, so a
        // steady store reallocates neither.
        if (isle.n < need || bk_isle.n < need || isleId.n < need || bk_isleId.n < need || !isle.p || !bk_isle.p) {
            // Half again on top of the need, at least doubling, and at least the manifold capacity (the store
            // rarely outgrows the contacts a step can hold): a store that fills as a batch settles reallocates (a
            // device synchronisation, slow to map) once or twice only, not inside a steady run of steps.
            const size_t cap = std::max<size_t>({size_t(need) + need / 2, size_t(1024), 2 * isle.n,
                                                 size_t(manifoldCap)});
            growKeep(isle, cap);
            growKeep(isleId, cap);
            DBuf<Manifold> nb;
            nb.reserve(cap);
            swap_bufs(bk_isle, nb);
            DBuf<uint32_t> nbi;
            nbi.reserve(cap);
            swap_bufs(bk_isleId, nbi);
            reserveIsleScratch(uint32_t(std::min<size_t>(cap, 0xFFFFFFFFu)));   // the scratch follows the store
        }
        reserveIsleScratch(stored);
        for (auto* b : {&sleepStay, &sleepMove, &sleepMoveOff, &sleepMoveIsland, &sleepMoveWorld}) b->reserve(manifoldCap);
        scanner.reserve(std::max(listN, stored));
        uint32_t* cnt = isleCounts.p;
        const bool batch = nWorlds > 1, checkAlive = nDestroyed > 0;
        const uint32_t gi = gridFor(stored), gl = gridFor(listN);
        if (slept) {
            k_isle_move_flags<<<gl, 256, 0, s>>>(wv, prevManifolds.p, nPrev.p, sleepStay.p, sleepMove.p,
                                                 sleepMoveIsland.p);
            scanner.run(sleepMove.p, sleepMoveOff.p, listN, cnt + 3, s, nPrev.p);
        } else {
            CK(cudaMemsetAsync(cnt + 3, 0, sizeof(uint32_t), s));
        }
        if (!batch && !removals) {
            // A single world that only gains records: they go after the kept ones, in place.
            k_isle_append_moved<<<gl, 256, 0, s>>>(prevManifolds.p, nPrev.p, sleepMove.p, sleepMoveOff.p,
                                                  sleepMoveIsland.p, nIsle.p, isle.p, isleId.p);
            k_isle_add_count<<<1, 32, 0, s>>>(nIsle.p, cnt + 3);
            CK(cudaGetLastError());
            launches += slept ? 4 : 2;
        } else {
            k_isle_keep_flags<<<gi, 256, 0, s>>>(wv, isle.p, isleId.p, nIsle.p, wakeIsland.p, checkAlive ? 1u : 0u,
                                                 isleFlag.p);
            scanner.run(isleFlag.p, isleOff.p, stored, cnt + 2, s, nIsle.p);
            if (batch)
                k_isle_sleep_worlds<<<gridFor(stored + listN), 256, 0, s>>>(wv, isle.p, nIsle.p, isleFlag.p,
                                                                           isleOff.p, prevManifolds.p, nPrev.p,
                                                                           slept ? sleepMove.p : nullptr,
                                                                           sleepMoveOff.p, sleepKeepWorld.p,
                                                                           sleepMoveWorld.p);
            k_isle_store_scatter<<<gridFor(stored + listN), 256, 0, s>>>(
                wv, isle.p, isleId.p, nIsle.p, isleFlag.p, isleOff.p, cnt + 2, prevManifolds.p, nPrev.p,
                slept ? sleepMove.p : nullptr, sleepMoveOff.p, cnt + 3, sleepMoveIsland.p,
                batch ? sleepKeepWorld.p : nullptr, batch ? sleepMoveWorld.p : nullptr, bk_isle.p, bk_isleId.p);
            k_isle_store_count<<<1, 32, 0, s>>>(cnt + 2, cnt + 3, nIsle.p);
            CK(cudaGetLastError());
            launches += (slept ? 2 : 0) + (batch ? 5 : 4);
            swap_bufs(isle, bk_isle);
            swap_bufs(isleId, bk_isleId);
        }
        if (slept) prevHoldsSleepers = true;
        isleUpper = uint32_t(need);
    }

    // Drops from the warm-start list the manifolds whose bodies sleep (they are in the store) or were destroyed:
    // the list as the reference's getBodyCollisionData holds it after a step. Called before the list is read or
    // packed.
    void compactPrev()
    {
        if (!prevHoldsSleepers) return;
        prevHoldsSleepers = false;
        prevSegValid = false;
        const cudaStream_t s = stream;
        const uint32_t listN = std::max<uint32_t>(prevCount, 1);
        for (auto* b : {&sleepStay, &sleepMove, &sleepStayOff, &sleepMoveIsland, &sleepColor}) b->reserve(manifoldCap);
        sleepList.reserve(manifoldCap);
        scanner.reserve(listN);
        uint32_t* cnt = isleCounts.p;
        k_isle_move_flags<<<gridFor(listN), 256, 0, s>>>(view(), prevManifolds.p, nPrev.p, sleepStay.p, sleepMove.p,
                                                         sleepMoveIsland.p);
        scanner.run(sleepStay.p, sleepStayOff.p, listN, cnt + 4, s, nPrev.p);
        k_isle_list_scatter<<<gridFor(listN), 256, 0, s>>>(prevManifolds.p, prevColor.p, nPrev.p, sleepStay.p,
                                                           sleepStayOff.p, sleepList.p, sleepColor.p);
        CK(cudaMemcpyAsync(nPrev.p, cnt + 4, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        CK(cudaGetLastError());
        launches += 3;
        swap_bufs(prevManifolds, sleepList);
        swap_bufs(prevColor, sleepColor);
        CK(cudaStreamSynchronize(s));
    }

    // Grows a buffer to at least 'count' elements, keeping its contents.
    template <class T>
    void growKeep(DBuf<T>& b, size_t count)
    {
        if (b.n >= count && b.p) return;
        DBuf<T> nb;
        nb.reserve(count);
        if (b.p) CK(cudaMemcpyAsync(nb.p, b.p, b.n * sizeof(T), cudaMemcpyDeviceToDevice, stream));
        CK(cudaStreamSynchronize(stream));
        swap_bufs(b, nb);
    }

    // Body constraints ---------------------------------------------------------------------------------------
    uint32_t jointTotal() const
    {
        uint32_t n = 0;
        for (const JointSystem& js : objects.jointSystems) n += uint32_t(js.joints.size());
        return n;
    }
    bool jointsActive() const
    {
        for (uint32_t k = 0; k < JOINT_KINDS; k++) if (jointActive[k]) return true;
        return false;
    }
    // The motors' accumulated impulses from the device into the host table (before the table is reordered or read).
    void pullMotorImpulses()
    {
        auto& motors = objects.jointSystems[JOINT_MOTOR].joints;
        const uint32_t n = std::min<uint32_t>(motorsOnDevice, uint32_t(motors.size()));
        if (n == 0) return;
        const std::vector<float> imp = download(motorImpulse.p, n, stream);
        for (uint32_t i = 0; i < n; i++) motors[i].impulse = imp[i];
    }
    // Before the host tables change (their dense order with them): the device impulses are read back first and
    // stop matching the table until the next rebuild.
    void beforeJointEdit()
    {
        pullMotorImpulses();
        motorsOnDevice = 0;
        jointsDirty = true;
    }
    // Regroups every constraint by its bodies' states (Sleeping when a body sleeps, Inactive when no body moves,
    // else Active: ObjectManager.cpp:1207-1220, 1330-1360), then uploads each kind's active constraints grouped by
    // level: level(j) = 1 + the highest level of the earlier active constraints of the kind (dense order) that
    // write one of j's moving bodies.
    void rebuildJoints()
    {
        jointsDirty = false;
        const cudaStream_t s = stream;
        pullMotorImpulses();
        const std::vector<uint8_t> state = download(bstate.p, nBodies, s);
        auto st = [&](uint32_t b) -> uint8_t { return b < state.size() ? state[b] : uint8_t(STATE_DESTROYED); };
        std::vector<uint32_t> last(std::max<uint32_t>(nBodies, 1));
        std::vector<uint2> edges;
        for (uint32_t k = 0; k < JOINT_KINDS; k++) {
            JointSystem& js = objects.jointSystems[k];
            std::vector<uint64_t> handles;
            for (uint32_t i = 0; i < js.joints.size(); i++) handles.push_back(js.handleOf(i));
            for (const uint64_t h : handles) {
                const uint32_t i = js.indexOf(h);
                const HJoint& j = js.joints[i];
                const uint8_t sa = st(j.bodyA), sb = j.bodyB == NO_BODY ? uint8_t(STATE_STATIC) : st(j.bodyB);
                const bool sleeping = sa == STATE_SLEEPING || sb == STATE_SLEEPING;
                const bool moves = sa == STATE_DYNAMIC || sb == STATE_DYNAMIC;
                const uint32_t g = sleeping ? JGROUP_SLEEPING : (moves ? JGROUP_ACTIVE : JGROUP_INACTIVE);
                if (js.groupOf(i) != g) js.moveToGroup(i, g);
            }
            const uint32_t begin = js.starts[JGROUP_ACTIVE], end = js.starts[JGROUP_UNUSED];
            std::fill(last.begin(), last.end(), 0u);
            std::vector<uint32_t> level(end - begin);
            uint32_t levels = 0;
            for (uint32_t i = begin; i < end; i++) {
                const HJoint& j = js.joints[i];
                uint32_t l = 0;
                if (st(j.bodyA) == STATE_DYNAMIC) l = std::max(l, last[j.bodyA]);
                if (j.bodyB != NO_BODY && st(j.bodyB) == STATE_DYNAMIC) l = std::max(l, last[j.bodyB]);
                level[i - begin] = ++l;
                if (st(j.bodyA) == STATE_DYNAMIC) last[j.bodyA] = l;
                if (j.bodyB != NO_BODY && st(j.bodyB) == STATE_DYNAMIC) last[j.bodyB] = l;
                levels = std::max(levels, l);
                if (k != JOINT_MOTOR) edges.push_back(make_uint2(j.bodyA, j.bodyB));
            }
            // Level-major order, dense order within a level.
            std::vector<uint32_t> start(levels + 2, 0);
            for (const uint32_t l : level) start[l + 1]++;
            for (uint32_t l = 1; l <= levels + 1; l++) start[l] += start[l - 1];
            std::vector<uint32_t> fill(start.begin(), start.end());
            std::vector<JointRec> recs(end - begin);
            for (uint32_t i = begin; i < end; i++) {
                const HJoint& j = js.joints[i];
                JointRec r{};
                r.bodyA = j.bodyA; r.bodyB = j.bodyB == NO_BODY ? j.bodyA : j.bodyB; r.index = i;
                r.ax = j.anchorAx; r.ay = j.anchorAy; r.bx = j.anchorBx; r.by = j.anchorBy;
                if (k == JOINT_SPRING) { r.p[0] = j.restLength; r.p[1] = j.stiffness; r.p[2] = j.damping; }
                else if (k == JOINT_REVOLUTE) { r.p[1] = j.stiffness; r.p[2] = j.damping; }
                else if (k == JOINT_MOTOR) { r.p[0] = j.targetSpeed; r.p[1] = j.maxTorque; }
                else {
                    r.p[0] = j.axisX; r.p[1] = j.axisY; r.p[2] = j.stiffness; r.p[3] = j.damping;
                    r.p[4] = j.lowerLimit; r.p[5] = j.upperLimit; r.p[6] = j.referenceAngle;
                    r.flags = j.enableLimit ? 1u : 0u;
                }
                recs[fill[level[i - begin]]++] = r;
            }
            jointActive[k] = end - begin;
            jointLevels[k] = levels;
            jointLevelHost[k].assign(start.begin() + 1, start.end());   // level l (from 1) starts at [l - 1]
            jointRec[k].upload(recs.data(), recs.size(), s);
            jointLevel[k].upload(jointLevelHost[k].data(), jointLevelHost[k].size(), s);
            jointData[k].reserve(std::max<size_t>(recs.size(), 1));
        }
        auto& motors = objects.jointSystems[JOINT_MOTOR].joints;
        std::vector<float> imp(motors.size());
        for (size_t i = 0; i < motors.size(); i++) imp[i] = motors[i].impulse;
        motorImpulse.upload(imp.data(), imp.size(), s);
        snapMotorImpulse.reserve(std::max<size_t>(imp.size(), 1));
        motorsOnDevice = uint32_t(imp.size());
        nJointEdges = uint32_t(edges.size());
        jointEdges.upload(edges.data(), edges.size(), s);
        CK(cudaStreamSynchronize(s));
    }
    void launchJoints()
    {
        JointLaunch L{};
        uint32_t maxIt = 0;
        for (uint32_t k = 0; k < JOINT_KINDS; k++) {
            L.rec[k] = jointRec[k].p;
            L.data[k] = jointData[k].p;
            L.levelStart[k] = jointLevel[k].p;
            L.count[k] = jointActive[k];
            L.levels[k] = jointLevels[k];
            L.iterations[k] = objects.jointSystems[k].iterations;
            if (jointActive[k]) maxIt = std::max(maxIt, L.iterations[k]);
        }
        L.maxIterations = maxIt;
        L.dt = settings.dt;
        L.motorImpulse = motorImpulse.p;
        k_joints<<<1, JOINT_THREADS, 0, stream>>>(view(), L);
        CK(cudaGetLastError());
        launches++;
    }

    // Collision events --------------------------------------------------------------------------------------
    // Colliders the world has: the host's (created worlds) or the device's (a world made by load_state).
    uint32_t colliderCount() const
    {
        return objects.colliders.empty() ? nColliders : uint32_t(objects.colliders.size());
    }
    ColliderEvent optIn(uint32_t c) const
    {
        if (!objects.colliders.empty()) return ColliderEvent{objects.colliders[c].callback, objects.colliders[c].eventThreshold};
        return c < loadedOptIn.size() ? loadedOptIn[c] : ColliderEvent{0u, 3.40282347e38f};
    }
    void setOptIn(uint32_t c, uint32_t id, float threshold)
    {
        if (!objects.colliders.empty()) {
            objects.colliders[c].callback = id;
            objects.colliders[c].eventThreshold = threshold;
        } else {
            if (loadedOptIn.size() < nColliders) loadedOptIn.resize(nColliders, ColliderEvent{0u, 3.40282347e38f});
            loadedOptIn[c] = ColliderEvent{id, threshold};
        }
        optInDirty = true;
    }
    // Uploads the colliders' opt-ins when they changed and sizes the ring (before a recording step).
    void prepareEvents()
    {
        if (optInDirty) {
            std::vector<ColliderEvent> v(nColliders);
            uint32_t with = 0;
            for (uint32_t c = 0; c < nColliders; c++) {
                v[c] = optIn(c);
                with += v[c].callback != 0u;
            }
            cevent.upload(v.data(), v.size(), stream);
            optInColliders = with;
            optInDirty = false;
        }
        if (eventCap == 0) {
            eventCap = 1024;
            eventRing.reserve(eventCap);
        }
    }
    void phaseEvents()
    {
        if (optInColliders == 0 || manifoldCap == 0) return;
        const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(gridFor(manifoldCap), 4 * dev.sms));
        k_collision_events<<<grid, 256, 0, stream>>>(view(), cevent.p, manifolds.p, nManifolds.p, manifoldCap,
                                                      eventRing.p, eventCap, dCounters.p);
        CK(cudaGetLastError());
        launches++;
    }
    // The step's events from the ring into lastEvents, in manifold order (side a first), with body handles.
    void collectEvents(uint32_t count)
    {
        std::vector<EventRecord> r(count);
        CK(cudaMemcpyAsync(r.data(), eventRing.p, sizeof(EventRecord) * count, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        std::sort(r.begin(), r.end(), [](const EventRecord& x, const EventRecord& y) {
            return x.manifold != y.manifold ? x.manifold < y.manifold : x.side < y.side;
        });
        auto handleOf = [&](uint32_t b) -> uint64_t {
            if (b >= objects.bodies.size()) return ~0ull;
            const uint32_t slot = objects.bodies[b].handleSlot;
            return (uint64_t(objects.slotGeneration[slot]) << 32) | slot;
        };
        lastEvents.resize(count);
        for (uint32_t k = 0; k < count; k++) {
            ag2d_collision_event& e = lastEvents[k];
            e.self = r[k].self; e.other = r[k].other;
            e.self_body = r[k].selfBody; e.other_body = r[k].otherBody;
            e.self_body_handle = handleOf(r[k].selfBody);
            e.other_body_handle = handleOf(r[k].otherBody);
            e.point_x = r[k].px; e.point_y = r[k].py; e.normal_x = r[k].nx; e.normal_y = r[k].ny;
            e.impulse = r[k].impulse;
            e.callback_id = uint16_t(r[k].callback);
            e.pad = 0;
        }
    }
    // CollisionCallbackManager::invoke over the step's events (Simulation::dispatchCollisionEvents,
    // Simulation.cpp:174-180): dead ids are skipped; the entry is read before the call, so a callback may create or
    // destroy callbacks.
    void dispatchEvents()
    {
        if (lastEvents.empty()) return;
        dispatching = true;
        struct Reset { bool& f; ~Reset() { f = false; } } reset{dispatching};
        const std::vector<ag2d_collision_event> events = lastEvents;
        for (const ag2d_collision_event& e : events) {
            const uint16_t id = e.callback_id;
            if (id == 0 || id >= callbacks.size() || !callbackAlive[id]) continue;
            const CallbackEntry entry = callbacks[id];
            entry.fn(&e, this, entry.user);
        }
    }

    void phaseSolve()
    {
        const cudaStream_t s = stream;
        CK(cudaMemsetAsync(bodyMax.p, 0, sizeof(unsigned long long) * std::max<uint32_t>(nBodies, 1), s));
        CK(cudaMemsetAsync(bodyMask.p, 0, sizeof(unsigned long long) * std::max<uint32_t>(nBodies, 1), s));
        CK(cudaMemsetAsync(bar.p, 0, 2 * sizeof(uint32_t), s));
        DeviceWorld w = view();
        Manifold* mm = manifolds.p;
        const uint32_t* nm = nManifolds.p;
        SolveScratch scratch{color.p, order.p, bodyMax.p, bodyMask.p, colorCount.p, colorStart.p, cons.p, nullptr,
                             listA.p, listB.p, pairBodies.p, hintsReady ? color.p : nullptr};
        hintsReady = false;
        uint32_t vi = settings.velocity_iterations, pi = settings.position_iterations;
        StepCounters* ctr = dCounters.p;
        pbegin(10);
        if (nWorlds > 1) {
            // One CTA per world over the world-grouped manifold list; the teams also link their islands
            // (phaseIslands then only decides sleep).
            CK(cudaMemsetAsync(nextWorld.p, 0, 2 * sizeof(uint32_t), s));
            k_island_init<<<gridFor(nBodies), 256, 0, s>>>(w, ufParent.p, ufFlag.p);
            islandsLinked = true;
            launches++;
            k_manifold_segments<<<gridFor(manifoldCap), 256, 0, s>>>(mm, nm, cbody.p, bodyWorld.p, nWorlds,
                                                                      manSeg.p);
            scratch.prio = prio.p;
            if (nBigTeams) {
                // Worlds larger than a team: their own wide CTAs on the side stream, overlapping the small teams.
                CK(cudaEventRecord(forkEvent, s));
                CK(cudaStreamWaitEvent(sideStream, forkEvent, 0));
                const TeamLaunch big{w, mm, manSeg.p, teamWorld.p, teamOrder.p + nTeams, nBigTeams, bigBodyCap,
                                     bigConsCap, scratch, vi, pi, nextWorld.p + 1, ctr, ufParent.p};
                CK(launch_color_solve_teams(bigThreads, bigPipelined, std::min(nBigTeams, bigBlocks), sideStream,
                                            big));
                launches++;
            }
            if (nTeams) {
                const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(nTeams, teamBlocks));
                const TeamLaunch args{w, mm, manSeg.p, teamWorld.p, teamOrder.p, nTeams, teamBodyCap, teamConsCap,
                                      scratch, vi, pi, nextWorld.p, ctr, ufParent.p};
                CK(launch_color_solve_teams(teamThreads, false, grid, s, args));
            }
            if (nBigTeams) {
                CK(cudaEventRecord(joinEvent, sideStream));
                CK(cudaStreamWaitEvent(s, joinEvent, 0));
            }
            launches++;
        } else if (lastManifolds <= GRID_SOLVE_THRESHOLD && dev.solveCluster > 1) {
            // One thread-block cluster, hardware barriers between colours.
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(dev.solveCluster);
            cfg.blockDim = dim3(SOLVE_CLUSTER_THREADS);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = dev.solveCluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            CK(cudaLaunchKernelEx(&cfg, k_color_solve_cluster, w, mm, nm, scratch, vi, pi, ctr));
        } else {
            // Whole-grid cooperative launch with the bounded software barrier.
            uint32_t* barp = bar.p;
            const uint32_t est = std::min<uint32_t>(manifoldCap, lastManifolds + lastManifolds / 2 + 1024);
            const int grid = std::max(1, std::min<int>(dev.coopSolveBlocks, int(div_up(est, 256))));
            void* args[] = {&w, &mm, &nm, &scratch, &vi, &pi, &barp, &ctr};
            CK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_color_solve_grid), dim3(grid), dim3(256), args,
                                           0, s));
        }
        pend(10);
        launches++;
    }

    void phaseIslands()
    {
        const cudaStream_t s = stream;
        const DeviceWorld w = view();
        pbegin(11);
        launches += islandsLinked ? 2 : 4;
        if (!islandsLinked) {
            k_island_init<<<gridFor(nBodies), 256, 0, s>>>(w, ufParent.p, ufFlag.p);
            k_island_union<<<gridFor(manifoldCap), 256, 0, s>>>(w, manifolds.p, nManifolds.p, ufParent.p);
        }
        if (nJointEdges) {   // after the teams' links too: union-find links in any order
            k_island_union_edges<<<gridFor(nJointEdges), 256, 0, s>>>(w, jointEdges.p, nJointEdges, ufParent.p);
            launches++;
        }
        islandsLinked = false;
        k_island_quiet<<<gridFor(nBodies), 256, 0, s>>>(w, ufParent.p, ufFlag.p, settings.dt, settings.sleep_speed,
                                                        settings.sleep_time);
        k_island_sleep<<<gridFor(nBodies), 256, 0, s>>>(w, ufParent.p, ufFlag.p, dCounters.p);
        CK(cudaGetLastError());
        pend(11);
    }

    void readCounters()
    {
        CK(cudaMemcpyAsync(hCounters, dCounters.p, sizeof(StepCounters), cudaMemcpyDeviceToHost, stream));
        const auto t0 = std::chrono::steady_clock::now();
        CK(cudaStreamSynchronize(stream));
        syncMs += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        pcollect();
    }

    static uint32_t scanLaunches(uint32_t) { return 1; }   // one k_scan per scan

    // Device milliseconds per step of one timed phase over 'steps' real steps.
    double timePhase(int phase, uint32_t steps)
    {
        phaseMs[phase] = 0.0;
        phaseCalls[phase] = 0;
        for (uint32_t i = 0; i < steps; i++) stepOnce();
        return phaseCalls[phase] ? phaseMs[phase] / double(phaseCalls[phase]) : 0.0;
    }

    // Launch-shape autotuner: times real steps under each candidate and keeps the fastest, one setting at a time
    // (solver team size for batches, then the pair-query and narrow-phase block sizes). The results of a step do not
    // depend on these settings, so tuning on the live world only advances it: one step, then per candidate one
    // settling step and stepsPer timed steps.
    void autotune(uint32_t stepsPer, ag2d_tuning& out)
    {
        const bool wasProfiling = profiling;
        profiling = true;
        stepOnce();   // first step: uploads, list build, buffer growth
        // Candidates are timed in interleaved rounds, so that all of them see the same stretch of the simulation
        // (the load changes from step to step); each first runs one untimed step (first launches load code).
        auto pick = [&](int phase, const std::vector<uint32_t>& cands, auto apply) {
            std::vector<double> total(cands.size(), 0.0);
            const bool log = std::getenv("AG2D_TUNE_LOG") != nullptr;   // per-candidate times on stderr
            for (uint32_t c : cands) {
                if (log) std::fprintf(stderr, "ag2d autotune phase %d trying %u\n", phase, c);
                apply(c);
                stepOnce();
            }
            for (uint32_t r = 0; r < stepsPer; r++)
                for (size_t k = 0; k < cands.size(); k++) {
                    apply(cands[k]);
                    total[k] += timePhase(phase, 1);
                }
            size_t best = 0;
            for (size_t k = 0; k < cands.size(); k++) {
                if (log) std::fprintf(stderr, "ag2d autotune phase %d candidate %u: %.4f ms\n", phase, cands[k],
                                      total[k] / stepsPer);
                if (total[k] < total[best]) best = k;
            }
            apply(cands[best]);
            return std::make_pair(cands[best], total[best] / stepsPer);
        };
        out.team_colliders = 0;
        out.team_threads = 0;
        out.big_team_mode = bigMode();
        out.team_cons_on_chip = consOnChip ? 1 : 0;
        out.solve_ms = 0.0f;
        if (nWorlds > 1) {
            // (colliders per team, threads per CTA, constraint records on chip), packed as
            // colliders << 16 | on-chip << 15 | threads.
            std::vector<uint32_t> cands;
            for (uint32_t t : {256u << 16 | 64, 512u << 16 | 64, 512u << 16 | 128, 1024u << 16 | 128,
                               1024u << 16 | 256, 2048u << 16 | 256, 2048u << 16 | 512})
                cands.push_back(t);
            // On chip: smaller teams, so that their records fit and several CTAs share an SM.
            for (uint32_t t : {128u << 16 | 64, 256u << 16 | 64, 256u << 16 | 128, 512u << 16 | 128,
                               512u << 16 | 256, 1024u << 16 | 256})
                cands.push_back(t | 1u << 15);
            const auto r = pick(10, cands, [&](uint32_t t) {
                consOnChip = (t >> 15) & 1;
                setTeams(t >> 16, t & 0x7FFF);
            });
            out.team_colliders = r.first >> 16;
            out.team_threads = r.first & 0x7FFF;
            out.team_cons_on_chip = (r.first >> 15) & 1;
            out.solve_ms = float(r.second);
            // Worlds larger than a team: CTA size and pipelined passes (modes 0-3, big_team_mode).
            if (nBigTeams) {
                const auto rb = pick(10, {0u, 1u, 2u, 3u}, [&](uint32_t mode) { setBigMode(mode); });
                out.big_team_mode = rb.first;
                out.solve_ms = float(rb.second);
            }
        }
        const auto q = pick(4, {64, 128, 256}, [&](uint32_t t) { queryThreads = t; });
        out.query_threads = q.first;
        out.query_ms = float(q.second);
        const auto nr = pick(5, {128, 256, 512}, [&](uint32_t t) { narrowThreads = t; });
        out.narrow_threads = nr.first;
        out.narrow_ms = float(nr.second);
        profiling = wasProfiling;
        for (int p = 0; p < NPHASE; p++) { phaseMs[p] = 0.0; phaseCalls[p] = 0; evPending[p] = false; }
    }

    // Applies the queued body commands to the device state, in call order, as ObjectManager::applyCommand does to
    // the reference's SoA (ObjectManager.cpp:662-790): every command but a stale one wakes the body's sleeping
    // island first (wakeBody, :1425-1436); a position is given for the body origin and moves the centre of mass
    // with the rotated local centre of mass; a rotation is wrapped into [0, 2 pi) with std::cos / std::sin of it
    // stored; a mass of 0 makes the body static (velocities zeroed), a positive one scales the inertia by
    // new / old mass; an inertia is ignored on a static body; a destroyed body leaves every work list and tree and
    // its handle goes stale. Body dense indices do not move (the reference's group moves are state flags here).
    // The next step then rebuilds the work lists and the static tree and poses every collider (spatialDirty).
    void flushCommands()
    {
        if (commands.empty() && jointCommands.empty()) return;
        if (nWorlds > 1) { commands.clear(); throw ApiError(AG2D_ERR_UNSUPPORTED, "body commands are per world"); }
        ensureUploaded();
        const cudaStream_t s = stream;
        std::vector<float4> vel = download(bvel.p, nBodies, s), pos = download(bpos.p, nBodies, s);
        std::vector<float2> rot = download(brot.p, nBodies, s);
        std::vector<uint8_t> state = download(bstate.p, nBodies, s);
        std::vector<float> timer = download(sleepTimer.p, nBodies, s), wraps = download(wrapCount.p, nBodies, s);
        const std::vector<uint32_t> island = download(sleepIsland.p, nBodies, s);
        HostObjects& o = objects;
        std::vector<uint32_t> wokenRoots;   // islands woken, in waking order
        auto wakeIsland = [&](uint32_t root) {   // every sleeping body of the island (k_wake_apply's rule)
            bool any = false;
            for (uint32_t i = 0; i < nBodies; i++)
                if (state[i] == STATE_SLEEPING && island[i] == root) { state[i] = STATE_DYNAMIC; timer[i] = 0.0f; any = true; }
            if (any) wokenRoots.push_back(root);
        };
        auto wake = [&](uint32_t b) {
            if (state[b] == STATE_SLEEPING) wakeIsland(island[b]);
        };
        // Static bodies whose pose, mass or existence a command changes (ObjectManager::applyCommand,
        // ObjectManager.cpp:678-687, and destroyColliderInternal): their colliders count as edited.
        std::vector<uint8_t> editedBody(nBodies, 0);
        bool anyEdited = false;
        // applyBodyMass (ObjectManager.cpp:867-905).
        auto applyMass = [&](uint32_t b, float m) {
            HBody& hb = o.bodies[b];
            const float newMass = std::fmax(0.0f, m);
            const float oldMass = hb.mass;
            if (newMass > 0.0f) {
                float inertia = hb.inertia;
                if (oldMass > 0.0f) inertia *= newMass / oldMass;
                hb.mass = newMass;
                hb.invMass = 1.0f / newMass;
                hb.inertia = inertia;
                hb.invInertia = inertia > 0.0f ? 1.0f / inertia : 0.0f;
                if (state[b] == STATE_STATIC) { state[b] = STATE_DYNAMIC; timer[b] = 0.0f; }
            } else {
                hb.mass = 0.0f; hb.invMass = 0.0f; hb.inertia = 0.0f; hb.invInertia = 0.0f;
                vel[b].x = 0.0f; vel[b].y = 0.0f; vel[b].z = 0.0f;
                state[b] = STATE_STATIC;
            }
            vel[b].w = hb.invMass;
            pos[b].w = hb.invInertia;
        };
        std::vector<uint32_t> editedColliders, reachBodies;   // device collider records and bound radii to refresh
        bool polygonsEdited = false;                          // the packed polygon tables need a new upload
        const float twoPi = float(3.14159265358979323846 * 2.0);
        auto wrap = [&](float r) { r = std::fmod(r, twoPi); if (r < 0.0f) r += twoPi; return r; };
        for (const BodyCommand& c : commands) {
            const bool colliderCmd = c.kind >= AG2D_COMMAND_COLLIDER_OFFSET && c.kind <= AG2D_COMMAND_POLYGON_SHAPE;
            const uint32_t ci = colliderCmd ? uint32_t(c.handle) : 0xFFFFFFFFu;
            if (colliderCmd && ci >= o.colliders.size()) continue;
            const uint32_t b = colliderCmd ? o.colliders[ci].body : o.indexOf(c.handle);
            if (b >= nBodies || b >= o.bodies.size() || state[b] == STATE_DESTROYED) continue;
            HBody& hb = o.bodies[b];
            if (state[b] == STATE_STATIC &&
                (colliderCmd || c.kind == AG2D_COMMAND_DESTROY || c.kind == AG2D_COMMAND_POSITION ||
                 c.kind == AG2D_COMMAND_ROTATION || c.kind == AG2D_COMMAND_MASS ||
                 c.kind == AG2D_COMMAND_LOCAL_CENTER_OF_MASS || c.kind == AG2D_COMMAND_MASS_FROM_DENSITY)) {
                editedBody[b] = 1;   // markStaticColliderEdited
                anyEdited = true;
            }
            wake(b);
            if (colliderCmd) {   // ObjectManager::applyCommand's collider branch (ObjectManager.cpp:785-852)
                HCollider& k = o.colliders[ci];
                bool shapeEdit = false;
                switch (c.kind) {
                case AG2D_COMMAND_COLLIDER_OFFSET:
                    k.locX = c.a; k.locY = c.b;
                    k.comOffX = k.locX - hb.lcomX; k.comOffY = k.locY - hb.lcomY;
                    break;
                case AG2D_COMMAND_COLLIDER_ROTATION: k.localRot = wrap(c.a); break;
                case AG2D_COMMAND_COLLIDER_MATERIAL: {
                    const float idx = c.a;
                    k.material = (idx >= 0.0f && idx < float(o.materialCount())) ? uint32_t(idx) : 0u;
                    break;
                }
                case AG2D_COMMAND_CIRCLE_RADIUS:
                    if (k.type != SHAPE_CIRCLE) break;
                    o.circleRadius[k.shape] = std::fmax(0.0f, c.a);
                    k.minExtent = k.maxExtent = o.circleRadius[k.shape];
                    shapeEdit = true;
                    break;
                case AG2D_COMMAND_BOX_SIZE:
                    if (k.type != SHAPE_BOX) break;
                    o.boxHalfW[k.shape] = std::fmax(0.0f, c.a) * 0.5f;
                    o.boxHalfH[k.shape] = std::fmax(0.0f, c.b) * 0.5f;
                    k.minExtent = std::fmin(o.boxHalfW[k.shape], o.boxHalfH[k.shape]);
                    k.maxExtent = std::fmax(o.boxHalfW[k.shape], o.boxHalfH[k.shape]);
                    shapeEdit = true;
                    break;
                case AG2D_COMMAND_CAPSULE_SHAPE:
                    if (k.type != SHAPE_CAPSULE) break;
                    o.boxHalfW[k.shape] = std::fmax(0.0f, c.a) * 0.5f;
                    o.boxHalfH[k.shape] = std::fmax(0.0f, c.b);
                    k.minExtent = o.boxHalfH[k.shape];
                    k.maxExtent = o.boxHalfW[k.shape] + o.boxHalfH[k.shape];
                    shapeEdit = true;
                    break;
                case AG2D_COMMAND_POLYGON_SHAPE: {   // ObjectManager.cpp:838-857: recentred on its centroid
                    if (k.type != SHAPE_POLYGON || c.slot >= pendingPolygons.size()) break;
                    std::vector<float> v = pendingPolygons[c.slot];
                    float unused = 0.0f, cx = 0.0f, cy = 0.0f;
                    polygon_inertia(1.0f, v, unused, cx, cy);
                    for (size_t i = 0; i < v.size() / 2; i++) { v[2 * i] -= cx; v[2 * i + 1] -= cy; }
                    const float cosL = std::cos(k.localRot), sinL = std::sin(k.localRot);
                    k.locX += cosL * cx - sinL * cy;
                    k.locY += sinL * cx + cosL * cy;
                    k.comOffX = k.locX - hb.lcomX; k.comOffY = k.locY - hb.lcomY;
                    HPolygon& poly = o.polygons[k.shape];
                    poly.verts = v;
                    poly.normals = polygon_normals(v);
                    float inR = FLT_MAX, outR2 = 0.0f;
                    for (size_t i = 0; i < v.size() / 2; i++) {
                        const float vx = poly.verts[2 * i], vy = poly.verts[2 * i + 1];
                        inR = std::fmin(inR, poly.normals[2 * i] * vx + poly.normals[2 * i + 1] * vy);
                        outR2 = std::fmax(outR2, vx * vx + vy * vy);
                    }
                    k.minExtent = std::fmax(inR, 0.0f);
                    k.maxExtent = std::sqrt(outR2);
                    polygonsEdited = true;
                    break;
                }
                default: break;
                }
                (void)shapeEdit;
                editedColliders.push_back(ci);
                reachBodies.push_back(b);
                continue;
            }
            switch (c.kind) {
            case AG2D_COMMAND_DESTROY:
                state[b] = STATE_DESTROYED;
                o.slotGeneration[uint32_t(c.handle & 0xFFFFFFFFu)]++;
                // Its constraints go with it, waking their other bodies (ObjectManager.cpp:400-410, 502-520).
                for (JointSystem& js : o.jointSystems) {
                    std::vector<uint64_t> doomed;
                    for (uint32_t i = 0; i < js.joints.size(); i++)
                        if (js.joints[i].bodyA == b || js.joints[i].bodyB == b) doomed.push_back(js.handleOf(i));
                    if (doomed.empty()) continue;
                    beforeJointEdit();
                    for (const uint64_t h : doomed) {
                        const uint32_t i = js.indexOf(h);
                        const uint32_t other = js.joints[i].bodyA == b ? js.joints[i].bodyB : js.joints[i].bodyA;
                        if (other != NO_BODY && other < nBodies) wake(other);
                        js.destroy(i);
                    }
                }
                break;
            case AG2D_COMMAND_POSITION: {
                const float r = pos[b].z, cosR = std::cos(r), sinR = std::sin(r);
                pos[b].x = c.a + cosR * hb.lcomX - sinR * hb.lcomY;
                pos[b].y = c.b + sinR * hb.lcomX + cosR * hb.lcomY;
                break;
            }
            case AG2D_COMMAND_ROTATION: {
                const float twoPi = float(3.14159265358979323846 * 2.0);
                float r = std::fmod(c.a, twoPi);
                if (r < 0.0f) r += twoPi;
                pos[b].z = r;
                rot[b] = make_float2(std::cos(r), std::sin(r));
                wraps[b] = 0.0f;
                break;
            }
            case AG2D_COMMAND_VELOCITY: vel[b].x = c.a; vel[b].y = c.b; break;
            case AG2D_COMMAND_ANGULAR_VELOCITY: vel[b].z = c.a; break;
            case AG2D_COMMAND_MASS: applyMass(b, c.a); break;
            case AG2D_COMMAND_LOCAL_CENTER_OF_MASS: {   // ObjectManager.cpp:751-771: the origin stays put
                const float r = pos[b].z, cosR = std::cos(r), sinR = std::sin(r);
                const float dx = c.a - hb.lcomX, dy = c.b - hb.lcomY;
                pos[b].x += cosR * dx - sinR * dy;
                pos[b].y += sinR * dx + cosR * dy;
                hb.lcomX = c.a;
                hb.lcomY = c.b;
                for (const uint32_t k : hb.colliders) {
                    o.colliders[k].comOffX = o.colliders[k].locX - hb.lcomX;
                    o.colliders[k].comOffY = o.colliders[k].locY - hb.lcomY;
                    editedColliders.push_back(k);
                }
                reachBodies.push_back(b);
                break;
            }
            case AG2D_COMMAND_RECOMPUTE_INERTIA: {   // ObjectManager.cpp:917-970
                const float mass = hb.mass;
                if (mass <= 0.0f) break;
                float totalArea = 0.0f;
                for (const uint32_t k : hb.colliders) totalArea += o.colliderArea(k);
                if (totalArea <= 0.0f) break;
                const float massPerArea = mass / totalArea;
                float inertia = 0.0f;
                for (const uint32_t k : hb.colliders) {
                    const float area = o.colliderArea(k);
                    if (area <= 0.0f) continue;
                    const float m = massPerArea * area;
                    const float dx = o.colliders[k].comOffX, dy = o.colliders[k].comOffY;
                    inertia += o.colliderOwnInertia(k, m) + m * (dx * dx + dy * dy);
                }
                hb.inertia = inertia;
                hb.invInertia = inertia > 0.0f ? 1.0f / inertia : 0.0f;
                pos[b].w = hb.invInertia;
                break;
            }
            case AG2D_COMMAND_MASS_FROM_DENSITY: {   // ObjectManager.cpp:907-915
                float totalArea = 0.0f;
                for (const uint32_t k : hb.colliders) totalArea += o.colliderArea(k);
                if (totalArea <= 0.0f) break;
                applyMass(b, std::fmax(0.0f, c.a) * totalArea);
                break;
            }
            case AG2D_COMMAND_INERTIA: {
                if (hb.invMass == 0.0f) break;
                const float inertia = std::fmax(0.0f, c.a);
                hb.inertia = inertia;
                hb.invInertia = inertia > 0.0f ? 1.0f / inertia : 0.0f;
                pos[b].w = hb.invInertia;
                break;
            }
            default: break;
            }
        }
        commands.clear();
        pendingPolygons.clear();
        if (polygonsEdited) {   // vertex counts may change: the packed tables are rebuilt whole
            std::vector<uint32_t> po, pc;
            std::vector<float2> pv, pn;
            for (const HPolygon& p : o.polygons) {
                po.push_back(uint32_t(pv.size()));
                pc.push_back(uint32_t(p.verts.size() / 2));
                for (size_t k = 0; k < p.verts.size() / 2; k++) {
                    pv.push_back(make_float2(p.verts[2 * k], p.verts[2 * k + 1]));
                    pn.push_back(make_float2(p.normals[2 * k], p.normals[2 * k + 1]));
                }
            }
            polyOffset.upload(po.data(), po.size(), s); polyCount.upload(pc.data(), pc.size(), s);
            polyVerts.upload(pv.data(), pv.size(), s); polyNormals.upload(pn.data(), pn.size(), s);
            nPolyVerts = uint32_t(pv.size());
            CK(cudaStreamSynchronize(s));
        }
        // Collider records and shape parameters the commands changed, and the bound radii that follow.
        for (const uint32_t k : editedColliders) {
            const HCollider& hc = o.colliders[k];
            const float4 off = make_float4(hc.comOffX, hc.comOffY, hc.localRot, 0.0f);
            CK(cudaMemcpyAsync(coff.p + k, &off, sizeof(float4), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(cmat.p + k, &hc.material, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(minExtent.p + k, &hc.minExtent, sizeof(float), cudaMemcpyHostToDevice, s));
            if (hc.type == SHAPE_CIRCLE)
                CK(cudaMemcpyAsync(circleRadius.p + hc.shape, &o.circleRadius[hc.shape], sizeof(float),
                                   cudaMemcpyHostToDevice, s));
            else if (hc.type == SHAPE_BOX || hc.type == SHAPE_CAPSULE) {
                const float2 h = make_float2(o.boxHalfW[hc.shape], o.boxHalfH[hc.shape]);
                CK(cudaMemcpyAsync(boxHalf.p + hc.shape, &h, sizeof(float2), cudaMemcpyHostToDevice, s));
            }
            CK(cudaStreamSynchronize(s));   // the sources are this loop's locals
        }
        for (const uint32_t b : reachBodies) {
            o.bodies[b].boundRadius = o.boundRadiusOf(b);
            CK(cudaMemcpyAsync(boundRadius.p + b, &o.bodies[b].boundRadius, sizeof(float), cudaMemcpyHostToDevice, s));
        }
        // Constraint destroys and edits (ConstraintSystemBase::flushImpl, ConstraintSystemBase.h:127-142, and the
        // systems' flushCommands): stale handles are dropped; the constraint's bodies wake.
        for (const JointCommand& c : jointCommands) {
            JointSystem& js = o.jointSystems[c.kind];
            const uint32_t i = js.indexOf(c.handle);
            if (i == NO_BODY) continue;
            beforeJointEdit();
            HJoint& j = js.joints[i];
            if (j.bodyA < nBodies) wake(j.bodyA);
            if (j.bodyB != NO_BODY && j.bodyB < nBodies) wake(j.bodyB);
            switch (c.field) {
            case -1: js.destroy(i); break;
            case AG2D_JOINT_ANCHOR_A: j.anchorAx = c.a; j.anchorAy = c.b; break;
            case AG2D_JOINT_ANCHOR_B: j.anchorBx = c.a; j.anchorBy = c.b; break;
            case AG2D_JOINT_REST_LENGTH: j.restLength = std::fmax(0.0f, c.a); break;
            case AG2D_JOINT_STIFFNESS: j.stiffness = std::fmax(0.0f, c.a); break;
            case AG2D_JOINT_DAMPING: j.damping = std::fmax(0.0f, c.a); break;
            case AG2D_JOINT_TARGET_SPEED: j.targetSpeed = c.a; break;
            case AG2D_JOINT_MAX_TORQUE: j.maxTorque = std::fmax(0.0f, c.a); break;
            case AG2D_JOINT_AXIS_A: {
                float x = c.a, y = c.b;
                if (normalize_axis(x, y)) { j.axisX = x; j.axisY = y; }
                break;
            }
            case AG2D_JOINT_LIMITS: j.lowerLimit = std::fmin(c.a, c.b); j.upperLimit = std::fmax(c.a, c.b); break;
            case AG2D_JOINT_ENABLE_LIMIT: j.enableLimit = c.a != 0.0f; break;
            case AG2D_JOINT_RESET_REFERENCE_ANGLE:
                if (j.bodyB != NO_BODY && j.bodyA < nBodies && j.bodyB < nBodies)
                    j.referenceAngle = reference_angle(pos[j.bodyA].z, pos[j.bodyB].z);
                break;
            default: break;
            }
        }
        jointCommands.clear();
        if (jointTotal()) jointsDirty = true;   // body states may have changed: constraint groups with them
        restoreWokenIslands(state, timer, island, wokenRoots, editedBody, anyEdited);
        if (nBodies) {
            CK(cudaMemcpyAsync(bvel.p, vel.data(), nBodies * sizeof(float4), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(bpos.p, pos.data(), nBodies * sizeof(float4), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(brot.p, rot.data(), nBodies * sizeof(float2), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(bstate.p, state.data(), nBodies, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(sleepTimer.p, timer.data(), nBodies * sizeof(float), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(wrapCount.p, wraps.data(), nBodies * sizeof(float), cudaMemcpyHostToDevice, s));
            CK(cudaStreamSynchronize(s));
        }
        nStatic = uint32_t(std::count(state.begin(), state.end(), uint8_t(STATE_STATIC)));
        nDestroyed = uint32_t(std::count(state.begin(), state.end(), uint8_t(STATE_DESTROYED)));
        listsDirty = true;
        otherDirty = true;
        fullPose = true;
    }

    // The command path's part of Simulation::flushCommands (Simulation.cpp:454-461): islands touching an edited
    // static body wake (wakeIslandsOfEditedStatics, :463-483, with takeContactsOfColliders,
    // NarrowPhaseCollisionDetector.cpp:415-456: their stored manifolds with an edited collider are dropped, awake
    // bodies touching one restart their sleep timers), then the stored manifolds of every woken island join the
    // warm-start list (wakeContactData, :338-412; none of their pairs can be in that list, so all are appended). A
    // single world, on the host: body commands are rare.
    void restoreWokenIslands(std::vector<uint8_t>& state, std::vector<float>& timer, const std::vector<uint32_t>& island,
                             std::vector<uint32_t>& wokenRoots, const std::vector<uint8_t>& editedBody, bool anyEdited)
    {
        const cudaStream_t s = stream;
        compactPrev();
        uint32_t counts[2] = {0, 0};
        CK(cudaMemcpyAsync(counts, nIsle.p, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(counts + 1, nPrev.p, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const uint32_t ni = counts[0], np = counts[1];
        if (ni == 0 && !anyEdited) return;
        std::vector<Manifold> store = download(isle.p, ni, s), prev = download(prevManifolds.p, np, s);
        std::vector<uint32_t> storeId = download(isleId.p, ni, s), prevCol = download(prevColor.p, np, s);
        const std::vector<uint32_t> owner = download(cbody.p, nColliders, s);
        auto edited = [&](uint32_t c) { return c < nColliders && editedBody[owner[c]] != 0; };
        std::vector<uint8_t> drop(ni, 0);
        if (anyEdited) {
            std::vector<uint32_t> hit;   // islands with a stored manifold on an edited collider, in island order
            for (uint32_t r = 0; r < ni; r++) {
                if (!edited(store[r].a) && !edited(store[r].b)) continue;
                drop[r] = 1;
                if (std::find(hit.begin(), hit.end(), storeId[r]) == hit.end()) hit.push_back(storeId[r]);
            }
            std::sort(hit.begin(), hit.end());
            for (uint32_t root : hit) {
                bool any = false;
                for (uint32_t i = 0; i < nBodies; i++)
                    if (state[i] == STATE_SLEEPING && island[i] == root) { state[i] = STATE_DYNAMIC; timer[i] = 0.0f; any = true; }
                if (any) wokenRoots.push_back(root);
            }
            for (const Manifold& m : prev) {
                const bool eA = edited(m.a), eB = edited(m.b);
                if (eA == eB) continue;
                const uint32_t partner = owner[eA ? m.b : m.a];
                if (state[partner] == STATE_DYNAMIC) timer[partner] = 0.0f;
            }
        }
        // Woken islands' records (colliders alive) in island order, first record of a pair only.
        std::vector<uint8_t> woken(nBodies, 0);
        for (uint32_t root : wokenRoots) if (root < nBodies) woken[root] = 1;
        auto alive = [&](uint32_t c) { return c < nColliders && state[owner[c]] != STATE_DESTROYED; };
        std::vector<unsigned long long> keys;
        bool storeChanged = anyEdited;
        for (uint32_t root : wokenRoots) {
            for (uint32_t r = 0; r < ni; r++) {
                if (drop[r] || storeId[r] != root) continue;
                drop[r] = 1;
                storeChanged = true;
                const Manifold& m = store[r];
                if (!alive(m.a) || !alive(m.b)) continue;
                const unsigned long long key = (uint64_t(std::min(m.a, m.b)) << 32) | std::max(m.a, m.b);
                if (std::find(keys.begin(), keys.end(), key) != keys.end()) continue;
                keys.push_back(key);
                prev.push_back(m);
                prevCol.push_back(NO_COLOR);
            }
        }
        if (!storeChanged) return;
        std::vector<Manifold> keptRec;
        std::vector<uint32_t> keptId;
        for (uint32_t r = 0; r < ni; r++)
            if (!drop[r]) { keptRec.push_back(store[r]); keptId.push_back(storeId[r]); }
        const uint32_t nk = uint32_t(keptRec.size()), nnp = uint32_t(prev.size());
        if (nnp > manifoldCap) reserveCapacities(std::max(nnp, pairCap), nnp);
        if (nk) {
            CK(cudaMemcpyAsync(isle.p, keptRec.data(), nk * sizeof(Manifold), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(isleId.p, keptId.data(), nk * 4, cudaMemcpyHostToDevice, s));
        }
        if (nnp) {
            CK(cudaMemcpyAsync(prevManifolds.p, prev.data(), nnp * sizeof(Manifold), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(prevColor.p, prevCol.data(), nnp * 4, cudaMemcpyHostToDevice, s));
        }
        CK(cudaMemcpyAsync(nIsle.p, &nk, 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(nPrev.p, &nnp, 4, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
        isleUpper = nk;
        prevCount = nnp;
        prevSegValid = false;
    }

    // One fixed step (Simulation::physicsStep order, Simulation.cpp:255-351).
    void stepOnce()
    {
        const auto tStart = std::chrono::steady_clock::now();
        struct HostTimer {
            double& acc;
            std::chrono::steady_clock::time_point t0;
            ~HostTimer() { acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
        } hostTimer{hostMs, tStart};
        ensureUploaded();
        flushCommands();
        if (jointsDirty) rebuildJoints();
        // BodyCollisionSolver::resetCollisionData and setCollisionEventRecording (Simulation.cpp:261-266).
        lastEvents.clear();
        recording = eventsEnabled && callbacksAlive > 0 && nWorlds <= 1;
        if (recording) prepareEvents();
        for (int attempt = 0; attempt < 8; attempt++) {
            if (attempt > 0) retries++;
            if (listsDirty) rebuildLists();
            const cudaStream_t s = stream;
            CK(cudaMemsetAsync(dCounters.p, 0, sizeof(StepCounters), s));
            CK(cudaMemcpyAsync(&dCounters.p->stored, nIsle.p, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
            snapshot(false);
            if (settings.ccd && nColliders) {
                // The poses continuous collision sweeps from; a retried step starts again from the same poses.
                if (attempt == 0)
                    CK(cudaMemcpyAsync(prevPose.p, cpose.p, sizeof(float4) * nColliders, cudaMemcpyDeviceToDevice, s));
                else
                    CK(cudaMemcpyAsync(cpose.p, prevPose.p, sizeof(float4) * nColliders, cudaMemcpyDeviceToDevice, s));
            }
            const bool fullPoseThisStep = fullPose;
            const bool otherDirtyThisStep = otherDirty;
            CK(cudaMemsetAsync(wrapCount.p, 0, sizeof(float) * std::max<uint32_t>(nBodies, 1), s));   // preUpdate
            phaseIntegrate();
            phasePose(fullPose);
            if (newWorldsPending && !fullPose) {
                // Worlds that joined a server batch: their first step poses every collider, as alone.
                const DeviceWorld wv = view();
                k_collider_pose<<<gridFor(nColliders), 256, 0, s>>>(wv, nullptr, nullptr, nColliders,
                                                                    nWorlds > 1 ? newWorldMask.p : nullptr);
                CK(cudaGetLastError());
                launches++;
            }
            if (settings.ccd) phaseCcd();
            phaseBroad();
            phaseNarrow();
            phaseWake();
            phaseRestore();
            if (recording) phaseEvents();
            phaseSolve();
            phaseIslands();
            readCounters();
            const uint32_t st = hCounters->status;
            if (st & STATUS_EVENT_OVERFLOW) {
                // The ring was too small for this step's events: grow it and step again from the saved state.
                snapshot(true);
                if (nWorlds > 1) CK(cudaMemsetAsync(worldDirty.p, 0, sizeof(uint32_t) * nWorlds, s));
                fullPose = fullPoseThisStep;
                otherDirty = true;
                eventCap = std::max<uint32_t>(2 * hCounters->events, 2 * eventCap);
                eventRing.reserve(eventCap);
                regrows++;
                CK(cudaStreamSynchronize(s));
                if (!(st & (STATUS_PAIR_OVERFLOW | STATUS_MANIFOLD_OVERFLOW))) continue;
            }
            if (st & (STATUS_PAIR_OVERFLOW | STATUS_MANIFOLD_OVERFLOW)) {
                snapshot(true);
                if (nWorlds > 1) CK(cudaMemsetAsync(worldDirty.p, 0, sizeof(uint32_t) * nWorlds, s));
                fullPose = fullPoseThisStep;
                otherDirty = true;
                (void)otherDirtyThisStep;
                const uint64_t needP = std::max<uint64_t>(hCounters->pairs, pairCap) * 2;
                const uint64_t needM = std::max<uint64_t>(hCounters->manifolds, manifoldCap) * 2;
                if (needP > (1ull << 30)) throw ApiError(AG2D_ERR_CAPACITY, "pair buffer would exceed 2^30 entries");
                reserveCapacities(uint32_t(needP), uint32_t(std::min<uint64_t>(needM, needP)));
                CK(cudaStreamSynchronize(s));
                continue;
            }
            if (st & (STATUS_BARRIER_TIMEOUT | STATUS_LOOKBACK_TIMEOUT)) {
                snapshot(true);
                CK(cudaStreamSynchronize(s));
                throw ApiError(AG2D_ERR_TIMEOUT, "a bounded device-side wait timed out (status " + std::to_string(st) + ")");
            }
            if (st & (STATUS_COLOR_OVERFLOW | STATUS_HASH_FULL | STATUS_STACK_OVERFLOW)) {
                snapshot(true);
                CK(cudaStreamSynchronize(s));
                throw ApiError(AG2D_ERR_CAPACITY, "capacity limit (colours, hash or traversal stack), status " + std::to_string(st));
            }
            fullPose = false;
            aabbValid = true;
            // The solved manifolds become the next step's warm-start source.
            swap_bufs(manifolds, prevManifolds);
            swap_bufs(color, prevColor);   // this step's colours: next step's hints
            newWorldsPending = false;
            manSegFresh = nWorlds > 1;
            CK(cudaMemcpyAsync(nPrev.p, nManifolds.p, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
            if (nWorlds > 1) {   // the solve's world starts describe the list that is now the warm-start list
                prevSeg.reserve(nWorlds + 1);
                CK(cudaMemcpyAsync(prevSeg.p, manSeg.p, (size_t(nWorlds) + 1) * sizeof(uint32_t),
                                   cudaMemcpyDeviceToDevice, s));
                prevSegValid = true;
            }
            lastManifolds = hCounters->manifolds;
            lastPairs = hCounters->pairs;
            prevCount = std::min(lastManifolds, manifoldCap);
            // The store as the step began (the restore reads it, the sleep pass rewrites it).
            isleUpper = hCounters->stored;
            prevHoldsSleepers = false;   // the list is this step's
            {
                // Records leave the store when their island woke (staged by the restore) or a collider is gone.
                const bool removals = hCounters->staged > 0 || (nDestroyed > 0 && hCounters->stored > 0);
                if (hCounters->slept || removals) phaseSleepStore(hCounters->stored, hCounters->slept > 0, removals);
            }
            if (hCounters->topoDirty && jointTotal()) jointsDirty = true;   // constraints change group
            if (hCounters->topoDirty) {
                // Woken or slept bodies: refresh the poses of every collider at the post-step state (the reference
                // rebuilds its spatial data in postUpdate, Simulation.cpp:640-647), then the work lists and the
                // static + sleeping tree before the next step.
                listsDirty = true;
                otherDirty = true;
                phasePose(true, true);
                if (nWorlds > 1) CK(cudaMemsetAsync(worldDirty.p, 0, sizeof(uint32_t) * nWorlds, s));
                rebuildLists();
            }
            // Grow ahead of need, geometrically (a reallocation synchronises the device).
            if (hCounters->pairs > pairCap / 2 || hCounters->manifolds > manifoldCap / 2) {
                const uint64_t p = hCounters->pairs > pairCap / 2 ? std::max<uint64_t>(2ull * pairCap, 2ull * hCounters->pairs) : pairCap;
                const uint64_t m = hCounters->manifolds > manifoldCap / 2
                                       ? std::max<uint64_t>(2ull * manifoldCap, 2ull * hCounters->manifolds)
                                       : manifoldCap;
                reserveCapacities(uint32_t(std::min<uint64_t>(p, 1ull << 30)), uint32_t(std::min<uint64_t>(m, 1ull << 30)));
            }
            if (recording && hCounters->events) collectEvents(hCounters->events);
            stepsTaken++;
            return;
        }
        throw ApiError(AG2D_ERR_CAPACITY, "step kept overflowing its buffers");
    }
};

// ---------------------------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------------------------
extern "C" {

const char* ag2d_last_error_string(void) { return g_error.c_str(); }

int32_t ag2d_version(void) { return 1; }

int32_t ag2d_device_count(int32_t* out_count)
{
    return guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
        if (out_count) *out_count = n;
    });
}

int32_t ag2d_world_create(const ag2d_world_settings* settings, ag2d_world** out_world)
{
    return guarded([&] {
        if (!settings || !out_world) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (!(settings->dt > 0.0f)) throw ApiError(AG2D_ERR_INVALID_ARG, "dt must be > 0");
        std::unique_ptr<ag2d_world> w(new ag2d_world());
        w->init(*settings);
        *out_world = w.release();
    });
}

int32_t ag2d_world_destroy(ag2d_world* world)
{
    return guarded([&] {
        if (world) cudaSetDevice(world->settings.device);
        delete world;
    });
}

int32_t ag2d_world_add_material(ag2d_world* world, float e, float sf, float df, uint32_t* out_index)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        const uint32_t idx = world->objects.addMaterial(e, sf, df);
        if (out_index) *out_index = idx;
        world->hostDirty = true;
    });
}

static void body_desc(const ag2d_body_desc* b, float* d)
{
    d[0] = b->x; d[1] = b->y; d[2] = b->rotation; d[3] = b->vx; d[4] = b->vy; d[5] = b->angular_velocity;
    d[6] = b->mass;
}

// Creation after the first step pulls the live device state back so new bodies join the running world.
static void pull_state(ag2d_world* w);

int32_t ag2d_world_add_circle(ag2d_world* world, const ag2d_body_desc* body, float radius, uint64_t* out_handle)
{
    return guarded([&] {
        if (!world || !body) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        pull_state(world);
        float d[7];
        body_desc(body, d);
        uint64_t h = 0;
        std::string err;
        if (!world->objects.addCircle(d, body->material, radius, h, err)) throw ApiError(AG2D_ERR_INVALID_ARG, err);
        world->hostDirty = true;
        if (out_handle) *out_handle = h;
    });
}

int32_t ag2d_world_add_box(ag2d_world* world, const ag2d_body_desc* body, float width, float height,
                           uint64_t* out_handle)
{
    return guarded([&] {
        if (!world || !body) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        pull_state(world);
        float d[7];
        body_desc(body, d);
        uint64_t h = 0;
        std::string err;
        if (!world->objects.addBox(d, body->material, width, height, h, err)) throw ApiError(AG2D_ERR_INVALID_ARG, err);
        world->hostDirty = true;
        if (out_handle) *out_handle = h;
    });
}

int32_t ag2d_world_add_polygon(ag2d_world* world, const ag2d_body_desc* body, const float* xy, uint32_t n,
                               uint64_t* out_handle)
{
    return guarded([&] {
        if (!world || !body) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        pull_state(world);
        float d[7];
        body_desc(body, d);
        uint64_t h = 0;
        std::string err;
        if (!world->objects.addPolygon(d, body->material, xy, n, h, err)) {
            throw ApiError(AG2D_ERR_INVALID_ARG, err);
        }
        world->hostDirty = true;
        if (out_handle) *out_handle = h;
    });
}

int32_t ag2d_world_add_capsule(ag2d_world* world, const ag2d_body_desc* body, float length, float radius,
                               uint64_t* out_handle)
{
    return guarded([&] {
        if (!world || !body) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        pull_state(world);
        float d[7];
        body_desc(body, d);
        uint64_t h = 0;
        std::string err;
        if (!world->objects.addCapsule(d, body->material, length, radius, h, err)) throw ApiError(AG2D_ERR_INVALID_ARG, err);
        world->hostDirty = true;
        if (out_handle) *out_handle = h;
    });
}

int32_t ag2d_world_create_body(ag2d_world* world, const ag2d_body_desc* body, float inertia, float com_x,
                               float com_y, uint64_t* out_handle)
{
    return guarded([&] {
        if (!world || !body) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        pull_state(world);
        float d[7];
        body_desc(body, d);
        uint64_t h = 0;
        std::string err;
        if (!world->objects.addBody(d, inertia, com_x, com_y, h, err)) throw ApiError(AG2D_ERR_INVALID_ARG, err);
        world->hostDirty = true;
        if (out_handle) *out_handle = h;
    });
}

int32_t ag2d_world_add_collider(ag2d_world* world, uint64_t body, int32_t shape, float local_x, float local_y,
                                float local_rotation, uint32_t material, const float* params, const float* xy,
                                uint32_t n_vertices, uint32_t* out_collider)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (shape < 0 || shape > 3) throw ApiError(AG2D_ERR_INVALID_ARG, "unknown shape kind");
        if (shape != SHAPE_POLYGON && !params) throw ApiError(AG2D_ERR_INVALID_ARG, "null shape parameters");
        const uint32_t b = world->objects.indexOf(body);
        if (b == 0xFFFFFFFFu) throw ApiError(AG2D_ERR_INVALID_ARG, "stale body handle");
        pull_state(world);
        uint32_t c = 0;
        std::string err;
        if (!world->objects.addCollider(b, uint32_t(shape), local_x, local_y, local_rotation, material, params, xy,
                                        n_vertices, c, err))
            throw ApiError(AG2D_ERR_INVALID_ARG, err);
        world->hostDirty = true;
        if (out_collider) *out_collider = c;
    });
}

int32_t ag2d_world_add_bodies(ag2d_world* world, uint32_t count, const ag2d_body_desc* bodies,
                              const uint32_t* kinds, const float* params, const uint32_t* poly_offsets,
                              const uint32_t* poly_counts, const float* poly_xy, uint64_t* out_handles)
{
    return guarded([&] {
        if (!world || (count && (!bodies || !kinds || !params)))
            throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        pull_state(world);
        for (uint32_t i = 0; i < count; i++) {
            float d[7];
            body_desc(bodies + i, d);
            uint64_t h = 0;
            std::string err;
            bool ok = false;
            int32_t code = AG2D_ERR_INVALID_ARG;
            switch (kinds[i]) {
            case SHAPE_CIRCLE: ok = world->objects.addCircle(d, bodies[i].material, params[2 * i], h, err); break;
            case SHAPE_BOX:
                ok = world->objects.addBox(d, bodies[i].material, params[2 * i], params[2 * i + 1], h, err);
                break;
            case SHAPE_CAPSULE:
                ok = world->objects.addCapsule(d, bodies[i].material, params[2 * i], params[2 * i + 1], h, err);
                break;
            case SHAPE_POLYGON:
                if (!poly_offsets || !poly_counts || !poly_xy) { err = "polygon without vertex arrays"; break; }
                ok = world->objects.addPolygon(d, bodies[i].material, poly_xy + 2 * size_t(poly_offsets[i]),
                                               poly_counts[i], h, err);
                break;
            default: err = "unknown shape kind"; break;
            }
            if (!ok) throw ApiError(code, "body " + std::to_string(i) + ": " + err);
            world->hostDirty = true;
            if (out_handles) out_handles[i] = h;
        }
    });
}

uint32_t ag2d_world_body_index(ag2d_world* world, uint64_t handle)
{
    return world ? world->objects.indexOf(handle) : 0xFFFFFFFFu;
}

static int32_t queue_command(ag2d_world* world, int32_t kind, uint64_t handle, float a, float b)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (world->nWorlds > 1) throw ApiError(AG2D_ERR_UNSUPPORTED, "body commands are per world");
        world->commands.push_back(BodyCommand{kind, handle, a, b});
    });
}

int32_t ag2d_world_destroy_body(ag2d_world* world, uint64_t body)
{
    return queue_command(world, AG2D_COMMAND_DESTROY, body, 0.0f, 0.0f);
}
int32_t ag2d_world_set_body_position(ag2d_world* world, uint64_t body, float x, float y)
{
    return queue_command(world, AG2D_COMMAND_POSITION, body, x, y);
}
int32_t ag2d_world_set_body_rotation(ag2d_world* world, uint64_t body, float rotation)
{
    return queue_command(world, AG2D_COMMAND_ROTATION, body, rotation, 0.0f);
}
int32_t ag2d_world_set_body_velocity(ag2d_world* world, uint64_t body, float vx, float vy)
{
    return queue_command(world, AG2D_COMMAND_VELOCITY, body, vx, vy);
}
int32_t ag2d_world_set_body_angular_velocity(ag2d_world* world, uint64_t body, float angular_velocity)
{
    return queue_command(world, AG2D_COMMAND_ANGULAR_VELOCITY, body, angular_velocity, 0.0f);
}
int32_t ag2d_world_set_body_mass(ag2d_world* world, uint64_t body, float mass)
{
    return queue_command(world, AG2D_COMMAND_MASS, body, mass, 0.0f);
}
int32_t ag2d_world_set_body_inertia(ag2d_world* world, uint64_t body, float inertia)
{
    return queue_command(world, AG2D_COMMAND_INERTIA, body, inertia, 0.0f);
}

int32_t ag2d_world_set_body_local_center_of_mass(ag2d_world* world, uint64_t body, float x, float y)
{
    return queue_command(world, AG2D_COMMAND_LOCAL_CENTER_OF_MASS, body, x, y);
}
int32_t ag2d_world_recompute_body_inertia(ag2d_world* world, uint64_t body)
{
    return queue_command(world, AG2D_COMMAND_RECOMPUTE_INERTIA, body, 0.0f, 0.0f);
}
int32_t ag2d_world_set_body_mass_from_density(ag2d_world* world, uint64_t body, float density)
{
    return queue_command(world, AG2D_COMMAND_MASS_FROM_DENSITY, body, density, 0.0f);
}
int32_t ag2d_world_set_collider(ag2d_world* world, uint32_t collider, int32_t command, float a, float b)
{
    if (command < AG2D_COMMAND_COLLIDER_OFFSET || command > AG2D_COMMAND_CAPSULE_SHAPE) {   // polygons: below
        g_error = "unknown collider command";
        return AG2D_ERR_INVALID_ARG;
    }
    return queue_command(world, command, uint64_t(collider), a, b);
}

int32_t ag2d_world_set_polygon_shape(ag2d_world* world, uint32_t collider, const float* xy, uint32_t n)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (world->nWorlds > 1) throw ApiError(AG2D_ERR_UNSUPPORTED, "body commands are per world");
        if (!xy || n < 3) throw ApiError(AG2D_ERR_INVALID_ARG, "polygon needs at least 3 vertices");
        std::vector<float> outline;
        std::string err;
        if (!prepare_outline(xy, n, outline, err)) throw ApiError(AG2D_ERR_INVALID_ARG, err);
        BodyCommand c{AG2D_COMMAND_POLYGON_SHAPE, uint64_t(collider), 0.0f, 0.0f};
        c.slot = uint32_t(world->pendingPolygons.size());
        world->pendingPolygons.push_back(std::move(outline));
        world->commands.push_back(c);
    });
}

int32_t ag2d_decompose_polygon(const float* xy, uint32_t n, float* out_xy, uint32_t out_capacity,
                               uint32_t* piece_counts, uint32_t piece_capacity, uint32_t* out_pieces)
{
    return guarded([&] {
        if (!xy || !out_pieces) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (n < 3) throw ApiError(AG2D_ERR_INVALID_ARG, "polygon needs at least 3 vertices");
        std::vector<float> outline;
        std::string err;
        if (!prepare_outline_any(xy, n, outline, err)) throw ApiError(AG2D_ERR_INVALID_ARG, err);
        const std::vector<std::vector<float>> pieces = decompose_outline(outline, 16);
        size_t verts = 0;
        for (const auto& p : pieces) verts += p.size() / 2;
        *out_pieces = uint32_t(pieces.size());
        if (pieces.size() > piece_capacity || verts > out_capacity || !piece_counts || !out_xy)
            throw ApiError(AG2D_ERR_CAPACITY, "output arrays too small: " + std::to_string(pieces.size()) +
                                                  " pieces, " + std::to_string(verts) + " vertices");
        size_t at = 0;
        for (size_t k = 0; k < pieces.size(); k++) {
            piece_counts[k] = uint32_t(pieces[k].size() / 2);
            std::copy(pieces[k].begin(), pieces[k].end(), out_xy + 2 * at);
            at += pieces[k].size() / 2;
        }
    });
}

int32_t ag2d_world_flush_commands(ag2d_world* world)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (world->commands.empty() && world->jointCommands.empty()) return;
        CK(cudaSetDevice(world->settings.device));
        world->flushCommands();
    });
}

int32_t ag2d_world_load_state(ag2d_world* world, const ag2d_state_desc* st)
{
    return guarded([&] {
        if (!world || !st) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        ag2d_world& w = *world;
        const uint32_t nb = st->n_bodies, nc = st->n_colliders;
        w.nBodies = nb;
        w.nColliders = nc;
        std::vector<float4> vel(nb), pos(nb);
        std::vector<float2> rot(nb);
        std::vector<float> wc(nb), br(nb), tm(nb);
        std::vector<uint8_t> state(nb);
        std::vector<uint32_t> isl(nb);
        for (uint32_t i = 0; i < nb; i++) {
            vel[i] = make_float4(st->vel_x[i], st->vel_y[i], st->angular_velocity[i], st->inv_mass[i]);
            pos[i] = make_float4(st->com_x[i], st->com_y[i], st->rotation[i], st->inv_inertia[i]);
            rot[i] = make_float2(st->rot_cos[i], st->rot_sin[i]);
            wc[i] = st->wrap_count ? st->wrap_count[i] : 0.0f;
            br[i] = st->bound_radius ? st->bound_radius[i] : 0.0f;
            tm[i] = st->sleep_timer ? st->sleep_timer[i] : 0.0f;
            const uint32_t* g = st->body_group_starts;
            state[i] = uint8_t(i < g[1] ? STATE_STATIC : (i < g[2] ? STATE_SLEEPING : STATE_DYNAMIC));
            isl[i] = st->sleep_island ? st->sleep_island[i] : 0xFFFFFFFFu;
        }
        // Sleeping islands are identified by their smallest member body index on the device (the union-find root
        // convention); the reference numbers them from 2 (FIRST_SLEEP_ISLAND_ID, SoA/BodySoA.h:45).
        {
            std::vector<std::pair<uint32_t, uint32_t>> ids;   // (reference id, first member)
            for (uint32_t i = 0; i < nb; i++) {
                if (state[i] != STATE_SLEEPING) { isl[i] = 0xFFFFFFFFu; continue; }
                auto it = std::find_if(ids.begin(), ids.end(), [&](const auto& p) { return p.first == isl[i]; });
                if (it == ids.end()) { ids.emplace_back(isl[i], i); isl[i] = i; }
                else isl[i] = it->second;
            }
        }
        std::vector<uint32_t> cb(nc), cs(nc), cm(nc);
        std::vector<float4> co(nc);
        const uint32_t nCaps = st->capsule_half_length && st->capsule_radius ? st->n_capsules : 0u;
        for (uint32_t i = 0; i < nc; i++) {
            cb[i] = st->col_body[i];
            const uint32_t type = st->col_shape_type[i];
            if (type > SHAPE_CAPSULE || (type == SHAPE_CAPSULE && st->col_shape_index[i] >= nCaps))
                throw ApiError(AG2D_ERR_INVALID_ARG, "collider " + std::to_string(i) + ": bad shape");
            // Capsules follow the boxes in the shared parameter table.
            const uint32_t idx = st->col_shape_index[i] + (type == SHAPE_CAPSULE ? st->n_boxes : 0u);
            cs[i] = (type << 30) | idx;
            cm[i] = st->col_material[i];
            co[i] = make_float4(st->col_com_offset_x[i], st->col_com_offset_y[i], st->col_local_rotation[i], 0.0f);
        }
        std::vector<float> cr(st->circle_radius, st->circle_radius + st->n_circles);
        std::vector<float2> bh(size_t(st->n_boxes) + nCaps);
        for (uint32_t i = 0; i < st->n_boxes; i++) bh[i] = make_float2(st->box_half_width[i], st->box_half_height[i]);
        for (uint32_t i = 0; i < nCaps; i++)
            bh[st->n_boxes + i] = make_float2(st->capsule_half_length[i], st->capsule_radius[i]);
        std::vector<uint32_t> po(st->n_polygons), pc(st->n_polygons);
        uint32_t total = 0;
        for (uint32_t i = 0; i < st->n_polygons; i++) { po[i] = total; pc[i] = st->poly_count[i]; total += pc[i]; }
        std::vector<float2> pv(total), pn(total);
        for (uint32_t k = 0; k < total; k++) {
            pv[k] = make_float2(st->poly_vertices[2 * k], st->poly_vertices[2 * k + 1]);
            pn[k] = make_float2(st->poly_normals[2 * k], st->poly_normals[2 * k + 1]);
        }
        std::vector<float4> mats(st->n_materials);
        w.objects.materials.assign(st->materials, st->materials + 3 * st->n_materials);
        for (uint32_t i = 0; i < st->n_materials; i++)
            mats[i] = make_float4(st->materials[3 * i], st->materials[3 * i + 1], st->materials[3 * i + 2], 0.0f);
        w.uploadArrays(vel, pos, rot, wc, br, tm, state, isl, cb, cs, cm, co, cr, bh, po, pc, pv, pn, mats);
        if (st->col_world_x && st->col_world_y && st->col_world_cos && st->col_world_sin) {
            std::vector<float4> pose(nc);
            for (uint32_t i = 0; i < nc; i++)
                pose[i] = make_float4(st->col_world_x[i], st->col_world_y[i], st->col_world_cos[i], st->col_world_sin[i]);
            if (nc) CK(cudaMemcpyAsync(w.cpose.p, pose.data(), nc * sizeof(float4), cudaMemcpyHostToDevice, w.stream));
            CK(cudaStreamSynchronize(w.stream));
        }
        if (st->col_aabb_min_x && st->col_aabb_min_y && st->col_aabb_max_x && st->col_aabb_max_y) {
            std::vector<float4> box(nc);
            for (uint32_t i = 0; i < nc; i++)
                box[i] = make_float4(st->col_aabb_min_x[i], st->col_aabb_min_y[i], st->col_aabb_max_x[i],
                                     st->col_aabb_max_y[i]);
            if (nc) CK(cudaMemcpyAsync(w.caabb.p, box.data(), nc * sizeof(float4), cudaMemcpyHostToDevice, w.stream));
            CK(cudaStreamSynchronize(w.stream));
            w.aabbValid = true;
        }
        // The loaded state replaces any host-created objects (and their colliders' event opt-ins).
        w.objects.bodies.clear();
        w.objects.colliders.clear();
        w.loadedOptIn.assign(nc, ColliderEvent{0u, 3.40282347e38f});
        w.optInDirty = true;
        for (JointSystem& js : w.objects.jointSystems) js = JointSystem();
        for (uint32_t k = 0; k < JOINT_KINDS; k++) w.jointActive[k] = w.jointLevels[k] = 0;
        w.nJointEdges = 0;
        w.jointsDirty = false;
        w.hostDirty = false;
    });
}

int32_t ag2d_world_step(ag2d_world* world, int32_t steps)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (steps < 0) throw ApiError(AG2D_ERR_INVALID_ARG, "steps must be >= 0");
        CK(cudaSetDevice(world->settings.device));
        if (world->dispatching) throw ApiError(AG2D_ERR_INVALID_ARG, "a collision callback may not step the world");
        for (int32_t i = 0; i < steps; i++) {
            world->stepOnce();
            world->dispatchEvents();
        }
    });
}

// Body constraints ------------------------------------------------------------------------------------------

// A body command that only wakes the body's island (constraint creation on a world that has run).
constexpr int32_t COMMAND_WAKE = 100;

static JointSystem& joint_system(ag2d_world* world, int32_t kind)
{
    if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
    if (kind < 0 || kind >= int32_t(JOINT_KINDS)) throw ApiError(AG2D_ERR_INVALID_ARG, "unknown constraint kind");
    if (world->nWorlds > 1) throw ApiError(AG2D_ERR_UNSUPPORTED, "body constraints are per world");
    return world->objects.jointSystems[kind];
}

static uint64_t body_handle_of(const HostObjects& o, uint32_t b)
{
    if (b == NO_BODY || b >= o.bodies.size()) return 0;
    const uint32_t slot = o.bodies[b].handleSlot;
    return (uint64_t(o.slotGeneration[slot]) << 32) | slot;
}

int32_t ag2d_world_create_joint(ag2d_world* world, const ag2d_joint_desc* d, uint64_t* out_handle)
{
    return guarded([&] {
        if (!d || !out_handle) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        JointSystem& js = joint_system(world, d->kind);
        HostObjects& o = world->objects;
        const bool single = d->kind == AG2D_JOINT_MOTOR;
        const uint32_t a = o.indexOf(d->body_a), b = single ? NO_BODY : o.indexOf(d->body_b);
        if (a == 0xFFFFFFFFu || (!single && b == 0xFFFFFFFFu))
            throw ApiError(AG2D_ERR_INVALID_ARG, "stale body handle");
        world->beforeJointEdit();
        HJoint j;
        j.bodyA = a;
        j.bodyB = b;
        j.anchorAx = d->anchor_a_x; j.anchorAy = d->anchor_a_y; j.anchorBx = d->anchor_b_x; j.anchorBy = d->anchor_b_y;
        j.restLength = d->rest_length; j.stiffness = d->stiffness; j.damping = d->damping;
        j.targetSpeed = d->target_speed; j.maxTorque = d->max_torque; j.impulse = 0.0f;
        j.axisX = d->axis_x; j.axisY = d->axis_y;
        if (!normalize_axis(j.axisX, j.axisY)) { j.axisX = 1.0f; j.axisY = 0.0f; }   // sanitizeAxis
        j.lowerLimit = d->lower_limit; j.upperLimit = d->upper_limit; j.enableLimit = d->enable_limit != 0;
        if (d->kind == AG2D_JOINT_PRISMATIC) {
            // The bodies' rotations now: the host's before the first upload, else the device's.
            float ra = o.bodies[a].rot, rb = o.bodies[b].rot;
            if (!world->hostDirty) {
                CK(cudaSetDevice(world->settings.device));
                float4 pa, pb;
                CK(cudaMemcpy(&pa, world->bpos.p + a, sizeof(float4), cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(&pb, world->bpos.p + b, sizeof(float4), cudaMemcpyDeviceToHost));
                ra = pa.z;
                rb = pb.z;
            }
            j.referenceAngle = reference_angle(ra, rb);
        }
        // refreshConstraintGroup (ObjectManager.cpp:1207-1220): Inactive when no body has mass.
        const bool inactive = o.bodies[a].invMass == 0.0f && (single || o.bodies[b].invMass == 0.0f);
        const uint32_t i = js.create(j, inactive ? JGROUP_INACTIVE : JGROUP_ACTIVE);
        *out_handle = js.handleOf(i);
        if (!world->hostDirty) {   // the bodies wake (createConstraint, ObjectManager.cpp:451-454) at the flush
            world->commands.push_back(BodyCommand{COMMAND_WAKE, d->body_a, 0.0f, 0.0f});
            if (!single) world->commands.push_back(BodyCommand{COMMAND_WAKE, d->body_b, 0.0f, 0.0f});
        }
    });
}

int32_t ag2d_world_destroy_joint(ag2d_world* world, int32_t kind, uint64_t handle)
{
    return guarded([&] {
        joint_system(world, kind);
        world->jointCommands.push_back(ag2d_world::JointCommand{kind, -1, handle, 0.0f, 0.0f});
    });
}

int32_t ag2d_world_set_joint(ag2d_world* world, int32_t kind, uint64_t handle, int32_t field, float a, float b)
{
    return guarded([&] {
        joint_system(world, kind);
        if (field < AG2D_JOINT_ANCHOR_A || field > AG2D_JOINT_RESET_REFERENCE_ANGLE)
            throw ApiError(AG2D_ERR_INVALID_ARG, "unknown constraint field");
        world->jointCommands.push_back(ag2d_world::JointCommand{kind, field, handle, a, b});
    });
}

int32_t ag2d_world_joint(ag2d_world* world, int32_t kind, uint64_t handle, ag2d_joint_desc* out)
{
    return guarded([&] {
        JointSystem& js = joint_system(world, kind);
        if (!out) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        const uint32_t i = js.indexOf(handle);
        if (i == NO_BODY) throw ApiError(AG2D_ERR_INVALID_ARG, "stale constraint handle");
        if (kind == AG2D_JOINT_MOTOR) world->pullMotorImpulses();
        const HJoint& j = js.joints[i];
        *out = ag2d_joint_desc{};
        out->kind = kind;
        out->body_a = body_handle_of(world->objects, j.bodyA);
        out->body_b = body_handle_of(world->objects, j.bodyB);
        out->anchor_a_x = j.anchorAx; out->anchor_a_y = j.anchorAy;
        out->anchor_b_x = j.anchorBx; out->anchor_b_y = j.anchorBy;
        out->rest_length = j.restLength; out->stiffness = j.stiffness; out->damping = j.damping;
        out->target_speed = j.targetSpeed; out->max_torque = j.maxTorque; out->impulse = j.impulse;
        out->axis_x = j.axisX; out->axis_y = j.axisY;
        out->lower_limit = j.lowerLimit; out->upper_limit = j.upperLimit; out->enable_limit = j.enableLimit ? 1 : 0;
        out->reference_angle = j.referenceAngle;
    });
}

int32_t ag2d_world_joint_count(ag2d_world* world, int32_t kind, uint32_t* out_count)
{
    return guarded([&] {
        JointSystem& js = joint_system(world, kind);
        if (!out_count) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        *out_count = uint32_t(js.joints.size());
    });
}

int32_t ag2d_world_joint_handle(ag2d_world* world, int32_t kind, uint32_t index, uint64_t* out_handle)
{
    return guarded([&] {
        JointSystem& js = joint_system(world, kind);
        if (!out_handle) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (index >= js.joints.size()) throw ApiError(AG2D_ERR_INVALID_ARG, "constraint index out of range");
        *out_handle = js.handleOf(index);
    });
}

int32_t ag2d_world_set_joint_iterations(ag2d_world* world, int32_t kind, uint32_t iterations)
{
    return guarded([&] { joint_system(world, kind).iterations = iterations; });
}

int32_t ag2d_device_allocs(uint64_t* out)
{
    return guarded([&] {
        if (!out) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        *out = g_deviceAllocs.load(std::memory_order_relaxed);
    });
}

int32_t ag2d_world_create_collision_callback(ag2d_world* world, ag2d_collision_callback function, void* user_data,
                                             uint16_t* out_id)
{
    return guarded([&] {
        if (!world || !out_id) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (!function) throw ApiError(AG2D_ERR_INVALID_ARG, "null callback function");
        if (world->nWorlds > 1) throw ApiError(AG2D_ERR_UNSUPPORTED, "collision events are per world");
        ag2d_world& w = *world;
        uint16_t id;
        if (!w.callbackFree.empty()) {
            id = w.callbackFree.back();
            w.callbackFree.pop_back();
        } else {
            if (w.callbacks.size() >= 65535) throw ApiError(AG2D_ERR_CAPACITY, "all collision callback ids are in use");
            id = uint16_t(w.callbacks.size());
            w.callbacks.emplace_back();
            w.callbackAlive.push_back(0);
        }
        w.callbacks[id] = ag2d_world::CallbackEntry{function, user_data};
        w.callbackAlive[id] = 1;
        w.callbacksAlive++;
        *out_id = id;
    });
}

int32_t ag2d_world_destroy_collision_callback(ag2d_world* world, uint16_t id)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        ag2d_world& w = *world;
        if (id == 0 || id >= w.callbacks.size() || !w.callbackAlive[id])
            throw ApiError(AG2D_ERR_INVALID_ARG, "collision callback " + std::to_string(id) + " is not alive");
        w.callbacks[id] = ag2d_world::CallbackEntry{};
        w.callbackAlive[id] = 0;
        w.callbackFree.push_back(id);
        w.callbacksAlive--;
        // Colliders using it go back to no callback (Simulation.cpp:140-149).
        const uint32_t n = w.colliderCount();
        for (uint32_t c = 0; c < n; c++)
            if (w.optIn(c).callback == id) w.setOptIn(c, 0u, 3.40282347e38f);
    });
}

int32_t ag2d_world_set_collider_collision_callback(ag2d_world* world, uint32_t collider, uint16_t id,
                                                   float impulse_threshold)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        ag2d_world& w = *world;
        if (w.nWorlds > 1) throw ApiError(AG2D_ERR_UNSUPPORTED, "collision events are per world");
        if (collider >= w.colliderCount())
            throw ApiError(AG2D_ERR_INVALID_ARG, "collider " + std::to_string(collider) + " out of range");
        if (id == 0) {
            w.setOptIn(collider, 0u, 3.40282347e38f);
            return;
        }
        if (id >= w.callbacks.size() || !w.callbackAlive[id])
            throw ApiError(AG2D_ERR_INVALID_ARG, "collision callback " + std::to_string(id) + " is not alive");
        if (!(impulse_threshold >= 0.0f)) throw ApiError(AG2D_ERR_INVALID_ARG, "threshold must be >= 0");
        w.setOptIn(collider, id, impulse_threshold);
    });
}

int32_t ag2d_world_set_collision_events(ag2d_world* world, int32_t enable)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        world->eventsEnabled = enable != 0;
    });
}

int32_t ag2d_world_collision_events(ag2d_world* world, ag2d_collision_event* out_events, uint32_t capacity,
                                    uint32_t* out_count)
{
    return guarded([&] {
        if (!world || !out_count) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        const auto& ev = world->lastEvents;
        *out_count = uint32_t(ev.size());
        const uint32_t k = std::min<uint32_t>(capacity, uint32_t(ev.size()));
        if (k && !out_events) throw ApiError(AG2D_ERR_INVALID_ARG, "null event buffer");
        if (k) std::memcpy(out_events, ev.data(), k * sizeof(ag2d_collision_event));
    });
}

int32_t ag2d_world_counters(ag2d_world* world, ag2d_counters* out)
{
    return guarded([&] {
        if (!world || !out) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        static const StepCounters none{};
        const StepCounters& c = world->hCounters ? *world->hCounters : none;
        out->status = c.status; out->pairs = c.pairs; out->manifolds = c.manifolds; out->colors = c.colors;
        out->woke = c.woke; out->slept = c.slept; out->warm_hits = c.warmHits;
        out->sleeping = world->nBodies - world->nDynBody - world->nStatic - world->nDestroyed;
        out->ccd_hits = c.ccdHits;
        out->restored = c.restored;
        out->device_allocs = g_deviceAllocs.load(std::memory_order_relaxed);
        out->events = uint32_t(world->lastEvents.size());
        out->stored = c.stored;
        out->steps = world->stepsTaken;
        out->launches = world->launches;
        out->list_rebuilds = world->listRebuilds;
        out->retries = world->retries;
        out->regrows = world->regrows;
        out->host_ms = world->hostMs;
        out->sync_ms = world->syncMs;
    });
}

int32_t ag2d_world_autotune(ag2d_world* world, int32_t steps_per_candidate, ag2d_tuning* out)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (steps_per_candidate < 1) throw ApiError(AG2D_ERR_INVALID_ARG, "steps_per_candidate must be >= 1");
        CK(cudaSetDevice(world->settings.device));
        world->ensureUploaded();
        ag2d_tuning t{};
        world->autotune(uint32_t(steps_per_candidate), t);
        if (out) *out = t;
    });
}

int32_t ag2d_world_set_tuning(ag2d_world* world, const ag2d_tuning* tuning)
{
    return guarded([&] {
        if (!world || !tuning) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        const ag2d_tuning& t = *tuning;
        auto oneOf = [](uint32_t v, std::initializer_list<uint32_t> ok) {
            return std::find(ok.begin(), ok.end(), v) != ok.end();
        };
        if (!oneOf(t.query_threads, {64, 128, 256}) || !oneOf(t.narrow_threads, {128, 256, 512}))
            throw ApiError(AG2D_ERR_INVALID_ARG, "query / narrow block size out of range");
        if (t.team_colliders && (!oneOf(t.team_threads, {64, 128, 256, 512}) || t.team_colliders < 64 ||
                                 t.team_colliders > MAX_TEAM_BODY_CAP))
            throw ApiError(AG2D_ERR_INVALID_ARG, "team size out of range");
        CK(cudaSetDevice(world->settings.device));
        world->ensureUploaded();
        world->queryThreads = t.query_threads;
        world->narrowThreads = t.narrow_threads;
        world->consOnChip = t.team_cons_on_chip != 0;
        if (t.big_team_mode > 3) throw ApiError(AG2D_ERR_INVALID_ARG, "big_team_mode out of range");
        world->bigThreads = (t.big_team_mode & 1u) ? 256u : 512u;
        world->bigPipelined = (t.big_team_mode & 2u) != 0;
        if (t.team_colliders) {
            world->teamColliders = t.team_colliders;
            world->teamThreads = t.team_threads;
            if (world->nWorlds > 1) world->setTeams(t.team_colliders, t.team_threads);
        }
    });
}

int32_t ag2d_world_set_profiling(ag2d_world* world, int32_t enable)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        world->profiling = enable != 0;
        for (int p = 0; p < ag2d_world::NPHASE; p++) {
            world->phaseMs[p] = 0.0;
            world->phaseCalls[p] = 0;
            world->evPending[p] = false;
        }
    });
}

int32_t ag2d_world_phase_times(ag2d_world* world, double* out_ms, uint64_t* out_calls, int32_t capacity)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        for (int p = 0; p < std::min<int>(capacity, ag2d_world::NPHASE); p++) {
            if (out_ms) out_ms[p] = world->phaseMs[p];
            if (out_calls) out_calls[p] = world->phaseCalls[p];
        }
    });
}

int32_t ag2d_world_stream(ag2d_world* world, void** out_stream)
{
    return guarded([&] {
        if (!world || !out_stream) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        world->ensureDevice();
        *out_stream = world->stream;
    });
}

int32_t ag2d_world_body_count(ag2d_world* world, uint32_t* out_bodies, uint32_t* out_colliders)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        const bool host = world->hostDirty;
        if (out_bodies) *out_bodies = host ? uint32_t(world->objects.bodies.size()) : world->nBodies;
        if (out_colliders) *out_colliders = host ? uint32_t(world->objects.colliders.size()) : world->nColliders;
    });
}

}  // extern "C"

// Field access ---------------------------------------------------------------------------------------------------

// Host memory the device can copy into directly: page-locked by cudaHostAlloc or cudaHostRegister (any CUDA runtime
// of the process; the driver tracks it).
static bool page_locked(const void* p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// How a per-body or per-collider field is read: its device array and how k_extract packs it.
struct FieldSpec {
    const void* src = nullptr;
    uint32_t kind = EXTRACT_DIRECT, comp = 0;
    uint32_t outBytes = 4;      // bytes per element as read
    bool perCollider = false;
};

static bool field_spec(const ag2d_world& w, int32_t field, FieldSpec& f)
{
    auto c4 = [&](const void* p, uint32_t c) { f.src = p; f.kind = EXTRACT_F4_COMP; f.comp = c; };
    auto c2 = [&](const void* p, uint32_t c) { f.src = p; f.kind = EXTRACT_F2_COMP; f.comp = c; };
    switch (field) {
    case AG2D_BODY_COM_X: c4(w.bpos.p, 0); break;
    case AG2D_BODY_COM_Y: c4(w.bpos.p, 1); break;
    case AG2D_BODY_ROTATION: c4(w.bpos.p, 2); break;
    case AG2D_BODY_INV_INERTIA: c4(w.bpos.p, 3); break;
    case AG2D_BODY_VEL_X: c4(w.bvel.p, 0); break;
    case AG2D_BODY_VEL_Y: c4(w.bvel.p, 1); break;
    case AG2D_BODY_ANGULAR_VELOCITY: c4(w.bvel.p, 2); break;
    case AG2D_BODY_INV_MASS: c4(w.bvel.p, 3); break;
    case AG2D_BODY_ROT_COS: c2(w.brot.p, 0); break;
    case AG2D_BODY_ROT_SIN: c2(w.brot.p, 1); break;
    case AG2D_BODY_WRAP_COUNT: f.src = w.wrapCount.p; break;
    case AG2D_BODY_SLEEP_TIMER: f.src = w.sleepTimer.p; break;
    case AG2D_BODY_STATE: f.src = w.bstate.p; f.kind = EXTRACT_U8_U32; break;
    case AG2D_BODY_SLEEP_ISLAND: f.src = w.sleepIsland.p; f.kind = EXTRACT_ISLAND; break;
    case AG2D_BODY_POSE: f.src = w.bpos.p; f.kind = EXTRACT_F4_XYZ; f.outBytes = 12; break;
    case AG2D_COL_WORLD_X: c4(w.cpose.p, 0); f.perCollider = true; break;
    case AG2D_COL_WORLD_Y: c4(w.cpose.p, 1); f.perCollider = true; break;
    case AG2D_COL_WORLD_COS: c4(w.cpose.p, 2); f.perCollider = true; break;
    case AG2D_COL_WORLD_SIN: c4(w.cpose.p, 3); f.perCollider = true; break;
    case AG2D_COL_WORLD_ROTATION: f.src = w.cworldRot.p; f.perCollider = true; break;
    case AG2D_COL_AABB_MIN_X: c4(w.caabb.p, 0); f.perCollider = true; break;
    case AG2D_COL_AABB_MIN_Y: c4(w.caabb.p, 1); f.perCollider = true; break;
    case AG2D_COL_AABB_MAX_X: c4(w.caabb.p, 2); f.perCollider = true; break;
    case AG2D_COL_AABB_MAX_Y: c4(w.caabb.p, 3); f.perCollider = true; break;
    case AG2D_COL_BODY: f.src = w.cbody.p; f.kind = EXTRACT_ISLAND; f.perCollider = true; break;   // biased like ids
    default: return false;
    }
    return true;
}

// Copies 'bytes' of device memory into host memory on the engine stream and waits for them: one transfer into a
// page-locked destination, else 8 MiB chunks through the two halves of a page-locked bounce buffer, the transfer
// of chunk c + 1 overlapping the host copy of chunk c.
static void copy_to_host(ag2d_world& w, void* dst, const void* src, size_t bytes)
{
    const cudaStream_t s = w.stream;
    if (!bytes) return;
    if (page_locked(dst)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return;
    }
    constexpr size_t CHUNK = size_t(8) << 20;
    w.readBounce.reserve(2 * CHUNK);
    for (auto& e : w.readEv)
        if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    const size_t chunks = (bytes + CHUNK - 1) / CHUNK;
    auto issue = [&](size_t c) {
        const size_t off = c * CHUNK, len = std::min(CHUNK, bytes - off);
        CK(cudaMemcpyAsync(w.readBounce.p + (c & 1) * CHUNK, static_cast<const uint8_t*>(src) + off, len,
                           cudaMemcpyDeviceToHost, s));
        CK(cudaEventRecord(w.readEv[c & 1], s));
    };
    issue(0);
    for (size_t c = 0; c < chunks; c++) {
        // Chunk c + 1 lands in the half whose contents the host copied out in the previous iteration.
        if (c + 1 < chunks) issue(c + 1);
        CK(cudaEventSynchronize(w.readEv[c & 1]));
        const size_t off = c * CHUNK, len = std::min(CHUNK, bytes - off);
        std::memcpy(static_cast<uint8_t*>(dst) + off, w.readBounce.p + (c & 1) * CHUNK, len);
    }
}

// Elements [lo, lo + n) of a field, packed, into host memory 'dst'; 'bias' is subtracted from sleeping-island ids
// (the first body of a batch's world). Returns the bytes written.
static uint64_t read_packed(ag2d_world& w, const FieldSpec& f, uint32_t lo, uint32_t n, uint32_t bias, void* dst)
{
    const uint64_t bytes = uint64_t(n) * f.outBytes;
    if (!bytes) return 0;
    const void* src = static_cast<const uint8_t*>(f.src) + size_t(lo) * f.outBytes;
    if (f.kind != EXTRACT_DIRECT) {
        w.readStage.reserve(bytes);
        k_extract<<<w.gridFor(n), 256, 0, w.stream>>>(f.src, lo, n, f.kind, f.comp, bias, w.readStage.p);
        CK(cudaGetLastError());
        src = w.readStage.p;
    }
    copy_to_host(w, dst, src, bytes);
    return bytes;
}

// Queues a read of elements [lo, lo + n) into page-locked 'dst': packed on the engine stream into a ring slot (a
// copy of the values as they are after the work queued so far), then copied on copyStream while later steps run.
static void read_async(ag2d_world& w, const FieldSpec& f, uint32_t lo, uint32_t n, uint32_t bias, void* dst)
{
    const uint64_t bytes = uint64_t(n) * f.outBytes;
    if (!bytes) return;
    if (!w.copyStream) CK(cudaStreamCreateWithFlags(&w.copyStream, cudaStreamNonBlocking));
    ag2d_world::AsyncSlot& a = w.asyncSlot[w.asyncNext++ % ag2d_world::NASYNC];
    if (!a.packed) {
        CK(cudaEventCreateWithFlags(&a.packed, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&a.done, cudaEventDisableTiming));
    }
    if (a.used) {
        if (a.buf.n < bytes) CK(cudaEventSynchronize(a.done));   // growing frees the buffer its last copy reads
        else CK(cudaStreamWaitEvent(w.stream, a.done, 0));       // the next pack waits for that copy on the device
    }
    a.buf.reserve(bytes);
    if (f.kind == EXTRACT_DIRECT) {
        CK(cudaMemcpyAsync(a.buf.p, static_cast<const uint8_t*>(f.src) + size_t(lo) * f.outBytes, bytes,
                           cudaMemcpyDeviceToDevice, w.stream));
    } else {
        k_extract<<<w.gridFor(n), 256, 0, w.stream>>>(f.src, lo, n, f.kind, f.comp, bias, a.buf.p);
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(a.packed, w.stream));
    CK(cudaStreamWaitEvent(w.copyStream, a.packed, 0));
    CK(cudaMemcpyAsync(dst, a.buf.p, bytes, cudaMemcpyDeviceToHost, w.copyStream));
    CK(cudaEventRecord(a.done, w.copyStream));
    a.used = true;
}


// The phase-tap fields (Morton order, pairs, manifolds, solve order, colour starts): element count from the device
// counters where the count lives there. With sizeOnly the bytes are counted but not read.
static std::vector<uint8_t> read_field(ag2d_world& w, int32_t field, bool sizeOnly, uint64_t* bytesOut)
{
    const cudaStream_t s = w.stream;
    auto pack = [](const auto& v) {
        std::vector<uint8_t> out(v.size() * sizeof(v[0]));
        if (!v.empty()) std::memcpy(out.data(), v.data(), out.size());
        return out;
    };
    auto devCount = [&](const uint32_t* p) {
        uint32_t n = 0;
        CK(cudaMemcpyAsync(&n, p, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return n;
    };
    auto get = [&](const auto* p, size_t n) {
        *bytesOut = n * sizeof(*p);
        using T = std::remove_const_t<std::remove_pointer_t<decltype(p)>>;
        return sizeOnly ? std::vector<uint8_t>() : pack(download(static_cast<const T*>(p), n, s));
    };
    switch (field) {
    case AG2D_DYN_SORTED: return get(w.dynTree.vals.p, uint32_t(w.dynTree.n));
    case AG2D_DYN_MORTON:
        return get(w.nWorlds > 1 ? w.dynTree.sortedKey.p : w.dynTree.keys.p, uint32_t(w.dynTree.n));
    case AG2D_PAIRS: return get(w.pairs.p, std::min(devCount(&w.dCounters.p->pairs), w.pairCap));
    case AG2D_MANIFOLDS: return get(w.manifolds.p, devCount(w.nManifolds.p));
    case AG2D_PREV_MANIFOLDS: w.compactPrev(); return get(w.prevManifolds.p, devCount(w.nPrev.p));
    case AG2D_SOLVE_ORDER: return get(w.order.p, devCount(w.nManifolds.p));
    case AG2D_COLOR_STARTS: return get(w.colorStart.p, devCount(&w.dCounters.p->colors) + 1);
    case AG2D_ISLAND_MANIFOLDS: return get(w.isle.p, devCount(w.nIsle.p));
    case AG2D_ISLAND_IDS: return get(w.isleId.p, devCount(w.nIsle.p));
    default: throw ApiError(AG2D_ERR_INVALID_ARG, "unknown field " + std::to_string(field));
    }
}

extern "C" {

int32_t ag2d_world_query_shape(ag2d_world* world, int32_t shape, const float* params, uint32_t trees,
                               uint32_t* out_colliders, uint32_t capacity, uint32_t* out_count)
{
    return guarded([&] {
        if (!world || !params || !out_count) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (shape != AG2D_QUERY_AABB && shape != AG2D_QUERY_CIRCLE)
            throw ApiError(AG2D_ERR_INVALID_ARG, "unknown query shape");
        if (capacity && !out_colliders) throw ApiError(AG2D_ERR_INVALID_ARG, "null output with a capacity");
        CK(cudaSetDevice(world->settings.device));
        ag2d_world& w = *world;
        w.ensureUploaded();
        *out_count = 0;
        const uint32_t n = w.nColliders;
        if (n == 0 || !w.aabbValid || (trees & AG2D_TREE_ALL) == 0) return;
        const cudaStream_t s = w.stream;
        w.queryFlag.reserve(n);
        w.queryOffset.reserve(n);
        w.queryList.reserve(n);
        w.queryCount.reserve(1);
        w.scanner.reserve(std::max({w.pairCap, w.nColliders, w.nBodies}));
        const float4 q = shape == AG2D_QUERY_AABB ? make_float4(params[0], params[1], params[2], params[3])
                                                   : make_float4(params[0], params[1], params[2], 0.0f);
        k_query_shape<<<w.gridFor(n), 256, 0, s>>>(w.caabb.p, w.cbody.p, w.bstate.p, n, uint32_t(shape), q,
                                                   trees & AG2D_TREE_ALL, w.queryFlag.p);
        CK(cudaGetLastError());
        w.scanner.run(w.queryFlag.p, w.queryOffset.p, n, w.queryCount.p, s);
        k_scatter_list<<<w.gridFor(n), 256, 0, s>>>(w.queryFlag.p, w.queryOffset.p, n, w.queryList.p);
        CK(cudaGetLastError());
        uint32_t count = 0;
        CK(cudaMemcpyAsync(&count, w.queryCount.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const uint32_t m = std::min(count, capacity);
        if (m) {
            CK(cudaMemcpyAsync(out_colliders, w.queryList.p, size_t(m) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        *out_count = count;
    });
}

int32_t ag2d_world_query_circle_contacts(ag2d_world* world, float x, float y, float radius, uint32_t trees,
                                         uint32_t* out_colliders, float* out_distance, uint32_t capacity,
                                         uint32_t* out_count)
{
    return guarded([&] {
        if (!world || !out_count) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (capacity && (!out_colliders || !out_distance))
            throw ApiError(AG2D_ERR_INVALID_ARG, "null output with a capacity");
        CK(cudaSetDevice(world->settings.device));
        ag2d_world& w = *world;
        w.ensureUploaded();
        *out_count = 0;
        const uint32_t n = w.nColliders;
        if (n == 0 || !w.aabbValid || (trees & AG2D_TREE_ALL) == 0) return;
        const cudaStream_t s = w.stream;
        w.queryFlag.reserve(n);
        w.queryOffset.reserve(n);
        w.queryList.reserve(n);
        w.queryDist.reserve(n);
        w.queryListDist.reserve(n);
        w.queryCount.reserve(1);
        w.scanner.reserve(std::max({w.pairCap, w.nColliders, w.nBodies}));
        k_circle_contacts<<<w.gridFor(n), 256, 0, s>>>(w.view(), x, y, radius, trees & AG2D_TREE_ALL, w.queryFlag.p,
                                                       w.queryDist.p);
        CK(cudaGetLastError());
        w.scanner.run(w.queryFlag.p, w.queryOffset.p, n, w.queryCount.p, s);
        k_scatter_contacts<<<w.gridFor(n), 256, 0, s>>>(w.queryFlag.p, w.queryOffset.p, w.queryDist.p, n,
                                                        w.queryList.p, w.queryListDist.p);
        CK(cudaGetLastError());
        uint32_t count = 0;
        CK(cudaMemcpyAsync(&count, w.queryCount.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const uint32_t m = std::min(count, capacity);
        if (m) {
            CK(cudaMemcpyAsync(out_colliders, w.queryList.p, size_t(m) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(out_distance, w.queryListDist.p, size_t(m) * sizeof(float), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        *out_count = count;
    });
}

int32_t ag2d_world_read(ag2d_world* world, int32_t field, void* dst, uint64_t cap, uint64_t* out_bytes)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        CK(cudaSetDevice(world->settings.device));
        world->ensureUploaded();
        FieldSpec f;
        if (field_spec(*world, field, f)) {
            // Body and collider fields: the size needs no device access; the values are packed on the device.
            const uint32_t n = f.perCollider ? world->nColliders : world->nBodies;
            const uint64_t bytes = uint64_t(n) * f.outBytes;
            if (out_bytes) *out_bytes = bytes;
            if (dst) {
                if (cap < bytes) throw ApiError(AG2D_ERR_INVALID_ARG, "destination too small");
                read_packed(*world, f, 0, n, 0, dst);
            }
            return;
        }
        uint64_t size = 0;
        const auto bytes = read_field(*world, field, dst == nullptr, &size);
        if (out_bytes) *out_bytes = size;
        if (dst) {
            if (cap < bytes.size()) throw ApiError(AG2D_ERR_INVALID_ARG, "destination too small");
            if (!bytes.empty()) std::memcpy(dst, bytes.data(), bytes.size());
        }
    });
}

int32_t ag2d_world_read_async(ag2d_world* world, int32_t field, void* dst, uint64_t cap, uint64_t* out_bytes)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        CK(cudaSetDevice(world->settings.device));
        world->ensureUploaded();
        FieldSpec f;
        if (!field_spec(*world, field, f))
            throw ApiError(AG2D_ERR_UNSUPPORTED, "asynchronous reads take body and collider fields");
        const uint32_t n = f.perCollider ? world->nColliders : world->nBodies;
        const uint64_t bytes = uint64_t(n) * f.outBytes;
        if (out_bytes) *out_bytes = bytes;
        if (!dst || cap < bytes) throw ApiError(AG2D_ERR_INVALID_ARG, "destination missing or too small");
        if (!page_locked(dst))
            throw ApiError(AG2D_ERR_INVALID_ARG, "asynchronous reads need a page-locked destination (ag2d_host_alloc)");
        read_async(*world, f, 0, n, 0, dst);
    });
}

int32_t ag2d_world_read_wait(ag2d_world* world)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        if (!world->copyStream) return;
        CK(cudaSetDevice(world->settings.device));
        CK(cudaStreamSynchronize(world->copyStream));
    });
}

int32_t ag2d_host_alloc(uint64_t bytes, void** out_ptr)
{
    return guarded([&] {
        if (!out_ptr) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        *out_ptr = nullptr;
        if (bytes == 0) throw ApiError(AG2D_ERR_INVALID_ARG, "zero bytes");
        const cudaError_t e = cudaHostAlloc(out_ptr, bytes, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            *out_ptr = nullptr;
            throw ApiError(e == cudaErrorMemoryAllocation ? AG2D_ERR_OOM : AG2D_ERR_CUDA,
                           std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
        }
    });
}

int32_t ag2d_host_free(void* ptr)
{
    return guarded([&] {
        if (ptr) CK(cudaFreeHost(ptr));
    });
}

int32_t ag2d_world_write(ag2d_world* world, int32_t field, const void* src, uint64_t bytes)
{
    return guarded([&] {
        if (!world || (!src && bytes)) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        ag2d_world& w = *world;
        CK(cudaSetDevice(w.settings.device));
        w.ensureUploaded();
        const cudaStream_t s = w.stream;
        auto set4 = [&](DBuf<float4>& b, int c) {
            if (bytes != uint64_t(w.nBodies) * 4) throw ApiError(AG2D_ERR_INVALID_ARG, "size mismatch");
            auto v = download(b.p, w.nBodies, s);
            const float* f = static_cast<const float*>(src);
            for (uint32_t i = 0; i < w.nBodies; i++) (c == 0 ? v[i].x : c == 1 ? v[i].y : c == 2 ? v[i].z : v[i].w) = f[i];
            b.upload(v.data(), v.size(), s);
        };
        switch (field) {
        case AG2D_BODY_COM_X: set4(w.bpos, 0); break;
        case AG2D_BODY_COM_Y: set4(w.bpos, 1); break;
        case AG2D_BODY_ROTATION: set4(w.bpos, 2); break;
        case AG2D_BODY_VEL_X: set4(w.bvel, 0); break;
        case AG2D_BODY_VEL_Y: set4(w.bvel, 1); break;
        case AG2D_BODY_ANGULAR_VELOCITY: set4(w.bvel, 2); break;
        case AG2D_PAIRS: {
            const uint32_t n = uint32_t(bytes / sizeof(uint2));
            if (n > w.pairCap) w.reserveCapacities(std::max(n, w.pairCap), std::max(n, w.manifoldCap));
            w.pairs.reserve(std::max(n, w.pairCap));
            if (n) CK(cudaMemcpyAsync(w.pairs.p, src, bytes, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(&w.dCounters.p->pairs, &n, 4, cudaMemcpyHostToDevice, s));
            break;
        }
        case AG2D_MANIFOLDS:
        case AG2D_PREV_MANIFOLDS: {
            const uint32_t n = uint32_t(bytes / sizeof(Manifold));
            if (n > w.manifoldCap) w.reserveCapacities(std::max(n, w.pairCap), n);
            const bool prev = field == AG2D_PREV_MANIFOLDS;
            if (n) CK(cudaMemcpyAsync(prev ? w.prevManifolds.p : w.manifolds.p, src, bytes, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(prev ? w.nPrev.p : w.nManifolds.p, &n, 4, cudaMemcpyHostToDevice, s));
            if (prev) {
                w.prevCount = n;
                w.prevHoldsSleepers = false;
                w.prevSegValid = false;
                // Written manifolds carry no solver colour: no colouring hints from them.
                if (n) CK(cudaMemsetAsync(w.prevColor.p, 0xFF, sizeof(uint32_t) * n, s));
            }
            break;
        }
        case AG2D_ISLAND_MANIFOLDS: {   // the store's records; their islands follow with AG2D_ISLAND_IDS
            const uint32_t n = uint32_t(bytes / sizeof(Manifold));
            w.isle.reserve(std::max<uint32_t>(n, 1));
            w.isleId.reserve(std::max<uint32_t>(n, 1));
            if (n) CK(cudaMemcpyAsync(w.isle.p, src, bytes, cudaMemcpyHostToDevice, s));
            CK(cudaMemsetAsync(w.isleId.p, 0xFF, sizeof(uint32_t) * std::max<uint32_t>(n, 1), s));
            CK(cudaMemcpyAsync(w.nIsle.p, &n, 4, cudaMemcpyHostToDevice, s));
            w.isleUpper = n;
            break;
        }
        case AG2D_ISLAND_IDS: {
            uint32_t n = 0;
            CK(cudaMemcpyAsync(&n, w.nIsle.p, 4, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (bytes != uint64_t(n) * 4) throw ApiError(AG2D_ERR_INVALID_ARG, "one island per stored manifold");
            if (n) CK(cudaMemcpyAsync(w.isleId.p, src, bytes, cudaMemcpyHostToDevice, s));
            break;
        }
        default: throw ApiError(AG2D_ERR_INVALID_ARG, "field is not writable");
        }
        CK(cudaStreamSynchronize(s));
    });
}

int32_t ag2d_world_run_phase(ag2d_world* world, int32_t phase)
{
    return guarded([&] {
        if (!world) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
        ag2d_world& w = *world;
        CK(cudaSetDevice(w.settings.device));
        w.ensureUploaded();
        if (w.listsDirty) w.rebuildLists();
        switch (phase) {
        case AG2D_PHASE_INTEGRATE:
            CK(cudaMemsetAsync(w.wrapCount.p, 0, sizeof(float) * std::max<uint32_t>(w.nBodies, 1), w.stream));
            w.snapshot(false);   // the pre-integration poses continuous collision sweeps from
            if (w.nColliders)
                CK(cudaMemcpyAsync(w.prevPose.p, w.cpose.p, sizeof(float4) * w.nColliders, cudaMemcpyDeviceToDevice,
                                   w.stream));
            w.phaseIntegrate();
            break;
        case AG2D_PHASE_CCD:
            CK(cudaMemsetAsync(w.dCounters.p, 0, sizeof(StepCounters), w.stream));
            w.phaseCcd();
            break;
        case AG2D_PHASE_SPATIAL_FULL: w.phasePose(true); break;
        case AG2D_PHASE_SPATIAL_DYNAMIC: w.phasePose(false); break;
        case AG2D_PHASE_BROAD:
            CK(cudaMemsetAsync(w.dCounters.p, 0, sizeof(StepCounters), w.stream));
            w.otherDirty = true;
            w.phaseBroad();
            break;
        case AG2D_PHASE_NARROW: w.phaseNarrow(); break;
        case AG2D_PHASE_COLLIDE: {
            auto pass = [&] {
                CK(cudaMemsetAsync(w.dCounters.p, 0, sizeof(StepCounters), w.stream));
                w.phasePose(false);
                w.phaseBroad();
                w.phaseNarrow(false);
            };
            if (w.profiling) {   // the phase timers record events between the launches: no graph
                pass();
                break;
            }
            // The pass's launches depend on these only; the kernels read their counts on the device.
            auto shape = [&](uint64_t* k) {
                // Any device reallocation (a buffer a captured kernel points at) changes the allocation count.
                const uint64_t v[9] = {w.nDynCol, w.nOther, w.pairCap, w.manifoldCap, w.queryThreads,
                                       w.narrowThreads, uint64_t(w.otherDirty), uint64_t(w.nColliders),
                                       g_deviceAllocs.load(std::memory_order_relaxed)};
                std::copy(v, v + 9, k);
            };
            uint64_t key[9];
            shape(key);
            if (w.collideExec && std::equal(key, key + 9, w.collideKey)) {
                CK(cudaGraphLaunch(w.collideExec, w.stream));
                w.launches += w.collideLaunches;
                break;
            }
            if (w.collideExec) { CK(cudaGraphExecDestroy(w.collideExec)); w.collideExec = nullptr; }
            if (!std::equal(key, key + 9, w.collideSeen)) {
                // A new shape: one pass as it is (it may grow buffers or rebuild the static tree), remembered.
                pass();
                shape(w.collideSeen);
                break;
            }
            // The second pass of a shape: captured (nothing left to allocate), then replayed while the shape holds.
            const uint64_t before = w.launches;
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal));
            try {
                pass();
            } catch (...) {
                cudaStreamEndCapture(w.stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            CK(cudaStreamEndCapture(w.stream, &graph));
            const cudaError_t ie = cudaGraphInstantiate(&w.collideExec, graph, 0);
            cudaGraphDestroy(graph);
            CK(ie);
            w.collideLaunches = w.launches - before;
            std::copy(key, key + 9, w.collideKey);
            CK(cudaGraphLaunch(w.collideExec, w.stream));
            break;
        }
        case AG2D_PHASE_WAKE:
            w.phaseWake();
            w.phaseRestore();
            break;
        case AG2D_PHASE_SOLVE: w.phaseSolve(); break;
        case AG2D_PHASE_ISLANDS: w.phaseIslands(); break;
        case AG2D_PHASE_EVENTS:
            if (w.nWorlds > 1) throw ApiError(AG2D_ERR_UNSUPPORTED, "collision events are per world");
            w.lastEvents.clear();
            w.prepareEvents();
            for (;;) {
                CK(cudaMemsetAsync(w.dCounters.p, 0, sizeof(StepCounters), w.stream));
                w.phaseEvents();
                w.readCounters();
                if (!(w.hCounters->status & STATUS_EVENT_OVERFLOW)) break;
                w.eventCap = std::max<uint32_t>(2 * w.hCounters->events, 2 * w.eventCap);
                w.eventRing.reserve(w.eventCap);
            }
            if (w.hCounters->events) w.collectEvents(w.hCounters->events);
            break;
        default: throw ApiError(AG2D_ERR_INVALID_ARG, "unknown phase");
        }
        w.readCounters();
        if (w.hCounters->status & (STATUS_BARRIER_TIMEOUT | STATUS_LOOKBACK_TIMEOUT))
            throw ApiError(AG2D_ERR_TIMEOUT, "a bounded device-side wait timed out");
        if (w.hCounters->status) throw ApiError(AG2D_ERR_CAPACITY, "phase status " + std::to_string(w.hCounters->status));
    });
}

}  // extern "C"

// Batches: several worlds packed into one engine instance (world-segmented arrays, trees and solver), stepped by
// one launch sequence per step. The source worlds are left as they were.
struct ag2d_batch {
    std::unique_ptr<ag2d_world> engine;
    uint32_t worlds = 0;
};

static bool same_settings(const ag2d_world_settings& a, const ag2d_world_settings& b)
{
    return a.dt == b.dt && a.velocity_iterations == b.velocity_iterations &&
           a.position_iterations == b.position_iterations && a.gravity_x == b.gravity_x &&
           a.gravity_y == b.gravity_y && a.angular_damping == b.angular_damping && a.sleep_speed == b.sleep_speed &&
           a.sleep_time == b.sleep_time && a.ccd == b.ccd && a.device == b.device;
}

extern "C" {

int32_t ag2d_batch_create(ag2d_world* const* worlds, uint32_t count, ag2d_batch** out)
{
    return guarded([&] {
        if (!out || !worlds || count == 0) throw ApiError(AG2D_ERR_INVALID_ARG, "a batch needs at least one world");
        for (uint32_t k = 0; k < count; k++) {
            if (!worlds[k]) throw ApiError(AG2D_ERR_INVALID_ARG, "null world");
            if (!same_settings(worlds[k]->settings, worlds[0]->settings))
                throw ApiError(AG2D_ERR_INVALID_ARG, "worlds of a batch must share their step settings");
        }
        CK(cudaSetDevice(worlds[0]->settings.device));
        PackedArrays all;
        std::vector<uint32_t> bodyStart{0}, colStart{0};
        for (uint32_t k = 0; k < count; k++) {
            PackedArrays one;
            CK(cudaSetDevice(worlds[k]->settings.device));
            worlds[k]->exportArrays(one);
            all.append(one);
            bodyStart.push_back(uint32_t(all.vel.size()));
            colStart.push_back(uint32_t(all.cb.size()));
        }
        std::unique_ptr<ag2d_batch> b(new ag2d_batch());
        b->worlds = count;
        b->engine.reset(new ag2d_world());
        ag2d_world& e = *b->engine;
        e.init(worlds[0]->settings);
        e.nBodies = uint32_t(all.vel.size());
        e.nColliders = uint32_t(all.cb.size());
        e.nWorlds = count;
        e.uploadArrays(all.vel, all.pos, all.rot, all.wc, all.br, all.st, all.state, all.isl, all.cb, all.cs, all.cm,
                       all.co, all.cr, all.bh, all.po, all.pc, all.pv, all.pn, all.mats);
        e.objects.materials.resize(size_t(all.mats.size()) * 3);   // material count for the device view
        for (size_t i = 0; i < all.mats.size(); i++) {
            e.objects.materials[3 * i] = all.mats[i].x;
            e.objects.materials[3 * i + 1] = all.mats[i].y;
            e.objects.materials[3 * i + 2] = all.mats[i].z;
        }
        e.setPartition(bodyStart, colStart);
        if (!all.cp.empty())   // collider poses of stepped worlds (continuous collision detection sweeps from them)
            CK(cudaMemcpyAsync(e.cpose.p, all.cp.data(), all.cp.size() * sizeof(float4), cudaMemcpyHostToDevice,
                               e.stream));
        const uint32_t np = uint32_t(all.prev.size());
        if (np > e.manifoldCap) e.reserveCapacities(std::max(np, e.pairCap), np);
        if (np) CK(cudaMemcpyAsync(e.prevManifolds.p, all.prev.data(), np * sizeof(Manifold), cudaMemcpyHostToDevice,
                                   e.stream));
        if (np) CK(cudaMemcpyAsync(e.prevColor.p, all.pcol.data(), np * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                   e.stream));
        CK(cudaMemcpyAsync(e.nPrev.p, &np, sizeof(uint32_t), cudaMemcpyHostToDevice, e.stream));
        e.prevCount = np;
        const uint32_t ni = uint32_t(all.isle.size());   // sleeping islands' manifolds, world after world
        e.isle.reserve(std::max<uint32_t>(ni, 1));
        e.isleId.reserve(std::max<uint32_t>(ni, 1));
        if (ni) {
            CK(cudaMemcpyAsync(e.isle.p, all.isle.data(), ni * sizeof(Manifold), cudaMemcpyHostToDevice, e.stream));
            CK(cudaMemcpyAsync(e.isleId.p, all.isleId.data(), ni * 4, cudaMemcpyHostToDevice, e.stream));
        }
        CK(cudaMemcpyAsync(e.nIsle.p, &ni, sizeof(uint32_t), cudaMemcpyHostToDevice, e.stream));
        e.isleUpper = ni;
        // Body constraints, world after world within each group (so each world's active constraints keep their
        // order), bodies shifted to the batch's indices; the engine owns new handles.
        for (uint32_t kind = 0; kind < JOINT_KINDS; kind++) {
            JointSystem& dst = e.objects.jointSystems[kind];
            for (uint32_t k = 0; k < count; k++) {
                CK(cudaSetDevice(worlds[k]->settings.device));
                if (kind == JOINT_MOTOR) worlds[k]->pullMotorImpulses();
            }
            CK(cudaSetDevice(e.settings.device));
            for (uint32_t g = 0; g < 3; g++) {
                for (uint32_t k = 0; k < count; k++) {
                    const JointSystem& js = worlds[k]->objects.jointSystems[kind];
                    for (uint32_t i = js.starts[g]; i < js.starts[g + 1]; i++) {
                        HJoint j = js.joints[i];
                        j.bodyA += bodyStart[k];
                        if (j.bodyB != NO_BODY) j.bodyB += bodyStart[k];
                        j.handleSlot = uint32_t(dst.joints.size());
                        dst.slotIndex.push_back(j.handleSlot);
                        dst.slotGeneration.push_back(0);
                        dst.joints.push_back(j);
                    }
                }
                dst.starts[g + 1] = uint32_t(dst.joints.size());
            }
            dst.starts[JGROUP_UNUSED] = uint32_t(dst.joints.size());
            dst.iterations = worlds[0]->objects.jointSystems[kind].iterations;
        }
        e.jointsDirty = e.jointTotal() > 0;
        CK(cudaStreamSynchronize(e.stream));
        *out = b.release();
    });
}

int32_t ag2d_batch_step(ag2d_batch* batch, int32_t steps)
{
    return guarded([&] {
        if (!batch) throw ApiError(AG2D_ERR_INVALID_ARG, "null batch");
        if (steps < 0) throw ApiError(AG2D_ERR_INVALID_ARG, "steps must be >= 0");
        CK(cudaSetDevice(batch->engine->settings.device));
        for (int32_t i = 0; i < steps; i++) batch->engine->stepOnce();
    });
}

int32_t ag2d_batch_engine(ag2d_batch* batch, ag2d_world** out_world)
{
    return guarded([&] {
        if (!batch || !out_world) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        *out_world = batch->engine.get();
    });
}

int32_t ag2d_batch_world_count(ag2d_batch* batch, uint32_t* out_count)
{
    return guarded([&] {
        if (!batch || !out_count) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        *out_count = batch->worlds;
    });
}

int32_t ag2d_batch_read(ag2d_batch* batch, uint32_t world, int32_t field, void* dst, uint64_t cap,
                        uint64_t* out_bytes)
{
    return guarded([&] {
        if (!batch) throw ApiError(AG2D_ERR_INVALID_ARG, "null batch");
        if (world >= batch->worlds) throw ApiError(AG2D_ERR_INVALID_ARG, "world index out of range");
        ag2d_world& e = *batch->engine;
        CK(cudaSetDevice(e.settings.device));
        const uint32_t b0 = e.hBodyStart[world], b1 = e.hBodyStart[world + 1];
        const uint32_t c0 = e.hColStart[world], c1 = e.hColStart[world + 1];
        FieldSpec f;
        if (field_spec(e, field, f)) {
            // The world's range only, packed on the device; sleeping-island ids become world-local.
            const uint32_t lo = f.perCollider ? c0 : b0, hi = f.perCollider ? c1 : b1;
            const uint64_t bytes = uint64_t(hi - lo) * f.outBytes;
            if (out_bytes) *out_bytes = bytes;
            if (dst) {
                if (cap < bytes) throw ApiError(AG2D_ERR_INVALID_ARG, "destination too small");
                read_packed(e, f, lo, hi - lo, b0, dst);
            }
            return;
        }
        std::vector<uint8_t> out;
        if (field == AG2D_MANIFOLDS || field == AG2D_PREV_MANIFOLDS) {
            uint64_t size = 0;
            const std::vector<uint8_t> all = read_field(e, field, false, &size);
            const Manifold* m = reinterpret_cast<const Manifold*>(all.data());
            const size_t n = all.size() / sizeof(Manifold);
            std::vector<Manifold> mine;
            for (size_t i = 0; i < n; i++) {
                if (m[i].a < c0 || m[i].a >= c1) continue;
                Manifold x = m[i];
                x.a -= c0;
                x.b -= c0;
                mine.push_back(x);
            }
            out.resize(mine.size() * sizeof(Manifold));
            if (!mine.empty()) std::memcpy(out.data(), mine.data(), out.size());
        } else if (field == AG2D_ISLAND_MANIFOLDS || field == AG2D_ISLAND_IDS) {
            // The world's stored records (collider indices and island roots made world-local).
            uint64_t size = 0;
            const std::vector<uint8_t> rec = read_field(e, AG2D_ISLAND_MANIFOLDS, false, &size);
            const std::vector<uint8_t> ids = read_field(e, AG2D_ISLAND_IDS, false, &size);
            const Manifold* m = reinterpret_cast<const Manifold*>(rec.data());
            const uint32_t* id = reinterpret_cast<const uint32_t*>(ids.data());
            const size_t n = rec.size() / sizeof(Manifold);
            std::vector<Manifold> mine;
            std::vector<uint32_t> mineId;
            for (size_t i = 0; i < n; i++) {
                if (m[i].a < c0 || m[i].a >= c1) continue;
                Manifold x = m[i];
                x.a -= c0;
                x.b -= c0;
                mine.push_back(x);
                mineId.push_back(id[i] == 0xFFFFFFFFu ? id[i] : id[i] - b0);
            }
            if (field == AG2D_ISLAND_MANIFOLDS) {
                out.resize(mine.size() * sizeof(Manifold));
                if (!mine.empty()) std::memcpy(out.data(), mine.data(), out.size());
            } else {
                out.resize(mineId.size() * 4);
                if (!mineId.empty()) std::memcpy(out.data(), mineId.data(), out.size());
            }
        } else {
            throw ApiError(AG2D_ERR_UNSUPPORTED, "field is not readable per world of a batch");
        }
        if (out_bytes) *out_bytes = out.size();
        if (dst) {
            if (cap < out.size()) throw ApiError(AG2D_ERR_INVALID_ARG, "destination too small");
            if (!out.empty()) std::memcpy(dst, out.data(), out.size());
        }
    });
}

int32_t ag2d_batch_destroy(ag2d_batch* batch)
{
    return guarded([&] {
        if (batch && batch->engine) cudaSetDevice(batch->engine->settings.device);
        delete batch;
    });
}

int32_t ag2d_batch_save(ag2d_batch* batch, void* dst, uint64_t cap, uint64_t* out_bytes)
{
    return guarded([&] {
        if (!batch) throw ApiError(AG2D_ERR_INVALID_ARG, "null batch");
        ag2d_world& e = *batch->engine;
        if (e.jointTotal()) throw ApiError(AG2D_ERR_UNSUPPORTED, "checkpoints hold no body constraints");
        CK(cudaSetDevice(e.settings.device));
        const CkptHeader h = e.checkpointLayout();
        if (out_bytes) *out_bytes = h.totalBytes;
        if (!dst) return;
        if (cap < h.totalBytes) throw ApiError(AG2D_ERR_INVALID_ARG, "destination too small");
        e.saveCheckpoint(h, static_cast<uint8_t*>(dst));
    });
}

// The header of a checkpoint blob, checked against its size and section table.
static CkptHeader checked_checkpoint(const void* src, uint64_t bytes)
{
    CkptHeader h;
    if (bytes < sizeof(h)) throw ApiError(AG2D_ERR_INVALID_ARG, "not a checkpoint (too short)");
    std::memcpy(&h, src, sizeof(h));
    if (std::memcmp(h.magic, CKPT_MAGIC, sizeof(h.magic)) != 0 || h.version != CKPT_VERSION ||
        h.headerBytes != sizeof(CkptHeader))
        throw ApiError(AG2D_ERR_INVALID_ARG, "not a checkpoint of this library version");
    if (h.totalBytes > bytes) throw ApiError(AG2D_ERR_INVALID_ARG, "checkpoint truncated");
    for (uint32_t k = 0; k < NCK; k++)
        if (h.off[k] > h.totalBytes || h.len[k] > h.totalBytes - h.off[k])
            throw ApiError(AG2D_ERR_INVALID_ARG, "checkpoint section out of range");
    if (h.len[CK_WBODY] != (uint64_t(std::max<uint32_t>(h.nWorlds, 1)) + 1) * 4 ||
        h.len[CK_WCOL] != h.len[CK_WBODY] || h.len[CK_VEL] != uint64_t(h.nBodies) * 16 ||
        h.len[CK_CBODY] != uint64_t(h.nColliders) * 4 || h.len[CK_ISLE] != uint64_t(h.nIsle) * sizeof(Manifold) ||
        h.len[CK_ISLEID] != uint64_t(h.nIsle) * 4 || h.len[CK_PREV] != uint64_t(h.nPrev) * sizeof(Manifold))
        throw ApiError(AG2D_ERR_INVALID_ARG, "checkpoint sizes inconsistent");
    return h;
}

int32_t ag2d_batch_restore(const void* src, uint64_t bytes, int32_t device, ag2d_batch** out)
{
    return guarded([&] {
        if (!src || !out) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        const CkptHeader h = checked_checkpoint(src, bytes);
        ag2d_world_settings st = h.settings;
        if (device >= 0) st.device = device;
        std::unique_ptr<ag2d_batch> b(new ag2d_batch());
        b->worlds = std::max<uint32_t>(h.nWorlds, 1);
        b->engine.reset(new ag2d_world());
        b->engine->init(st);
        CK(cudaSetDevice(st.device));
        b->engine->restoreCheckpoint(h, static_cast<const uint8_t*>(src));
        *out = b.release();
    });
}

int32_t ag2d_batch_load(ag2d_batch* batch, const void* src, uint64_t bytes)
{
    return guarded([&] {
        if (!batch || !src) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        const CkptHeader h = checked_checkpoint(src, bytes);
        ag2d_world& e = *batch->engine;
        ag2d_world_settings st = h.settings;
        st.device = e.settings.device;
        if (!same_settings(st, e.settings))
            throw ApiError(AG2D_ERR_INVALID_ARG, "the checkpoint's settings differ from the batch's");
        CK(cudaSetDevice(e.settings.device));
        batch->worlds = std::max<uint32_t>(h.nWorlds, 1);
        e.restoreCheckpoint(h, static_cast<const uint8_t*>(src));
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------
// Request server: one resident batch engine and a host thread that admits, steps and retires requests in rounds.
// ---------------------------------------------------------------------------------------------------------------
namespace {

struct ServerRequest {
    uint64_t id = 0;
    StagedWorld staged;             // dropped once resident
    WorldExtent ext;
    uint64_t bytes = 0;             // device memory estimate
    uint32_t steps = 0, done = 0;
    int32_t state = AG2D_REQUEST_WAITING;
    std::chrono::steady_clock::time_point submitted, finished;
    std::vector<float4> vel, pos;   // final body state
    std::vector<uint8_t> bstate;
};

// Device bytes a resident request may take: its arrays (front and back copies), per-step scratch and the pair /
// manifold capacities reserved per collider (80 bytes a candidate pair, about 330 a manifold slot).
uint64_t request_bytes(const WorldExtent& e)
{
    return uint64_t(e.body) * 200 + uint64_t(e.col) * (200 + INITIAL_PAIRS_PER_COLLIDER * 410) +
           uint64_t(e.vert) * 32 + 4096;
}

}  // namespace

struct ag2d_server {
    ag2d_server_settings settings{};
    std::unique_ptr<ag2d_world> engine;
    std::mutex mu;
    std::condition_variable cv, doneCv;
    std::deque<std::shared_ptr<ServerRequest>> waiting;
    std::vector<std::shared_ptr<ServerRequest>> resident;   // in engine world order
    std::map<uint64_t, std::shared_ptr<ServerRequest>> requests;
    std::thread worker;
    bool stop = false;
    int32_t failCode = AG2D_OK;
    std::string failMessage;
    uint64_t nextId = 1, submitted = 0, completed = 0, rounds = 0, bodySteps = 0, residentBytes = 0;
    uint64_t peakResident = 0;
    double busyMs = 0.0, stepMs = 0.0, repackMs = 0.0;
    std::vector<double> latencies;

    void loop()
    {
        try {
            CK(cudaSetDevice(settings.world.device));
            const uint32_t perRound = settings.steps_per_round ? settings.steps_per_round : 8u;
            while (true) {
                ag2d_world& e = *engine;
                // Finished requests leave; their budget is free for this round's admissions.
                std::vector<uint32_t> keep;
                std::vector<std::shared_ptr<ServerRequest>> leaving;
                uint64_t keptBytes = 0;
                for (uint32_t k = 0; k < resident.size(); k++) {
                    if (resident[k]->done >= resident[k]->steps) {
                        leaving.push_back(resident[k]);
                    } else {
                        keep.push_back(k);
                        keptBytes += resident[k]->bytes;
                    }
                }
                std::vector<std::shared_ptr<ServerRequest>> join;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    if (stop) return;
                    if (resident.empty() && waiting.empty()) {
                        cv.wait_for(lk, std::chrono::milliseconds(20));
                        continue;
                    }
                    // Admission in arrival order under the memory budget and the world limit (a request larger
                    // than the whole budget still runs, alone).
                    uint64_t bytes = keptBytes;
                    size_t worlds = keep.size();
                    while (!waiting.empty()) {
                        const auto& r = waiting.front();
                        const bool fits = bytes + r->bytes <= settings.memory_budget_bytes || worlds == 0;
                        if (!fits || (settings.max_worlds && worlds >= settings.max_worlds)) break;
                        bytes += r->bytes;
                        worlds++;
                        join.push_back(r);
                        waiting.pop_front();
                    }
                }
                const auto t0 = std::chrono::steady_clock::now();
                if (!leaving.empty()) {
                    // The leaving requests' final body state, in one gather and transfer per field.
                    std::vector<uint32_t> idx;
                    for (uint32_t k = 0; k < resident.size(); k++)
                        if (resident[k]->done >= resident[k]->steps) idx.push_back(k);
                    std::vector<float4> vel, pos;
                    std::vector<uint8_t> st;
                    e.exportBodies(idx, vel, pos, st);
                    size_t at = 0;
                    for (const auto& r : leaving) {
                        const size_t nb = r->ext.body;
                        r->vel.assign(vel.begin() + at, vel.begin() + at + nb);
                        r->pos.assign(pos.begin() + at, pos.begin() + at + nb);
                        r->bstate.assign(st.begin() + at, st.begin() + at + nb);
                        at += nb;
                    }
                }
                if (!leaving.empty() || !join.empty()) {
                    std::vector<const StagedWorld*> add;
                    for (const auto& r : join) add.push_back(&r->staged);
                    e.repack(keep, add);
                    std::vector<std::shared_ptr<ServerRequest>> next;
                    for (uint32_t k : keep) next.push_back(resident[k]);
                    for (const auto& r : join) next.push_back(r);
                    std::lock_guard<std::mutex> lk(mu);
                    const auto now = std::chrono::steady_clock::now();
                    for (const auto& r : leaving) {
                        r->state = AG2D_REQUEST_DONE;
                        r->finished = now;
                        completed++;
                        bodySteps += uint64_t(r->ext.body) * r->steps;
                        latencies.push_back(std::chrono::duration<double, std::milli>(now - r->submitted).count());
                    }
                    for (const auto& r : join) {
                        r->state = AG2D_REQUEST_RUNNING;
                        r->staged = StagedWorld();
                    }
                    resident = next;
                    residentBytes = bytesOf(resident);
                    peakResident = std::max<uint64_t>(peakResident, resident.size());
                    doneCv.notify_all();
                }
                if (resident.empty()) continue;
                // A round: as many steps as the closest request still needs, up to the round length.
                uint32_t k = perRound;
                for (const auto& r : resident) k = std::min(k, r->steps - r->done);
                const auto t1 = std::chrono::steady_clock::now();
                for (uint32_t i = 0; i < k; i++) e.stepOnce();
                for (const auto& r : resident) r->done += k;
                const auto t2 = std::chrono::steady_clock::now();
                rounds++;
                repackMs += std::chrono::duration<double, std::milli>(t1 - t0).count();
                stepMs += std::chrono::duration<double, std::milli>(t2 - t1).count();
                busyMs += std::chrono::duration<double, std::milli>(t2 - t0).count();
            }
        } catch (const ApiError& err) {
            std::lock_guard<std::mutex> lk(mu);
            failCode = err.code;
            failMessage = err.what();
        } catch (const std::exception& err) {
            std::lock_guard<std::mutex> lk(mu);
            failCode = AG2D_ERR_CUDA;
            failMessage = err.what();
        }
        doneCv.notify_all();
    }

    static uint64_t bytesOf(const std::vector<std::shared_ptr<ServerRequest>>& v)
    {
        uint64_t b = 0;
        for (const auto& r : v) b += r->bytes;
        return b;
    }

    void checkFailed()
    {
        if (failCode != AG2D_OK) throw ApiError(failCode, "server loop stopped: " + failMessage);
    }
};

extern "C" {

int32_t ag2d_server_create(const ag2d_server_settings* settings, ag2d_server** out)
{
    return guarded([&] {
        if (!settings || !out) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (!(settings->world.dt > 0.0f)) throw ApiError(AG2D_ERR_INVALID_ARG, "dt must be > 0");
        std::unique_ptr<ag2d_server> sv(new ag2d_server());
        sv->settings = *settings;
        sv->engine.reset(new ag2d_world());
        sv->engine->init(settings->world);
        sv->engine->hostDirty = false;
        sv->engine->ensureDevice();
        if (settings->reserve_bodies) sv->engine->reserveResident(settings->reserve_bodies);
        ag2d_server* p = sv.get();
        sv->worker = std::thread([p] { p->loop(); });
        *out = sv.release();
    });
}

int32_t ag2d_server_submit(ag2d_server* server, ag2d_world* world, uint32_t steps, uint64_t* out_request)
{
    return guarded([&] {
        if (!server || !world) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        if (!same_settings(world->settings, server->settings.world))
            throw ApiError(AG2D_ERR_INVALID_ARG, "the request's world settings differ from the server's");
        if (world->jointTotal())
            throw ApiError(AG2D_ERR_UNSUPPORTED, "a world with body constraints cannot join a batch");
        auto r = std::make_shared<ServerRequest>();
        {
            // Packed on the caller's thread: the server loop only copies the blob to the device.
            PackedArrays a;
            world->exportArrays(a);
            r->staged = stage_world(a);
        }
        r->ext = r->staged.ext;
        r->bytes = request_bytes(r->ext);
        r->steps = steps;
        r->submitted = std::chrono::steady_clock::now();
        std::lock_guard<std::mutex> lk(server->mu);
        server->checkFailed();
        r->id = server->nextId++;
        server->requests[r->id] = r;
        server->waiting.push_back(r);
        server->submitted++;
        if (out_request) *out_request = r->id;
        server->cv.notify_all();
    });
}

int32_t ag2d_server_poll(ag2d_server* server, uint64_t request, int32_t* out_state, double* out_latency_ms)
{
    return guarded([&] {
        if (!server) throw ApiError(AG2D_ERR_INVALID_ARG, "null server");
        std::lock_guard<std::mutex> lk(server->mu);
        server->checkFailed();
        auto it = server->requests.find(request);
        if (it == server->requests.end()) throw ApiError(AG2D_ERR_INVALID_ARG, "unknown request");
        const ServerRequest& r = *it->second;
        if (out_state) *out_state = r.state;
        if (out_latency_ms)
            *out_latency_ms = r.state == AG2D_REQUEST_DONE
                                  ? std::chrono::duration<double, std::milli>(r.finished - r.submitted).count()
                                  : -1.0;
    });
}

int32_t ag2d_server_wait_all(ag2d_server* server, double timeout_ms)
{
    return guarded([&] {
        if (!server) throw ApiError(AG2D_ERR_INVALID_ARG, "null server");
        std::unique_lock<std::mutex> lk(server->mu);
        auto done = [&] { return server->failCode != AG2D_OK || server->completed == server->submitted; };
        if (timeout_ms < 0) server->doneCv.wait(lk, done);
        else if (!server->doneCv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done))
            throw ApiError(AG2D_ERR_TIMEOUT, "requests still running after the timeout");
        server->checkFailed();
    });
}

int32_t ag2d_server_read(ag2d_server* server, uint64_t request, int32_t field, void* dst, uint64_t cap,
                         uint64_t* out_bytes)
{
    return guarded([&] {
        if (!server) throw ApiError(AG2D_ERR_INVALID_ARG, "null server");
        std::shared_ptr<ServerRequest> r;
        {
            std::lock_guard<std::mutex> lk(server->mu);
            auto it = server->requests.find(request);
            if (it == server->requests.end()) throw ApiError(AG2D_ERR_INVALID_ARG, "unknown request");
            r = it->second;
            if (r->state != AG2D_REQUEST_DONE) throw ApiError(AG2D_ERR_INVALID_ARG, "request not finished");
        }
        const size_t nb = r->vel.size();
        std::vector<float> f;
        std::vector<uint32_t> u;
        auto comp = [&](const std::vector<float4>& v, int c) {
            f.resize(nb);
            for (size_t i = 0; i < nb; i++) f[i] = c == 0 ? v[i].x : c == 1 ? v[i].y : c == 2 ? v[i].z : v[i].w;
        };
        switch (field) {
        case AG2D_BODY_COM_X: comp(r->pos, 0); break;
        case AG2D_BODY_COM_Y: comp(r->pos, 1); break;
        case AG2D_BODY_ROTATION: comp(r->pos, 2); break;
        case AG2D_BODY_VEL_X: comp(r->vel, 0); break;
        case AG2D_BODY_VEL_Y: comp(r->vel, 1); break;
        case AG2D_BODY_ANGULAR_VELOCITY: comp(r->vel, 2); break;
        case AG2D_BODY_POSE:
            f.resize(nb * 3);
            for (size_t i = 0; i < nb; i++) { f[3 * i] = r->pos[i].x; f[3 * i + 1] = r->pos[i].y; f[3 * i + 2] = r->pos[i].z; }
            break;
        case AG2D_BODY_STATE: u.assign(r->bstate.begin(), r->bstate.end()); break;
        default: throw ApiError(AG2D_ERR_UNSUPPORTED, "field is not kept for finished requests");
        }
        const size_t bytes = field == AG2D_BODY_STATE ? u.size() * 4 : f.size() * 4;
        if (out_bytes) *out_bytes = bytes;
        if (dst) {
            if (cap < bytes) throw ApiError(AG2D_ERR_INVALID_ARG, "destination too small");
            if (bytes) std::memcpy(dst, field == AG2D_BODY_STATE ? static_cast<const void*>(u.data()) : f.data(), bytes);
        }
    });
}

int32_t ag2d_server_release(ag2d_server* server, uint64_t request)
{
    return guarded([&] {
        if (!server) throw ApiError(AG2D_ERR_INVALID_ARG, "null server");
        std::lock_guard<std::mutex> lk(server->mu);
        auto it = server->requests.find(request);
        if (it == server->requests.end()) throw ApiError(AG2D_ERR_INVALID_ARG, "unknown request");
        if (it->second->state != AG2D_REQUEST_DONE) throw ApiError(AG2D_ERR_INVALID_ARG, "request not finished");
        server->requests.erase(it);
    });
}

int32_t ag2d_server_stats_get(ag2d_server* server, ag2d_server_stats* out)
{
    return guarded([&] {
        if (!server || !out) throw ApiError(AG2D_ERR_INVALID_ARG, "null argument");
        std::lock_guard<std::mutex> lk(server->mu);
        out->submitted = server->submitted;
        out->completed = server->completed;
        out->waiting = server->waiting.size();
        out->resident = server->resident.size();
        out->peak_resident = server->peakResident;
        out->rounds = server->rounds;
        out->body_steps = server->bodySteps;
        out->busy_ms = server->busyMs;
        out->step_ms = server->stepMs;
        out->repack_ms = server->repackMs;
        std::vector<double> l = server->latencies;
        std::sort(l.begin(), l.end());
        auto q = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, size_t(p * double(l.size())))]; };
        out->p50_ms = q(0.50);
        out->p99_ms = q(0.99);
        out->max_ms = l.empty() ? 0.0 : l.back();
    });
}

int32_t ag2d_server_destroy(ag2d_server* server)
{
    return guarded([&] {
        if (!server) return;
        {
            std::lock_guard<std::mutex> lk(server->mu);
            server->stop = true;
        }
        server->cv.notify_all();
        if (server->worker.joinable()) server->worker.join();
        cudaSetDevice(server->settings.world.device);
        delete server;
    });
}

}  // extern "C"

static void pull_state(ag2d_world* w)
{
    // Bodies created after the world has run: bring the simulated state back into the host objects first.
    if (w->hostDirty || w->objects.bodies.empty() || w->nBodies != w->objects.bodies.size()) return;
    const cudaStream_t s = w->stream;
    const auto vel = download(w->bvel.p, w->nBodies, s);
    const auto pos = download(w->bpos.p, w->nBodies, s);
    const auto rot = download(w->brot.p, w->nBodies, s);
    const auto tm = download(w->sleepTimer.p, w->nBodies, s);
    for (uint32_t i = 0; i < w->nBodies; i++) {
        HBody& b = w->objects.bodies[i];
        b.vx = vel[i].x; b.vy = vel[i].y; b.w = vel[i].z;
        b.comX = pos[i].x; b.comY = pos[i].y; b.rot = pos[i].z;
        b.cos = rot[i].x; b.sin = rot[i].y; b.sleepTimer = tm[i];
    }
}
