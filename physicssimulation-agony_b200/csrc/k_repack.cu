// Batch repacking for the request server: the resident worlds' arrays are rebuilt on the device from the current
// arrays (worlds that stay) and the staged blobs of the worlds that join (one blob per world, one section per
// array, at the byte offsets of a [world][section] table), one gather per array. Every world keeps its
// elements in order; only the indices stored inside the records move with their targets (body of a collider, shape
// of a collider, material, polygon vertex offset, sleeping island, colliders of a warm-start manifold).
#include "ag2d_kernels.cuh"

namespace ag2d {

// Destination element e lies in the last segment whose dst <= e (segments sorted by dst, covering [0, total)).
__device__ __forceinline__ uint32_t find_segment(const GatherSeg* segs, uint32_t nsegs, uint32_t e)
{
    uint32_t lo = 0, hi = nsegs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (segs[mid].dst <= e) lo = mid; else hi = mid;
    }
    return lo;
}

template <class T>
__device__ __forceinline__ T remap(T v, const GatherSeg&, uint32_t) { return v; }

template <>
__device__ __forceinline__ uint32_t remap<uint32_t>(uint32_t v, const GatherSeg& g, uint32_t mode)
{
    switch (mode) {
    case GATHER_ISLAND: return v == 0xFFFFFFFFu ? v : uint32_t(int32_t(v) + g.dBody);
    case GATHER_BODY: return uint32_t(int32_t(v) + g.dBody);
    case GATHER_SHAPE: {
        const uint32_t type = shape_type(v);
        // Boxes and capsules share one parameter table.
        const int32_t d = type == SHAPE_CIRCLE ? g.dCircle : (type == SHAPE_POLYGON ? g.dPoly : g.dBox);
        return (type << 30) | uint32_t(int32_t(shape_index(v)) + d);
    }
    case GATHER_MATERIAL: return uint32_t(int32_t(v) + g.dMat);
    case GATHER_VERTEX: return uint32_t(int32_t(v) + g.dVert);
    default: return v;
    }
}

template <>
__device__ __forceinline__ Manifold remap<Manifold>(Manifold v, const GatherSeg& g, uint32_t)
{
    v.a = uint32_t(int32_t(v.a) + g.dCol);
    v.b = uint32_t(int32_t(v.b) + g.dCol);
    return v;
}

// A staged segment (fromNew) starts at byte offset sections[src * nsec + section] of srcNew; sections are aligned
// to 64 bytes, a multiple of every element size gathered here.
template <class T>
__global__ void k_gather(T* __restrict__ dst, const T* __restrict__ srcOld, const T* __restrict__ srcNew,
                         const GatherSeg* __restrict__ segs, uint32_t nsegs, uint32_t total, uint32_t mode,
                         const unsigned long long* __restrict__ sections, uint32_t nsec, uint32_t section)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const GatherSeg g = segs[find_segment(segs, nsegs, e)];
        const T* src = srcOld;
        unsigned long long base = g.src;
        if (g.fromNew) {
            src = srcNew;
            base = sections[(unsigned long long)g.src * nsec + section] / sizeof(T);
        }
        dst[e] = remap<T>(src[base + (e - g.dst)], g, mode);
    }
}

template <class T>
cudaError_t launch_gather(T* dst, const T* srcOld, const T* srcNew, const GatherSeg* segs, uint32_t nsegs,
                          uint32_t total, uint32_t mode, uint32_t grid, cudaStream_t stream,
                          const unsigned long long* sections, uint32_t nsec, uint32_t section)
{
    if (total == 0) return cudaSuccess;
    k_gather<T><<<grid, 256, 0, stream>>>(dst, srcOld, srcNew, segs, nsegs, total, mode, sections, nsec, section);
    return cudaGetLastError();
}

template cudaError_t launch_gather<float4>(float4*, const float4*, const float4*, const GatherSeg*, uint32_t,
                                           uint32_t, uint32_t, uint32_t, cudaStream_t, const unsigned long long*,
                                           uint32_t, uint32_t);
template cudaError_t launch_gather<float2>(float2*, const float2*, const float2*, const GatherSeg*, uint32_t,
                                           uint32_t, uint32_t, uint32_t, cudaStream_t, const unsigned long long*,
                                           uint32_t, uint32_t);
template cudaError_t launch_gather<float>(float*, const float*, const float*, const GatherSeg*, uint32_t,
                                           uint32_t, uint32_t, uint32_t, cudaStream_t, const unsigned long long*,
                                           uint32_t, uint32_t);
template cudaError_t launch_gather<uint8_t>(uint8_t*, const uint8_t*, const uint8_t*, const GatherSeg*, uint32_t,
                                           uint32_t, uint32_t, uint32_t, cudaStream_t, const unsigned long long*,
                                           uint32_t, uint32_t);
template cudaError_t launch_gather<uint32_t>(uint32_t*, const uint32_t*, const uint32_t*, const GatherSeg*, uint32_t,
                                           uint32_t, uint32_t, uint32_t, cudaStream_t, const unsigned long long*,
                                           uint32_t, uint32_t);
template cudaError_t launch_gather<Manifold>(Manifold*, const Manifold*, const Manifold*, const GatherSeg*, uint32_t,
                                           uint32_t, uint32_t, uint32_t, cudaStream_t, const unsigned long long*,
                                           uint32_t, uint32_t);

// World of each element: the last world whose start is <= the element (starts sorted, [worlds + 1]).
__global__ void k_world_of(const uint32_t* __restrict__ starts, uint32_t worlds, uint32_t n, uint32_t* __restrict__ out)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = worlds;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (starts[mid] <= e) lo = mid; else hi = mid;
        }
        out[e] = lo;
    }
}

__global__ void k_fill_u32(uint32_t* __restrict__ out, uint32_t n, uint32_t value)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) out[e] = value;
}

// Packs elements [lo, lo + n) of one field into the dense layout a host read returns, so that the transfer carries
// only the bytes the caller asked for (a float4 record's component is 4 of its 16 bytes).
__global__ void k_extract(const void* __restrict__ src, uint32_t lo, uint32_t n, uint32_t kind, uint32_t comp,
                          uint32_t bias, void* __restrict__ out)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t i = lo + e;
        switch (kind) {
        case EXTRACT_F4_COMP:
            static_cast<float*>(out)[e] = static_cast<const float*>(src)[4 * size_t(i) + comp];
            break;
        case EXTRACT_F4_XYZ: {
            const float4 v = static_cast<const float4*>(src)[i];
            float* o = static_cast<float*>(out) + 3 * size_t(e);
            o[0] = v.x;
            o[1] = v.y;
            o[2] = v.z;
            break;
        }
        case EXTRACT_F2_COMP:
            static_cast<float*>(out)[e] = static_cast<const float*>(src)[2 * size_t(i) + comp];
            break;
        case EXTRACT_U8_U32:
            static_cast<uint32_t*>(out)[e] = static_cast<const uint8_t*>(src)[i];
            break;
        case EXTRACT_ISLAND: {
            const uint32_t v = static_cast<const uint32_t*>(src)[i];
            static_cast<uint32_t*>(out)[e] = v == 0xFFFFFFFFu ? v : v - bias;
            break;
        }
        default:
            break;
        }
    }
}

}  // namespace ag2d
