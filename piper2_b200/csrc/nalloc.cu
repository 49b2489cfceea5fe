// nalloc.cu -- closest-hit tracing for callers that cannot allocate device memory.
//
// Some host applications cannot let a library call cudaMalloc/cudaFree: they run on a fixed device
// memory budget handed out by their own allocator, or they cannot afford the implicit device-wide
// synchronisation those calls carry in the middle of a frame.  pb2_trace_closest_nalloc serves them:
// it builds the 8-wide BVH over the caller's triangles and traces the caller's rays with every
// intermediate buffer (build temporaries, the BVH itself, the trace work counter) carved from one
// file-scope device array of fixed size, so the call allocates nothing.
//
// The array is a static __device__ symbol: every GPU that loads this library holds it until the
// process exits.  Host code cannot take its address directly (the host-side symbol is only a stand-in),
// so the first call on each device looks the device address up with cudaGetSymbolAddress, with that
// device current, and caches it per device.  The cached address belongs to the device's primary
// context: after cudaDeviceReset the array may live elsewhere, so the call must not be used across a
// reset of a device it has already run on.
//
// A traversal whose 48-entry stack overflows drops nodes; the call then returns
// PB2_ERR_QUEUE_OVERFLOW instead of hits that could be wrong.  Reading that flag back needs the trace
// to finish, so the call returns after the work it queued is done.
#include <mutex>

#include "pb2_internal.h"

namespace pb2 {
namespace {

constexpr uint32_t kNallocMaxTriangles = 16384;
constexpr size_t kNallocScratchBytes = 8u << 20;  // 8 MiB

static __device__ __align__(256) unsigned char g_nalloc_scratch[kNallocScratchBytes];

std::mutex g_nalloc_mutex;
void* g_nalloc_ptr[kMaxDevices] = {};

__global__ void k_pack_triangles(const float* __restrict__ tri, uint32_t n, TriSlot* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* t = tri + 9 * (size_t)i;
    TriSlot s;
    s.v0 = make_float4(t[0], t[1], t[2], __uint_as_float(i));
    s.v1 = make_float4(t[3], t[4], t[5], 0.0f);
    s.v2 = make_float4(t[6], t[7], t[8], 0.0f);
    out[i] = s;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace
}  // namespace pb2

using namespace pb2;

extern "C" int pb2_trace_closest_nalloc(const float* triangles_dev, uint32_t tri_count, const pb2_ray* rays_dev,
                                        uint32_t n, pb2_hit* hits_dev, void* stream_ptr) {
    if (tri_count > kNallocMaxTriangles)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_trace_closest_nalloc: at most 16384 triangles (its fixed device "
                                              "scratch is sized for that); use pb2_accel_create for larger meshes");
    if ((tri_count && !triangles_dev) || (n && (!rays_dev || !hits_dev)))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_trace_closest_nalloc: null argument");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(PB2_ERR_NOT_SUPPORTED, "device index out of range");
    char* base;
    {
        std::lock_guard<std::mutex> lock(g_nalloc_mutex);
        if (!g_nalloc_ptr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_nalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the static scratch");
            g_nalloc_ptr[dev] = ptr;
        }
        base = static_cast<char*>(g_nalloc_ptr[dev]);
    }
    // carve: packed input triangles | BVH nodes | leaf triangles | trace work counters | build scratch
    const size_t m = tri_count ? tri_count : 1;
    char* p = base;
    TriSlot* tin = reinterpret_cast<TriSlot*>(p);
    p += align256(sizeof(TriSlot) * m);
    WideNode* nodes = reinterpret_cast<WideNode*>(p);
    p += align256(sizeof(WideNode) * m);
    TriSlot* tris = reinterpret_cast<TriSlot*>(p);
    p += align256(sizeof(TriSlot) * m);
    uint32_t* work = reinterpret_cast<uint32_t*>(p);
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(p + 64);
    uint32_t* error_flag = reinterpret_cast<uint32_t*>(p + 128);
    p += 256;
    const size_t used = (size_t)(p - base);
    const size_t build_bytes = build_scratch_bytes(tri_count);
    if (used + build_bytes > kNallocScratchBytes)
        return fail(PB2_ERR_NOT_SUPPORTED, "pb2_trace_closest_nalloc: static scratch too small on this device");
    // the array keeps the previous call's contents: reset what the kernels expect to start at zero
    if ((e = cudaMemsetAsync(work, 0, 256, stream))) return cuda_fail(e, "clear nalloc counters");
    uint32_t node_count = 0;
    if (tri_count) {
        k_pack_triangles<<<(tri_count + 255) / 256, 256, 0, stream>>>(triangles_dev, tri_count, tin);
        if ((e = cudaGetLastError())) return cuda_fail(e, "k_pack_triangles");
        e = build_wide_bvh_prealloc(tin, tri_count, nodes, tris, p, kNallocScratchBytes - used, stream, &node_count);
        if (e != cudaSuccess) return cuda_fail(e, "BVH build (static scratch)");
    }
    BvhView view{};
    view.nodes = nodes;
    view.tris = tris;
    view.planes = nullptr;
    view.node_count = node_count;
    view.tri_count = tri_count;
    view.plane_count = 0;
    view.root_is_leaf = tri_count <= 1;
    e = launch_trace_api(view, rays_dev, n, hits_dev, nullptr, true, false, work, counters, error_flag, stream);
    if (e != cudaSuccess) return cuda_fail(e, "trace launch (static scratch)");
    // the stack-overflow flag, into pageable host memory (no allocation), after the trace
    uint32_t overflow = 0;
    if ((e = cudaMemcpyAsync(&overflow, error_flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)))
        return cuda_fail(e, "read the nalloc traversal flag");
    if ((e = cudaStreamSynchronize(stream))) return cuda_fail(e, "pb2_trace_closest_nalloc");
    if (overflow)
        return fail(PB2_ERR_QUEUE_OVERFLOW, "pb2_trace_closest_nalloc: a ray's traversal stack overflowed (BVH "
                                            "deeper than 48 entries); its hits are not valid");
    return PB2_OK;
}
