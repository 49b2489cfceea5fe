// traverse.cu -- persistent closest-hit / any-hit kernels over batches of rays.
//
// Each warp keeps 32 rays in flight.  When at least kRefill lanes have finished, the warp fetches
// that many new rays with one atomic on the work counter and hands them to the idle lanes (warp-level
// compaction of the active ray set, as in Aila and Laine, HPG 2009, "dynamic fetch").  Lanes run
// kSteps traversal iterations between refill checks (kSteps and kRefill were tuned on a B200).
#include "pb2_internal.h"
#include "traverse.cuh"

namespace pb2 {

constexpr int kTraceThreads = 128;
#ifndef PB2_TRACE_REFILL
#define PB2_TRACE_REFILL 4
#endif
#ifndef PB2_TRACE_STEPS
#define PB2_TRACE_STEPS 4
#endif
constexpr int kRefill = PB2_TRACE_REFILL;
constexpr int kSteps = PB2_TRACE_STEPS;
// Resident blocks per SM the register budget is sized for, closest hit / any hit (tuned on a B200:
// 10 / 9 of 8-12 tried).
#ifndef PB2_TRACE_MIN_BLOCKS
#define PB2_TRACE_MIN_BLOCKS 10
#endif
#ifndef PB2_TRACE_MIN_BLOCKS_ANY
#define PB2_TRACE_MIN_BLOCKS_ANY 9
#endif
constexpr int kMinBlocks = PB2_TRACE_MIN_BLOCKS;
constexpr int kMinBlocksAny = PB2_TRACE_MIN_BLOCKS_ANY;

struct ApiRays {
    const float4* rays;
    pb2_hit* hits;
    uint32_t* occluded;
    __device__ __forceinline__ void load(uint32_t i, float4& a, float4& b) const {
        a = __ldg(rays + 2 * i);
        b = __ldg(rays + 2 * i + 1);
    }
};

template <bool kClosest, bool kCount>
__global__ void __launch_bounds__(kTraceThreads, kClosest ? kMinBlocks : kMinBlocksAny) k_trace_api(BvhView bvh, ApiRays io, uint32_t n, uint32_t* work,
                                                              unsigned long long* counters, uint32_t* error_flag) {
    __shared__ uint2 stack_smem[kSharedStack * kTraceThreads];
    Traverser<kClosest, kCount, kTraceThreads> tr;
    tr.bind_stack(stack_smem);
    bool active = false;
    uint32_t ray_index = 0;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t nv = 0, nt = 0;
    for (;;) {
        const unsigned inactive = __ballot_sync(0xFFFFFFFFu, !active);
        if (__popc(inactive) >= kRefill) {
            const int leader = __ffs(inactive) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(work, (uint32_t)__popc(inactive));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (!active) {
                const uint32_t idx = base + __popc(inactive & lt_mask);
                if (idx < n) {
                    float4 a, b;
                    io.load(idx, a, b);
                    tr.init(bvh, a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w);
                    ray_index = idx;
                    active = true;
                }
            }
            if (__ballot_sync(0xFFFFFFFFu, active) == 0u) break;
        }
        if (active) {
            // not unrolled: copies of the traversal body would overflow the instruction cache
#pragma unroll 1
            for (int it = 0; it < kSteps && !tr.done; ++it) tr.iteration(bvh);
            if (tr.done) {
                if (kCount) { nv += tr.node_visits; nt += tr.tri_tests; }
                if (tr.overflow) atomicOr(error_flag, 1u);
                if (kClosest) {
                    bool front;
                    tr.finish_planes(bvh, front);
                    pb2_hit h;
                    h.t = tr.tbest;
                    h.prim = tr.best_prim;
                    h.u = tr.bu;
                    h.v = tr.bv;
                    reinterpret_cast<float4*>(io.hits)[ray_index] =
                        make_float4(h.t, __uint_as_float(h.prim), h.u, h.v);
                } else {
                    io.occluded[ray_index] = tr.best_prim != kInvalidPrim ? 1u : 0u;
                }
                active = false;
            }
        }
    }
    if (kCount) {
        for (int o = 16; o > 0; o >>= 1) {
            nv += __shfl_xor_sync(0xFFFFFFFFu, nv, o);
            nt += __shfl_xor_sync(0xFFFFFFFFu, nt, o);
        }
        if (lane == 0) {
            atomicAdd(counters + 0, (unsigned long long)nv);
            atomicAdd(counters + 1, (unsigned long long)nt);
        }
    }
}

cudaError_t launch_trace_api(const BvhView& bvh, const pb2_ray* rays, uint32_t n, pb2_hit* hits, uint32_t* occluded,
                             bool closest, bool count, uint32_t* work, unsigned long long* counters,
                             uint32_t* error_flag, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    cudaError_t err = cudaMemsetAsync(work, 0, sizeof(uint32_t), stream);
    if (err != cudaSuccess) return err;
    ApiRays io{ reinterpret_cast<const float4*>(rays), hits, occluded };
    const void* kernel;
    if (closest) kernel = count ? (const void*)k_trace_api<true, true> : (const void*)k_trace_api<true, false>;
    else kernel = count ? (const void*)k_trace_api<false, true> : (const void*)k_trace_api<false, false>;
    static std::atomic<int> blocks[4][kMaxDevices];
    const int slot = (closest ? 2 : 0) + (count ? 1 : 0);
    int grid = resident_grid_cached(kernel, kTraceThreads, 0, blocks[slot]);
    const int needed = (int)((n + kTraceThreads - 1) / kTraceThreads);
    if (grid > needed) grid = needed;
    if (closest) {
        if (count) k_trace_api<true, true><<<grid, kTraceThreads, 0, stream>>>(bvh, io, n, work, counters, error_flag);
        else k_trace_api<true, false><<<grid, kTraceThreads, 0, stream>>>(bvh, io, n, work, counters, error_flag);
    } else {
        if (count) k_trace_api<false, true><<<grid, kTraceThreads, 0, stream>>>(bvh, io, n, work, counters, error_flag);
        else k_trace_api<false, false><<<grid, kTraceThreads, 0, stream>>>(bvh, io, n, work, counters, error_flag);
    }
    return cudaGetLastError();
}

}  // namespace pb2
