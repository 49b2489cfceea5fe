// guiding_tc.cu -- the batched forward pass of the guiding network on the tcgen05 tensor cores
// (pb2_guide_forward); the tile loop is in guiding_tc.cuh.
#include "guiding_tc.cuh"
#include "pb2_internal.h"

namespace pb2 {
namespace guide {
namespace {

// features: n rows of 12 floats (pos01 xyz, normal xyz, wo xyz, unused); out: n rows of 48 raw outputs
struct FeatureRows {
    static constexpr bool kStaged = true;  // a tile's outputs are contiguous: write them with coalesced stores
    const float* feat;
    float* out;
    __device__ __forceinline__ void features(uint32_t row, float (&f)[9], uint32_t& key) const {
        const float4* p = reinterpret_cast<const float4*>(feat + 12 * (size_t)row);
        const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
        f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w;
        f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
        f[8] = c.x;
        key = row;
    }
    __device__ __forceinline__ void store_tile(uint32_t row0, uint32_t count, const float* staged, int t,
                                               int threads) const {
        const float4* src = reinterpret_cast<const float4*>(staged);
        float4* dst = reinterpret_cast<float4*>(out + (size_t)row0 * kOut);
        const uint32_t n4 = count * (kOut / 4);
        for (uint32_t i = t; i < n4; i += threads) dst[i] = src[i];
    }
    __device__ __forceinline__ void output(uint32_t, const float (&)[kOut]) const {}
};

using FwdLayout = TcLayout<kTcGroupsForward>;

__global__ void __launch_bounds__(FwdLayout::kThreads, 1) k_forward_tc(GuideView gv, const float* __restrict__ features,
                                                                     uint32_t n, float* __restrict__ out,
                                                                     uint32_t* __restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem[];
    forward_tc_tiles<kTcGroupsForward>(gv, n, FeatureRows{ features, out }, error, smem);
}

}  // namespace
}  // namespace guide
cudaError_t guide_forward_tc(const GuideView& gv, const float* features, uint32_t n, float* out, uint32_t* error,
                             cudaStream_t stream) {
    using namespace guide;
    if (n == 0) return cudaSuccess;
    static std::atomic<int> attr[kMaxDevices];
    const cudaError_t e = smem_attr_once((const void*)k_forward_tc, forward_tc_smem<kTcGroupsForward>(), attr);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const int grid = (int)std::min<uint32_t>((tiles + kTcGroupsForward - 1) / kTcGroupsForward, (uint32_t)sms);
    k_forward_tc<<<grid, FwdLayout::kThreads, forward_tc_smem<kTcGroupsForward>(), stream>>>(gv, features, n, out,
                                                                                              error);
    return cudaGetLastError();
}

}  // namespace pb2
