// guiding_tc.cu -- the batched forward pass of the guiding network on the tcgen05 tensor cores
// (pb2_guide_forward); the tile loop is in guiding_tc.cuh.
#include "guiding_tc.cuh"
#include "pb2_internal.h"

namespace pb2 {
namespace guide {
namespace {

// features: n rows of 12 floats (pos01 xyz, normal xyz, wo xyz, unused); out: n rows of 48 raw outputs
struct FeatureRows {
    const float* feat;
    float* out;
    __device__ __forceinline__ void features(uint32_t row, float (&f)[9], uint32_t& key) const {
        for (int i = 0; i < 9; ++i) f[i] = feat[12 * (size_t)row + i];
        key = row;
    }
    __device__ __forceinline__ void output(uint32_t key, const float (&y)[kOut]) const {
        float* o = out + (size_t)key * kOut;
#pragma unroll
        for (int i = 0; i < kOut; i += 4) *reinterpret_cast<float4*>(o + i) = make_float4(y[i], y[i + 1], y[i + 2], y[i + 3]);
    }
};

__global__ void __launch_bounds__(kTcThreads) k_forward_tc(GuideView gv, const float* __restrict__ features, uint32_t n,
                                                           float* __restrict__ out, uint32_t* __restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem[];
    forward_tc_tiles(gv, n, FeatureRows{ features, out }, error, smem);
}

}  // namespace
}  // namespace guide
cudaError_t guide_forward_tc(const GuideView& gv, const float* features, uint32_t n, float* out, uint32_t* error,
                             cudaStream_t stream) {
    using namespace guide;
    if (n == 0) return cudaSuccess;
    static std::atomic<int> attr[kMaxDevices];
    const cudaError_t e = smem_attr_once((const void*)k_forward_tc, forward_tc_smem(), attr);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const int grid = (int)std::min<uint32_t>(tiles, (uint32_t)sms * 2u);
    k_forward_tc<<<grid, kTcThreads, forward_tc_smem(), stream>>>(gv, features, n, out, error);
    return cudaGetLastError();
}

}  // namespace pb2
