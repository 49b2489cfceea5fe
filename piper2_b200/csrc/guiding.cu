// guiding.cu -- the guiding network as a library object: parameters, batched forward, the loss gradient
// over a batch of radiance samples, and Adam.  The integrator (render.cu) evaluates the same network
// inside its bounce loop and feeds training samples back.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "guiding.cuh"
#include "pb2_internal.h"

namespace pb2 {
namespace guide {

// features: n rows of 12 floats (pos01 xyz, normal xyz, wo xyz, unused); out: n rows of 48 raw outputs
__global__ void __launch_bounds__(kThreads) k_forward(GuideView gv, const float* __restrict__ features, uint32_t n,
                                                      float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* w_s = reinterpret_cast<__nv_bfloat16*>(smem);
    float* b_s = reinterpret_cast<float*>(smem + kW16Elems * 2);
    FwdTile* tiles = reinterpret_cast<FwdTile*>(smem + kW16Elems * 2 + kBiasElems * 4);
    load_weights(gv, w_s, b_s);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    FwdTile& T = tiles[warp];
    const uint32_t tiles_total = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * kWarps + warp; tile < tiles_total; tile += gridDim.x * kWarps) {
        const uint32_t row0 = tile * 16;
        if (lane < 16) {
            float f[9] = { 0, 0, 0, 0, 0, 1, 0, 0, 1 };
            if (row0 + lane < n)
                for (int i = 0; i < 9; ++i) f[i] = features[12 * (size_t)(row0 + lane) + i];
            encode_row(f, T.x + lane * kXStride);
        }
        __syncwarp();
        forward_tile(w_s, b_s, T.x, T.h[0], T.h[1], T.y);
        for (int i = lane; i < 16 * kOut; i += 32) {
            const uint32_t r = row0 + i / kOut;
            if (r < n) out[(size_t)r * kOut + i % kOut] = T.y[i];
        }
        __syncwarp();
    }
}

__global__ void k_weight_sum(const float* __restrict__ rec, uint32_t n, float* scalars) {
    float s = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += rec[16 * (size_t)i + 12];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&scalars[0], s);
}

// records: n rows of 16 floats (pos01 xyz, normal xyz, wo xyz, wi xyz, weight, unused x3)
__global__ void __launch_bounds__(kThreads) k_gradient(GuideView gv, const float* __restrict__ rec, uint32_t n,
                                                       const float* __restrict__ scalars, float* __restrict__ grad,
                                                       float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* w_s = reinterpret_cast<__nv_bfloat16*>(smem);
    float* b_s = reinterpret_cast<float*>(smem + kW16Elems * 2);
    float* g_s = b_s + kBiasElems;  // kParams floats, flat parameter layout
    TrainTile* tiles = reinterpret_cast<TrainTile*>(g_s + kParams);
    load_weights(gv, w_s, b_s);
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) g_s[i] = 0.f;
    __syncthreads();
    const float wsum = scalars[0];
    const float gscale = -(wsum > 0.f ? (float)n / wsum : 1.f) / (float)n;  // -(w / mean w) / B = -w * gscale'
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TrainTile& T = tiles[warp];
    float loss_acc = 0.f;
    const uint32_t tiles_total = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * kWarps + warp; tile < tiles_total; tile += gridDim.x * kWarps) {
        const uint32_t row0 = tile * 16;
        if (lane < 16) {
            float* f = T.feat + lane * 16;
            if (row0 + lane < n) {
                for (int i = 0; i < 16; ++i) f[i] = rec[16 * (size_t)(row0 + lane) + i];
            } else {
                for (int i = 0; i < 16; ++i) f[i] = 0.f;
                f[5] = 1.f; f[8] = 1.f; f[11] = 1.f;  // unit directions, zero weight
            }
            encode_row(f, T.x + lane * kXStride);
        }
        __syncwarp();
        const __nv_bfloat16* x = T.x;
        dense_forward<kIn, kHid, true>(x, kXStride, w_s + w16_offset(0), layer_stride(0), b_s + bias_offset(0), T.h[0],
                                       kHStride, nullptr, 0);
        __syncwarp();
        for (int l = 1; l < 4; ++l) {
            dense_forward<kHid, kHid, true>(T.h[l - 1], kHStride, w_s + w16_offset(l), layer_stride(l),
                                            b_s + bias_offset(l), T.h[l], kHStride, nullptr, 0);
            __syncwarp();
        }
        dense_forward<kHid, kOut, false>(T.h[3], kHStride, w_s + w16_offset(4), layer_stride(4), b_s + bias_offset(4),
                                         nullptr, 0, T.y, kOut);
        __syncwarp();
        // loss gradient per row: dY (bf16, 16 x 48 in dz[0]) and the output-layer bias gradient
        if (lane < 16) {
            const float* f = T.feat + lane * 16;
            const float g = f[12] * gscale;
            float dy[kOut];
            const float lq = mixture_loss_grad(T.y + lane * kOut, f[9], f[10], f[11], g, dy);
            if (row0 + lane < n) loss_acc += g * lq;
            __nv_bfloat16* d = T.dz[0] + lane * kHStride;
            for (int i = 0; i < kOut; ++i) {
                d[i] = __float2bfloat16_rn(dy[i]);
                if (dy[i] != 0.f) atomicAdd(&g_s[param_offset(4) + kOut * kHid + i], dy[i]);
            }
        }
        __syncwarp();
        // output layer
        dense_backward_weight<kHid, kOut>(T.dz[0], kHStride, T.h[3], kHStride, g_s + param_offset(4));
        dense_backward_data<kHid, kOut>(T.dz[0], kHStride, w_s + w16_offset(4), layer_stride(4), T.h[3], kHStride,
                                        T.dz[1], kHStride);
        __syncwarp();
        int cur = 1;
        for (int l = 3; l >= 0; --l) {
            // bias gradient of layer l: column sums of dZ_l
            for (int c = lane; c < kHid; c += 32) {
                float s = 0.f;
                for (int r = 0; r < 16; ++r) s += __bfloat162float(T.dz[cur][r * kHStride + c]);
                atomicAdd(&g_s[param_offset(l) + layer_out(l) * layer_in(l) + c], s);
            }
            const __nv_bfloat16* in = l == 0 ? T.x : T.h[l - 1];
            const int ins = l == 0 ? kXStride : kHStride;
            if (l == 0) {
                dense_backward_weight<kIn, kHid>(T.dz[cur], kHStride, in, ins, g_s + param_offset(0));
            } else {
                dense_backward_weight<kHid, kHid>(T.dz[cur], kHStride, in, ins, g_s + param_offset(l));
                dense_backward_data<kHid, kHid>(T.dz[cur], kHStride, w_s + w16_offset(l), layer_stride(l), T.h[l - 1],
                                                kHStride, T.dz[cur ^ 1], kHStride);
            }
            __syncwarp();
            cur ^= 1;
        }
    }
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xFFFFFFFFu, loss_acc, o);
    if (lane == 0 && loss_acc != 0.f) atomicAdd(loss, loss_acc);
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
        if (g_s[i] != 0.f) atomicAdd(&grad[i], g_s[i]);
}

// Adam on the flat fp32 parameters; refreshes the bf16 weight image and fp32 biases.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, float* __restrict__ grad,
                       float lr, float bc1, float bc2, __nv_bfloat16* __restrict__ w16, float* __restrict__ b32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float g = grad[i];
    grad[i] = 0.f;
    const float mi = kBeta1 * m[i] + (1.f - kBeta1) * g;
    const float vi = kBeta2 * v[i] + (1.f - kBeta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + kEps);
    p[i] = pi;
    int l = 0;
    while (l < kLayers - 1 && i >= param_offset(l + 1)) ++l;
    const int local = i - param_offset(l);
    const int nw = layer_out(l) * layer_in(l);
    if (local < nw) {
        const int o = local / layer_in(l), c = local % layer_in(l);
        w16[w16_offset(l) + o * layer_stride(l) + c] = __float2bfloat16_rn(pi);
    } else {
        b32[bias_offset(l) + (local - nw)] = pi;
    }
}

// writes the bf16 weight image (pad columns stay as cleared) and the fp32 biases from the parameters
__global__ void k_image(const float* __restrict__ p, __nv_bfloat16* __restrict__ w16, float* __restrict__ b32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    int l = 0;
    while (l < kLayers - 1 && i >= param_offset(l + 1)) ++l;
    const int local = i - param_offset(l);
    const int nw = layer_out(l) * layer_in(l);
    if (local < nw) w16[w16_offset(l) + (local / layer_in(l)) * layer_stride(l) + local % layer_in(l)] =
        __float2bfloat16_rn(p[i]);
    else b32[bias_offset(l) + (local - nw)] = p[i];
}

size_t forward_smem() { return kW16Elems * 2 + kBiasElems * 4 + sizeof(FwdTile) * kWarps; }
size_t gradient_smem() { return kW16Elems * 2 + kBiasElems * 4 + kParams * 4 + sizeof(TrainTile) * kWarps; }

}  // namespace guide

cudaError_t guide_forward(const GuideView& gv, const float* features, uint32_t n, float* out, cudaStream_t stream) {
    using namespace guide;
    if (n == 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)forward_smem());
        attr = true;
    }
    const uint32_t tiles = (n + 15) / 16;
    const int grid = (int)std::min<uint32_t>((tiles + kWarps - 1) / kWarps, 148u * 2u);
    k_forward<<<grid, kThreads, forward_smem(), stream>>>(gv, features, n, out);
    return cudaGetLastError();
}

cudaError_t guide_gradient(const GuideView& gv, const float* records, uint32_t n, float* grad, float* scalars,
                           cudaStream_t stream) {
    using namespace guide;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gradient, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gradient_smem());
        attr = true;
    }
    cudaError_t e = cudaMemsetAsync(scalars, 0, 2 * sizeof(float), stream);
    if (e != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    k_weight_sum<<<128, 256, 0, stream>>>(records, n, scalars);
    const uint32_t tiles = (n + 15) / 16;
    const int grid = (int)std::min<uint32_t>((tiles + kWarps - 1) / kWarps, 148u);
    k_gradient<<<grid, kThreads, gradient_smem(), stream>>>(gv, records, n, scalars, grad, scalars + 1);
    return cudaGetLastError();
}

}  // namespace pb2

using namespace pb2;

extern "C" {

uint32_t pb2_guide_param_count(void) { return (uint32_t)guide::kParams; }

int pb2_guide_create(uint32_t seed, pb2_guide** out) {
    if (!out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_create: null argument");
    *out = nullptr;
    auto* g = new pb2_guide();
    const size_t P = guide::kParams;
    cudaError_t e;
    if ((e = cudaMalloc(&g->params, P * 4)) || (e = cudaMalloc(&g->m, P * 4)) || (e = cudaMalloc(&g->v, P * 4)) ||
        (e = cudaMalloc(&g->grad, P * 4)) || (e = cudaMalloc(&g->w16, guide::kW16Elems * 2)) ||
        (e = cudaMalloc(&g->b32, guide::kBiasElems * 4)) || (e = cudaMalloc(&g->scalars, 16))) {
        pb2_guide_destroy(g);
        return cuda_fail(e, "pb2_guide_create");
    }
    // He-uniform weights, zero biases (splitmix64 stream from the seed)
    std::vector<float> p(P, 0.0f);
    uint64_t s = 0x9E3779B97F4A7C15ull * (seed + 1);
    auto next = [&]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < guide::kLayers; ++l) {
        const double lim = std::sqrt(6.0 / guide::layer_in(l));
        const int nw = guide::layer_out(l) * guide::layer_in(l);
        for (int i = 0; i < nw; ++i) p[guide::param_offset(l) + i] = (float)((2.0 * next() - 1.0) * lim);
    }
    int rc = pb2_guide_set_params(g, p.data(), (uint32_t)P);
    if (rc) {
        pb2_guide_destroy(g);
        return rc;
    }
    *out = g;
    return PB2_OK;
}

int pb2_guide_destroy(pb2_guide* g) {
    if (!g) return PB2_OK;
    cudaFree(g->params);
    cudaFree(g->m);
    cudaFree(g->v);
    cudaFree(g->grad);
    cudaFree(g->w16);
    cudaFree(g->b32);
    cudaFree(g->scalars);
    delete g;
    return PB2_OK;
}

int pb2_guide_set_params(pb2_guide* g, const float* params, uint32_t count) {
    if (!g || !params || count != (uint32_t)guide::kParams)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_set_params: wrong parameter count");
    const size_t P = guide::kParams;
    cudaError_t e;
    if ((e = cudaMemcpy(g->params, params, P * 4, cudaMemcpyHostToDevice)) || (e = cudaMemset(g->m, 0, P * 4)) ||
        (e = cudaMemset(g->v, 0, P * 4)) || (e = cudaMemset(g->grad, 0, P * 4)))
        return cuda_fail(e, "pb2_guide_set_params");
    if ((e = cudaMemset(g->w16, 0, guide::kW16Elems * 2))) return cuda_fail(e, "clear weight image");
    guide::k_image<<<(guide::kParams + 255) / 256, 256>>>(g->params, g->w16, g->b32);
    if ((e = cudaDeviceSynchronize())) return cuda_fail(e, "pb2_guide_set_params image");
    g->step = 0;
    return PB2_OK;
}

int pb2_guide_get_params(const pb2_guide* g, float* params, uint32_t count) {
    if (!g || !params || count != (uint32_t)guide::kParams)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_get_params: wrong parameter count");
    const cudaError_t e = cudaMemcpy(params, g->params, guide::kParams * 4, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "pb2_guide_get_params");
}

int pb2_guide_forward(const pb2_guide* g, const float* features, uint32_t n, float* out, void* stream) {
    if (!g || (n && (!features || !out))) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_forward: null argument");
    const cudaError_t e = guide_forward(g->view(), features, n, out, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "pb2_guide_forward");
}

int pb2_guide_gradient(pb2_guide* g, const float* records, uint32_t n, float* grad_host, float* loss_host, void* stream) {
    if (!g || (n && !records)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_gradient: null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s))) return cuda_fail(e, "memset grad");
    if ((e = guide_gradient(g->view(), records, n, g->grad, g->scalars, s))) return cuda_fail(e, "guide gradient");
    float sc[2] = { 0, 0 };
    if ((e = cudaMemcpyAsync(sc, g->scalars, 8, cudaMemcpyDeviceToHost, s))) return cuda_fail(e, "read loss");
    if (grad_host && (e = cudaMemcpyAsync(grad_host, g->grad, guide::kParams * 4, cudaMemcpyDeviceToHost, s)))
        return cuda_fail(e, "read grad");
    if ((e = cudaStreamSynchronize(s))) return cuda_fail(e, "sync");
    if ((e = cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s))) return cuda_fail(e, "memset grad");
    if (loss_host) *loss_host = sc[1];
    return PB2_OK;
}

int pb2_guide_train(pb2_guide* g, const float* records, uint32_t n, float learning_rate, float* loss_host, void* stream) {
    if (!g || (n && !records)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_train: null argument");
    if (n == 0) return PB2_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = guide_gradient(g->view(), records, n, g->grad, g->scalars, s))) return cuda_fail(e, "guide gradient");
    g->step += 1;
    const float bc1 = 1.0f - std::pow(guide::kBeta1, (float)g->step);
    const float bc2 = 1.0f - std::pow(guide::kBeta2, (float)g->step);
    guide::k_adam<<<(guide::kParams + 255) / 256, 256, 0, s>>>(g->params, g->m, g->v, g->grad, learning_rate, bc1, bc2,
                                                               g->w16, g->b32);
    if ((e = cudaGetLastError())) return cuda_fail(e, "k_adam");
    if (loss_host) {
        float sc[2];
        if ((e = cudaMemcpyAsync(sc, g->scalars, 8, cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
            return cuda_fail(e, "read loss");
        *loss_host = sc[1];
    }
    return PB2_OK;
}

}  // extern "C"
