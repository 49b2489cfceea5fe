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

// ---- loss gradient over a batch, in three passes ------------------------------------------------------
// The weight gradient dW_l = sum over records of dZ_l^T x input_l is a GEMM whose reduction runs over the
// batch.  Pass 1 runs forward and backward-data per 16-record tile and stages the bf16 layer inputs and
// deltas (1.3 KB per record); pass 2 runs the weight-gradient GEMMs with the batch as K, each block
// accumulating all 168 16x8 output tiles in registers over its records; pass 3 sums the blocks' partials.
// The bias gradients (column sums of the deltas) are reduced per block in pass 1.
constexpr int kStageX = kIn + 4 * kHid;   // 352: input X | H1 | H2 | H3 | H4 (the input of layer l)
constexpr int kStageD = 4 * kHid + kOut;  // 304: dZ0 | dZ1 | dZ2 | dZ3 | dY (the delta of layer l)
constexpr uint32_t kChunkRows = 1u << 16; // records staged per pass
constexpr int kGwThreads = 256;           // pass 2: 8 warps x 21 output tiles
constexpr int kGwRows = 64;               // pass 2: records per shared-memory chunk
constexpr int kGwXs = kStageX + 8, kGwDs = kStageD + 8;  // padded rows (conflict-free ldmatrix)
constexpr int kOutTiles = 48 + 3 * 32 + 24;
constexpr uint32_t kGwMaxBlocks = 128;
constexpr int kGrWarps = 8;  // pass 1: warps per block (one 16-record tile each at a time)
constexpr int kGrThreads = kGrWarps * 32;
__host__ __device__ constexpr int stage_x_offset(int l) { return l == 0 ? 0 : kIn + (l - 1) * kHid; }
__host__ __device__ constexpr int stage_d_offset(int l) { return l * kHid; }

// Pass 1.  records: n rows of 16 floats (pos01 xyz, normal xyz, wo xyz, wi xyz, weight, unused x3); `total`
// is the batch size the loss is normalised by.  Writes staged rows (all 16 rows of every tile; rows past n
// carry zero deltas), adds bias gradients to grad and the loss to *loss.
__global__ void __launch_bounds__(kGrThreads) k_grad_rows(GuideView gv, const float* __restrict__ rec, uint32_t n,
                                                        uint32_t total, const float* __restrict__ scalars,
                                                        __nv_bfloat16* __restrict__ sx, __nv_bfloat16* __restrict__ sd,
                                                        float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* w_s = reinterpret_cast<__nv_bfloat16*>(smem);
    float* b_s = reinterpret_cast<float*>(smem + kW16Elems * 2);
    float* gb_s = b_s + kBiasElems;  // bias gradients, bias_offset layout
    TrainTile* tiles = reinterpret_cast<TrainTile*>(gb_s + kBiasElems);
    load_weights(gv, w_s, b_s);
    for (int i = threadIdx.x; i < kBiasElems; i += blockDim.x) gb_s[i] = 0.f;
    __syncthreads();
    const float wsum = scalars[0];
    const float gscale = -(wsum > 0.f ? (float)total / wsum : 1.f) / (float)total;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TrainTile& T = tiles[warp];
    float loss_acc = 0.f;
    const uint32_t tiles_total = (n + 15) / 16;
    auto stage = [&](const __nv_bfloat16* src, int src_stride, int cols, __nv_bfloat16* dst, int dst_stride,
                     uint32_t row0) {
        // 16 rows x cols bf16 (cols a multiple of 8) in 16-byte pieces
        const int pieces = cols / 8;
        for (int i = lane; i < 16 * pieces; i += 32) {
            const int r = i / pieces, c = (i % pieces) * 8;
            *reinterpret_cast<int4*>(dst + (size_t)(row0 + r) * dst_stride + c) =
                *reinterpret_cast<const int4*>(src + r * src_stride + c);
        }
    };
    for (uint32_t tile = blockIdx.x * kGrWarps + warp; tile < tiles_total; tile += gridDim.x * kGrWarps) {
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
        dense_forward<kIn, kHid, true>(T.x, kXStride, w_s + w16_offset(0), layer_stride(0), b_s + bias_offset(0), T.h[0],
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
        stage(T.x, kXStride, kIn, sx + stage_x_offset(0), kStageX, row0);
        for (int l = 1; l <= 4; ++l) stage(T.h[l - 1], kHStride, kHid, sx + stage_x_offset(l), kStageX, row0);
        // loss gradient per row: dY (bf16) and the output-layer bias gradient (from the fp32 dY)
        if (lane < 16) {
            const float* f = T.feat + lane * 16;
            const float g = f[12] * gscale;
            float dy[kOut];
            const float lq = mixture_loss_grad(T.y + lane * kOut, f[9], f[10], f[11], g, dy);
            if (row0 + lane < n) loss_acc += g * lq;
            __nv_bfloat16* d = T.dz[0] + lane * kHStride;
            for (int i = 0; i < kOut; ++i) {
                d[i] = __float2bfloat16_rn(dy[i]);
                if (dy[i] != 0.f) atomicAdd(&gb_s[bias_offset(4) + i], dy[i]);
            }
        }
        __syncwarp();
        stage(T.dz[0], kHStride, kOut, sd + stage_d_offset(4), kStageD, row0);
        dense_backward_data<kHid, kOut>(T.dz[0], kHStride, w_s + w16_offset(4), layer_stride(4), T.h[3], kHStride,
                                        T.dz[1], kHStride);
        __syncwarp();
        int cur = 1;
        for (int l = 3; l >= 0; --l) {
            for (int c = lane; c < kHid; c += 32) {
                float sum = 0.f;
                for (int r = 0; r < 16; ++r) sum += __bfloat162float(T.dz[cur][r * kHStride + c]);
                atomicAdd(&gb_s[bias_offset(l) + c], sum);
            }
            stage(T.dz[cur], kHStride, kHid, sd + stage_d_offset(l), kStageD, row0);
            if (l > 0) {
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
    for (int i = threadIdx.x; i < kBiasElems; i += blockDim.x) {
        const int l = i < 4 * kHid ? i / kHid : 4;
        const int c = i - bias_offset(l);
        if (gb_s[i] != 0.f) atomicAdd(&grad[param_offset(l) + layer_out(l) * layer_in(l) + c], gb_s[i]);
    }
}

// (layer, output row tile, input column tile) of output tile t (48 tiles of layer 0, 32 of layers 1-3,
// 24 of layer 4)
__device__ __forceinline__ void out_tile(int t, int& l, int& mt, int& nt) {
    if (t < 48) {
        l = 0; mt = t / 12; nt = t % 12;
    } else if (t < 144) {
        const int r = t - 48;
        l = 1 + r / 32; mt = (r % 32) / 8; nt = r % 8;
    } else {
        const int r = t - 144;
        l = 4; mt = r / 8; nt = r % 8;
    }
}

// Pass 2: partial[block][param] for the weight entries, over records [block * per, (block + 1) * per).
__global__ void __launch_bounds__(kGwThreads) k_grad_weights(const __nv_bfloat16* __restrict__ sx,
                                                              const __nv_bfloat16* __restrict__ sd, uint32_t n,
                                                              uint32_t per, float* __restrict__ partial) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* ds = xs + kGwRows * kGwXs;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kPerWarp = kOutTiles / (kGwThreads / 32);  // 21
    float acc[kPerWarp][4];
#pragma unroll
    for (int j = 0; j < kPerWarp; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const uint32_t begin = blockIdx.x * per, end = min(n, begin + per);
    const int jj = lane >> 3, rr = lane & 7;
    for (uint32_t r0 = begin; r0 < end; r0 += kGwRows) {
        // stage kGwRows records (zeros past `end`) into padded shared rows
        constexpr int kXp = kStageX / 8, kDp = kStageD / 8;
        for (int i = threadIdx.x; i < kGwRows * (kXp + kDp); i += kGwThreads) {
            const int r = i / (kXp + kDp), c = i % (kXp + kDp);
            int4 v = make_int4(0, 0, 0, 0);
            if (r0 + r < end) {
                v = c < kXp ? *reinterpret_cast<const int4*>(sx + (size_t)(r0 + r) * kStageX + c * 8)
                            : *reinterpret_cast<const int4*>(sd + (size_t)(r0 + r) * kStageD + (c - kXp) * 8);
            }
            if (c < kXp) *reinterpret_cast<int4*>(xs + r * kGwXs + c * 8) = v;
            else *reinterpret_cast<int4*>(ds + r * kGwDs + (c - kXp) * 8) = v;
        }
        __syncthreads();
#pragma unroll 1
        for (int ks = 0; ks < kGwRows / 16; ++ks) {
            const __nv_bfloat16* X = xs + ks * 16 * kGwXs;
            const __nv_bfloat16* D = ds + ks * 16 * kGwDs;
#pragma unroll
            for (int j = 0; j < kPerWarp; ++j) {
                int l, mt, nt;
                out_tile(warp + j * (kGwThreads / 32), l, mt, nt);
                uint32_t a[4], b[2];
                // A[m = out][k = record] = D^T, B[k = record][n = in] = X
                ldsm_x4_t(a, D + ((jj >> 1) * 8 + rr) * kGwDs + stage_d_offset(l) + mt * 16 + (jj & 1) * 8);
                ldsm_x2_t(b, X + (lane & 15) * kGwXs + stage_x_offset(l) + nt * 8);
                mma16816(acc[j], a, b);
            }
        }
        __syncthreads();
    }
    float* out = partial + (size_t)blockIdx.x * kParams;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < kPerWarp; ++j) {
        int l, mt, nt;
        out_tile(warp + j * (kGwThreads / 32), l, mt, nt);
        const int o0 = mt * 16 + g, i0 = nt * 8 + 2 * t, in = layer_in(l);
        float* w = out + param_offset(l);
        w[o0 * in + i0] = acc[j][0];
        w[o0 * in + i0 + 1] = acc[j][1];
        w[(o0 + 8) * in + i0] = acc[j][2];
        w[(o0 + 8) * in + i0 + 1] = acc[j][3];
    }
}

// Pass 3: grad[weight entries] += the blocks' partials.
__global__ void k_grad_reduce(const float* __restrict__ partial, uint32_t blocks, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    int l = 0;
    while (l < kLayers - 1 && i >= param_offset(l + 1)) ++l;
    if (i - param_offset(l) >= layer_out(l) * layer_in(l)) return;  // a bias entry (pass 1)
    float s = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) s += partial[(size_t)b * kParams + i];
    grad[i] += s;
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
size_t grad_rows_smem() { return kW16Elems * 2 + 2 * kBiasElems * 4 + sizeof(TrainTile) * kGrWarps; }
size_t grad_weights_smem() { return (size_t)kGwRows * (kGwXs + kGwDs) * 2; }

}  // namespace guide

cudaError_t guide_forward(const GuideView& gv, const float* features, uint32_t n, float* out, cudaStream_t stream) {
    using namespace guide;
    if (n == 0) return cudaSuccess;
    static std::atomic<int> attr[kMaxDevices];
    cudaError_t e = smem_attr_once((const void*)k_forward, forward_smem(), attr);
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (n + 15) / 16;
    const int grid = (int)std::min<uint32_t>((tiles + kWarps - 1) / kWarps, 148u * 2u);
    k_forward<<<grid, kThreads, forward_smem(), stream>>>(gv, features, n, out);
    return cudaGetLastError();
}

size_t guide_workspace_bytes() {
    using namespace guide;
    return (size_t)kChunkRows * (kStageX + kStageD) * 2 + (size_t)kGwMaxBlocks * kParams * 4;
}

cudaError_t guide_gradient_mma(const GuideView& gv, const float* records, uint32_t n, float* grad, float* scalars,
                               void* workspace, cudaStream_t stream) {
    using namespace guide;
    static std::atomic<int> attr_rows[kMaxDevices], attr_weights[kMaxDevices];
    cudaError_t e = smem_attr_once((const void*)k_grad_rows, grad_rows_smem(), attr_rows);
    if (e == cudaSuccess) e = smem_attr_once((const void*)k_grad_weights, grad_weights_smem(), attr_weights);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(scalars, 0, 2 * sizeof(float), stream);
    if (e != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    __nv_bfloat16* sx = static_cast<__nv_bfloat16*>(workspace);
    __nv_bfloat16* sd = sx + (size_t)kChunkRows * kStageX;
    float* partial = reinterpret_cast<float*>(sd + (size_t)kChunkRows * kStageD);
    k_weight_sum<<<128, 256, 0, stream>>>(records, n, scalars);
    for (uint32_t c0 = 0; c0 < n; c0 += kChunkRows) {
        const uint32_t rows = std::min(kChunkRows, n - c0);
        const uint32_t tiles = (rows + 15) / 16;
        const int g1 = (int)std::min<uint32_t>((tiles + kGrWarps - 1) / kGrWarps, 148u);
        k_grad_rows<<<g1, kGrThreads, grad_rows_smem(), stream>>>(gv, records + 16 * (size_t)c0, rows, n, scalars, sx, sd,
                                                                grad, scalars + 1);
        const uint32_t chunks = (rows + kGwRows - 1) / kGwRows;
        const uint32_t blocks = std::min(kGwMaxBlocks, chunks);
        const uint32_t per = (chunks + blocks - 1) / blocks * kGwRows;
        k_grad_weights<<<blocks, kGwThreads, grad_weights_smem(), stream>>>(sx, sd, rows, per, partial);
        k_grad_reduce<<<(kParams + 255) / 256, 256, 0, stream>>>(partial, blocks, grad);
        if ((e = cudaGetLastError())) return e;
    }
    return cudaSuccess;
}

}  // namespace pb2

using namespace pb2;

extern "C" {

uint32_t pb2_guide_param_count(void) { return (uint32_t)guide::kParams; }

}  // extern "C"

namespace {
// scalars[4..7] of a guide: set by a training step whose tensor-core wait timed out (flag, stage, tile,
// block); sticky until read by a call that synchronises, which reports and clears them.
uint32_t* train_error(pb2_guide* g) { return reinterpret_cast<uint32_t*>(g->scalars + 4); }
bool train_failed(pb2_guide* g) {
    uint32_t v[4] = { 0, 0, 0, 0 };
    cudaMemcpy(v, g->scalars + 4, sizeof(v), cudaMemcpyDeviceToHost);
    if (!v[0]) return false;
    cudaMemset(g->scalars + 4, 0, sizeof(v));
    set_error("a tensor-core wait of the guide's training timed out (stage " + std::to_string(v[1]) + ", tile " +
              std::to_string(v[2]) + ", block " + std::to_string(v[3]) + ")");
    return true;
}
}  // namespace

extern "C" {

int pb2_guide_create(uint32_t seed, pb2_guide** out) {
    if (!out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_create: null argument");
    *out = nullptr;
    auto* g = new pb2_guide();
    const size_t P = guide::kParams;
    cudaError_t e;
    if ((e = cudaMalloc(&g->params, P * 4)) || (e = cudaMalloc(&g->m, P * 4)) || (e = cudaMalloc(&g->v, P * 4)) ||
        (e = cudaMalloc(&g->grad, P * 4)) || (e = cudaMalloc(&g->w16, guide::kW16Elems * 2)) ||
        (e = cudaMalloc(&g->b32, guide::kBiasElems * 4)) || (e = cudaMalloc(&g->scalars, 64)) ||
        (e = cudaMalloc(&g->workspace, guide_workspace_bytes()))) {
        pb2_guide_destroy(g);
        return cuda_fail(e, "pb2_guide_create");
    }
    // loss scalars and the training's time-out record start cleared (device memory comes uninitialised)
    if ((e = cudaMemset(g->scalars, 0, 64))) {
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
    cudaFree(g->workspace);
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
    if (n == 0) return PB2_OK;
    if ((reinterpret_cast<uintptr_t>(features) | reinterpret_cast<uintptr_t>(out)) & 15u)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_forward: features and outputs must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* flag = reinterpret_cast<uint32_t*>(g->scalars + 3);
    cudaError_t e;
    uint32_t h = 0;
    if ((e = cudaMemsetAsync(flag, 0, 4, s)) || (e = guide_forward_tc(g->view(), features, n, out, flag, s)) ||
        (e = cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
        return cuda_fail(e, "pb2_guide_forward");
    if (h) return fail(PB2_ERR_DEVICE_TIMEOUT, "pb2_guide_forward: a tensor-core wait timed out");
    return PB2_OK;
}

int pb2_guide_forward_async(const pb2_guide* g, const float* features, uint32_t n, float* out, uint32_t* status,
                            void* stream) {
    if (!g || !status || (n && (!features || !out)))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_forward_async: null argument");
    if (n == 0) return PB2_OK;
    if ((reinterpret_cast<uintptr_t>(features) | reinterpret_cast<uintptr_t>(out)) & 15u)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_forward_async: features and outputs must be 16-byte aligned");
    const cudaError_t e = guide_forward_tc(g->view(), features, n, out, status, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "pb2_guide_forward_async");
}

int pb2_guide_forward_mma(const pb2_guide* g, const float* features, uint32_t n, float* out, void* stream) {
    if (!g || (n && (!features || !out))) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_forward_mma: null argument");
    const cudaError_t e = guide_forward(g->view(), features, n, out, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "pb2_guide_forward_mma");
}

int pb2_guide_gradient(pb2_guide* g, const float* records, uint32_t n, float* grad_host, float* loss_host, void* stream) {
    if (!g || (n && !records)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_gradient: null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s))) return cuda_fail(e, "memset grad");
    if ((e = guide_gradient_tc(g->view(), records, n, g->grad, g->scalars, g->workspace, train_error(g), s)))
        return cuda_fail(e, "guide gradient");
    float sc[3] = { 0, 0, 0 };
    if ((e = cudaMemcpyAsync(sc, g->scalars, 12, cudaMemcpyDeviceToHost, s))) return cuda_fail(e, "read loss");
    if (grad_host && (e = cudaMemcpyAsync(grad_host, g->grad, guide::kParams * 4, cudaMemcpyDeviceToHost, s)))
        return cuda_fail(e, "read grad");
    if ((e = cudaStreamSynchronize(s))) return cuda_fail(e, "sync");
    if ((e = cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s))) return cuda_fail(e, "memset grad");
    if (loss_host) *loss_host = sc[1];
    if (train_failed(g)) return PB2_ERR_DEVICE_TIMEOUT;
    return PB2_OK;
}

int pb2_guide_gradient_mma(pb2_guide* g, const float* records, uint32_t n, float* grad_host, float* loss_host,
                           void* stream) {
    if (!g || (n && !records)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_gradient_mma: null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s))) return cuda_fail(e, "memset grad");
    if ((e = guide_gradient_mma(g->view(), records, n, g->grad, g->scalars, g->workspace, s)))
        return cuda_fail(e, "guide gradient");
    float sc[2] = { 0, 0 };
    if ((e = cudaMemcpyAsync(sc, g->scalars, 8, cudaMemcpyDeviceToHost, s))) return cuda_fail(e, "read loss");
    if (grad_host && (e = cudaMemcpyAsync(grad_host, g->grad, guide::kParams * 4, cudaMemcpyDeviceToHost, s)))
        return cuda_fail(e, "read grad");
    if ((e = cudaStreamSynchronize(s))) return cuda_fail(e, "sync");
    if ((e = cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s))) return cuda_fail(e, "memset grad");
    if (loss_host) *loss_host = sc[1];
    return PB2_OK;
}

int pb2_guide_set_gradient_hook(pb2_guide* g, pb2_gradient_hook hook, void* user) {
    if (!g) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_set_gradient_hook: null guide");
    g->hook = hook;
    g->hook_user = hook ? user : nullptr;
    return PB2_OK;
}

int pb2_guide_train(pb2_guide* g, const float* records, uint32_t n, float learning_rate, float* loss_host, void* stream) {
    if (!g || (n && !records)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_guide_train: null argument");
    if (n == 0) return PB2_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = guide_gradient_tc(g->view(), records, n, g->grad, g->scalars, g->workspace, train_error(g), s)))
        return cuda_fail(e, "guide gradient");
    if (g->hook) {
        const int rc = g->hook(g->grad, guide::kParams, stream, g->hook_user);
        if (rc != PB2_OK) {
            cudaMemsetAsync(g->grad, 0, guide::kParams * 4, s);  // the next step starts from a zero gradient
            return fail(rc, "pb2_guide_train: the gradient hook failed");
        }
    }
    g->step += 1;
    const float bc1 = 1.0f - std::pow(guide::kBeta1, (float)g->step);
    const float bc2 = 1.0f - std::pow(guide::kBeta2, (float)g->step);
    guide::k_adam<<<(guide::kParams + 255) / 256, 256, 0, s>>>(g->params, g->m, g->v, g->grad, learning_rate, bc1, bc2,
                                                               g->w16, g->b32);
    if ((e = cudaGetLastError())) return cuda_fail(e, "k_adam");
    if (loss_host) {
        float sc[3];
        if ((e = cudaMemcpyAsync(sc, g->scalars, 12, cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
            return cuda_fail(e, "read loss");
        *loss_host = sc[1];
        if (train_failed(g)) return PB2_ERR_DEVICE_TIMEOUT;
    }
    return PB2_OK;
}

}  // extern "C"
