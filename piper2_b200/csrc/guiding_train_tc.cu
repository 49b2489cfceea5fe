// guiding_train_tc.cu -- the guiding network's loss gradient on the 5th-generation tensor cores (tcgen05).
//
// One CTA of 8 warps per SM walks 128-record tiles.  Thread t < 128 owns record t; thread t + 128 (warp w + 4)
// serves the same record and TMEM lane: it drains alternate 16-column chunks of the hidden-layer, backward-data and
// final epilogues and computes lobes 4-7 of the record's loss gradient.  Per tile:
//   forward   5 MMAs  a_l (128 x in_l, K-major) x W_l^T -> TMEM; epilogue bias + ReLU -> bf16 a_{l+1}
//   loss      per record: dY = d(-g log q)/dy from the 48 raw outputs (fp32; bf16 copy for the MMAs)
//   backward  for l = 4 .. 0:
//               dW_l^T += a_l^T (features x records) . dZ_l (records x out_l)   -- accumulated in TMEM over
//                         all the CTA's tiles; both operands read "MN-major" from the same shared-memory
//                         tiles the forward wrote K-major (a core matrix is 8 records x 8 features either way)
//               dA_l    = dZ_l . W_l (records x in_l)                             -- W_l read MN-major from
//                         the forward's weight image
//               dZ_{l-1} = bf16(dA_l) where a_l > 0, written over a_l in place (a_l is consumed)
// The activation tiles carry one extra feature fixed at 1 (column 64 of a_1..a_4, the encoding's constant
// column 84 of a_0), so row 64 / 84 of dW_l^T is the column sum of dZ_l: the bias gradient comes out of the
// same MMA.  The output layer's bias gradient is summed from the fp32 dY instead (as the loss defines it).
// dW^T has the layer's input features as its 128 rows (M = 128; rows past the layer's inputs read whatever
// follows the tile in shared memory and are never used) and out_l columns; the five accumulators take 304
// TMEM columns, the forward/backward accumulator 64 more.  At the end each CTA writes its partial gradient
// (all parameters) to `partial`; a reduction over CTAs adds them to the gradient.
//
// Waits on the mbarrier are bounded: on time-out the CTA records an error, stops, gives the tensor core a
// bounded time to drain, frees its TMEM and returns.
#include <algorithm>
#include <cstdlib>

#include "guiding_tc.cuh"
#include "pb2_internal.h"

namespace pb2 {
namespace guide {
namespace {

constexpr int kTrThreads = 256;  // two warps per TMEM lane quarter: warps w and w + 4 split a layer's columns
constexpr int kActDim = 72;                            // a_1..a_4: 64 features, the constant 1, 7 zeros
constexpr int kTrXBytes = kTcRows * kIn * 2;           // a_0: 24,576
constexpr int kTrABytes = kTcRows * kActDim * 2;       // a_1..a_4: 18,432 each
constexpr int kTrDYBytes = kTcRows * kOut * 2;         // dY: 12,288
constexpr int kTrOffW = 0;
constexpr int kTrOffX = kTcWBytes;                     // 43,008 (1024-aligned)
constexpr int kTrOffA1 = kTrOffX + kTrXBytes;
constexpr int kTrOffDY = kTrOffA1 + 4 * kTrABytes;
constexpr int kTrOffSlack = kTrOffDY + kTrDYBytes;     // rows past a tile's features are read from here on
constexpr int kTrOffBias = kTrOffSlack + 2048;
constexpr int kTrOffBias4 = kTrOffBias + kBiasElems * 4;  // fp32 output-bias gradient of this CTA
constexpr int kTrOffBar = kTrOffBias4 + kOut * 4;
// the loss gradient's exchange between a record's two threads, per record: the raw outputs of lobes 4-7 (20), the
// sampled direction and loss weight (4), the two halves' softmax maxima, sums and density parts (6), the second
// half's output deltas (20); 52 floats with padding
constexpr int kXchStride = 52;
constexpr int kTrOffXch = kTrOffBar + 16;
constexpr int kTrSmem = kTrOffXch + kTcRows * kXchStride * 4;
static_assert(kTrOffX % 1024 == 0 && kTrOffA1 % 1024 == 0 && kTrABytes % 1024 == 0 && kTrOffDY % 1024 == 0,
              "operand alignment");
static_assert(kTrSmem <= 227 * 1024, "shared memory per CTA");

constexpr uint32_t kTrTmemCols = 512;
constexpr uint32_t kAccCol = 0;                        // forward / backward-data accumulator (64 columns)
__host__ __device__ constexpr uint32_t dw_col(int l) { return 64u + 64u * (uint32_t)l; }  // dW_l^T: out_l columns

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Waits for the mbarrier phase for at most kTrWaitNs of device time (not a poll count, so that a busy GPU does
// not shorten it); false on time-out.
constexpr unsigned long long kTrWaitNs = 200ull * 1000 * 1000;  // 200 ms
__device__ __forceinline__ bool mbar_wait_timed(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = now_ns();
    for (;;) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (now_ns() - t0 > kTrWaitNs) return false;
    }
}

// A bf16 (low 16 bits of h) greater than zero: sign clear and not +0 (activations are ReLU outputs, never NaN).
__device__ __forceinline__ bool bf16_positive(uint32_t h) { return h != 0u && (h & 0x8000u) == 0u; }

// kind::f16 instruction descriptor with operand majorness: a_mn / b_mn = 1 reads that operand MN-major.
__device__ __forceinline__ uint32_t instr_desc_major(uint32_t n, uint32_t a_mn, uint32_t b_mn) {
    return instr_desc(n) | (a_mn << 15) | (b_mn << 16);
}

__device__ __forceinline__ unsigned char* act(unsigned char* smem, int l) {  // input tile of layer l
    return l == 0 ? smem + kTrOffX : smem + kTrOffA1 + (l - 1) * kTrABytes;
}
__host__ __device__ constexpr uint32_t act_dim(int l) { return l == 0 ? (uint32_t)kIn : (uint32_t)kActDim; }

__global__ void __launch_bounds__(kTrThreads, 1) k_grad_tc(GuideView gv, const float* __restrict__ rec, uint32_t n,
                                                          const float* __restrict__ scalars,
                                                          float* __restrict__ partial, float* __restrict__ loss,
                                                          uint32_t* __restrict__ error, uint32_t skip_commit) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // warps 0-3 own the tile's records (thread tid = record and TMEM lane tid); warp w + 4 serves the same 32
    // TMEM lanes as warp w and drains the other half of each accumulator's 16-column chunks
    const bool owner = tid < kTcRows;
    const int rowt = (warp & 3) * 32 + lane;        // this thread's record row / TMEM lane
    const uint32_t half = (uint32_t)(warp >> 2);     // its chunks: c0 = 16 half, 16 half + 32, ...
    unsigned char* w_s = smem + kTrOffW;
    float* b_s = reinterpret_cast<float*>(smem + kTrOffBias);
    float* gb4 = reinterpret_cast<float*>(smem + kTrOffBias4);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTrOffBar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTrOffBar + 8);
    volatile uint32_t& s_fail = *reinterpret_cast<uint32_t*>(smem + kTrOffBar + 12);

    // weights in the forward's K-major core-matrix image, biases, the constant-1 columns of a_1..a_4
    for (int l = 0; l < kLayers; ++l) {
        const int in = layer_in(l), outd = layer_out(l), chunks = outd * (in / 8);
        for (int c = tid; c < chunks; c += kTrThreads) {
            const int o = c / (in / 8), kc = c % (in / 8);
            const int4 v = *reinterpret_cast<const int4*>(gv.w16 + w16_offset(l) + o * layer_stride(l) + kc * 8);
            *reinterpret_cast<int4*>(w_s + tc_w_offset(l) + core_offset(o, kc * 8, in)) = v;
        }
    }
    for (int i = tid; i < kBiasElems; i += kTrThreads) b_s[i] = gv.b32[i];
    for (int i = tid; i < kOut; i += kTrThreads) gb4[i] = 0.f;
    for (int l = 1; l < kLayers && owner; ++l) {
        __align__(16) __nv_bfloat16 one[8];
        for (int i = 0; i < 8; ++i) one[i] = __float2bfloat16_rn(i == 0 ? 1.f : 0.f);
        *reinterpret_cast<int4*>(act(smem, l) + core_offset(tid, 64, kActDim)) = *reinterpret_cast<const int4*>(one);
    }
    for (int i = tid; i < 2048 / 16; i += kTrThreads)
        reinterpret_cast<int4*>(smem + kTrOffSlack)[i] = make_int4(0, 0, 0, 0);
    if (tid == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTrTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t bar_addr = smem_u32(bar);
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's 32 TMEM lanes
    uint32_t phase = 0;
    bool failed = false;
    const float wsum = scalars[0];
    const float gscale = -(wsum > 0.f ? 1.f / wsum : 1.f / (float)(n ? n : 1));
    float loss_acc = 0.f;

    // commits the MMAs thread 0 issued and waits for them (all threads); false if the wait timed out.  On
    // time-out error[0] = 1 and, from the first CTA to fail, error[1..3] = the wait's stage (1 + layer for the
    // forward, 16 + layer for the backward), the tile and the block.
    uint32_t stage = 0, cur_tile = 0;
    bool first = true;  // this CTA's first tile: the weight-gradient accumulators start from zero
    auto commit_wait = [&]() -> bool {
        // skip_commit (failure-detection tests only): the first tile's wait at that stage gets no arrival
        if (tid == 0 && !(first && stage == skip_commit)) mma_commit(bar_addr);
        bool ok = mbar_wait_timed(bar_addr, phase);
        phase ^= 1u;
        if (!ok) {
            s_fail = 1u;
            if (atomicExch(error, 1u) == 0u) {
                error[1] = stage;
                error[2] = cur_tile;
                error[3] = blockIdx.x;
            }
        }
        tc_fence_after();
        __syncthreads();
        return s_fail == 0u;
    };
    auto publish = [&]() {  // shared-memory operands written by threads -> visible to the next MMAs
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    };

    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    for (uint32_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const uint32_t row = tile * kTcRows + tid;
        cur_tile = tile;
        float r[16];
        if (!owner) {
#pragma unroll
            for (int q = 0; q < 16; ++q) r[q] = 0.f;
        } else if (row < n) {
            const float4* p = reinterpret_cast<const float4*>(rec + 16 * (size_t)row);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = __ldg(p + q);
                r[4 * q] = v.x; r[4 * q + 1] = v.y; r[4 * q + 2] = v.z; r[4 * q + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) r[q] = 0.f;
            r[5] = 1.f; r[8] = 1.f; r[11] = 1.f;  // unit directions, zero weight: no contribution
        }
        if (owner) {
            __align__(16) __nv_bfloat16 enc[kIn];
            encode_row(r, enc);
#pragma unroll
            for (int kc = 0; kc < kIn / 8; ++kc)
                *reinterpret_cast<int4*>(act(smem, 0) + core_offset(tid, kc * 8, kIn)) =
                    *reinterpret_cast<const int4*>(enc + kc * 8);
        }
        publish();
        // ---- forward ----
        float y[kOut];
        for (int l = 0; l < kLayers && !failed; ++l) {
            const uint32_t kdim = layer_in(l), ndim = layer_out(l);
            stage = 1u + (uint32_t)l;
            if (tid == 0) {
                const uint32_t a0 = smem_u32(act(smem, l)), b0 = smem_u32(w_s + tc_w_offset(l));
                for (uint32_t s = 0; s < kdim / 16; ++s)
                    mma_bf16(tmem + kAccCol, smem_desc(a0 + 256 * s, 128, act_dim(l) * 16),
                             smem_desc(b0 + 256 * s, 128, kdim * 16), instr_desc(ndim), s > 0 ? 1u : 0u);
            }
            if (!commit_wait()) {
                failed = true;
                break;
            }
            if (l < kLayers - 1) {
                // hidden layers: both warps of a lane quarter, alternate 16-column chunks
                for (uint32_t c0 = 16u * half; c0 < ndim; c0 += 32u) {
                    float v[16];
                    tmem_ld16(lane_base + kAccCol + c0, v);
                    tmem_wait_ld();
                    const float* bias = b_s + bias_offset(l) + c0;
                    // bias, ReLU and the bf16 rounding of two columns per instruction
                    uint32_t hw[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) hw[i] = pack_relu_bf16x2(v[2 * i] + bias[2 * i], v[2 * i + 1] + bias[2 * i + 1]);
                    unsigned char* dst = act(smem, l + 1);
                    *reinterpret_cast<uint4*>(dst + core_offset(rowt, c0, kActDim)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                    *reinterpret_cast<uint4*>(dst + core_offset(rowt, c0 + 8, kActDim)) =
                        make_uint4(hw[4], hw[5], hw[6], hw[7]);
                }
            } else if (owner) {
                // the output layer: the record owners, all 48 columns (y stays in registers for the loss gradient)
#pragma unroll
                for (int c0 = 0; c0 < kOut; c0 += 16) {
                    float v[16];
                    tmem_ld16(lane_base + kAccCol + c0, v);
                    tmem_wait_ld();
                    const float* bias = b_s + bias_offset(l) + c0;
#pragma unroll
                    for (int i = 0; i < 16; ++i) y[c0 + i] = v[i] + bias[i];
                }
            }
            publish();
        }
        if (failed) break;
        // ---- loss gradient of this record (fp32), its bf16 copy for the MMAs, the output-bias sums ----
        // The record's two threads split the mixture's eight lobes (half 0: lobes 0-3, half 1: lobes 4-7, as
        // mixture_loss_grad computes them) and combine the softmax maximum and sum and the density q through xr.
        {
            float* xr = reinterpret_cast<float*>(smem + kTrOffXch) + (size_t)rowt * kXchStride;
            float g = 0.f, wx = 0.f, wy = 0.f, wz = 0.f;
            float yl[20];
            if (owner) {
                g = r[12] * gscale;
                wx = r[9];
                wy = r[10];
                wz = r[11];
#pragma unroll
                for (int i = 0; i < 20; ++i) xr[i] = y[20 + i];
                xr[20] = wx;
                xr[21] = wy;
                xr[22] = wz;
                xr[23] = g;
            }
            __syncthreads();
            if (owner) {
#pragma unroll
                for (int i = 0; i < 20; ++i) yl[i] = y[i];
            } else {
#pragma unroll
                for (int i = 0; i < 20; ++i) yl[i] = xr[i];
                wx = xr[20];
                wy = xr[21];
                wz = xr[22];
                g = xr[23];
            }
            float mx = -3.0e38f;
#pragma unroll
            for (int k = 0; k < 4; ++k) mx = fmaxf(mx, yl[5 * k]);
            xr[24 + half] = mx;
            __syncthreads();
            mx = fmaxf(xr[24], xr[25]);
            float wl[4], sum = 0.f;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                wl[k] = expf(yl[5 * k] - mx);
                sum += wl[k];
            }
            xr[26 + half] = sum;
            __syncthreads();
            sum = xr[26] + xr[27];
            float mu[4][3], kap[4], comp[4], qpart = 0.f;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                wl[k] /= sum;
                const float vx = yl[5 * k + 1], vy = yl[5 * k + 2], vz = yl[5 * k + 3];
                const float nv = sqrtf(vx * vx + vy * vy + vz * vz);
                if (nv > 1e-12f) { mu[k][0] = vx / nv; mu[k][1] = vy / nv; mu[k][2] = vz / nv; }
                else { mu[k][0] = 0.f; mu[k][1] = 0.f; mu[k][2] = 1.f; }
                kap[k] = fminf(softplus(yl[5 * k + 4]) + kKappaMin, kKappaMax);
                comp[k] = vmf_eval(mu[k], kap[k], wx, wy, wz);
                qpart += wl[k] * comp[k];
            }
            xr[28 + half] = qpart;
            __syncthreads();
            const float qs = fmaxf(xr[28] + xr[29], 1e-30f);
            float dl[20];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float resp = wl[k] * comp[k] / qs;
                dl[5 * k] = g * (resp - wl[k]);
                const float kk = kap[k];
                const float mdw = mu[k][0] * wx + mu[k][1] * wy + mu[k][2] * wz;
                const float dlogk = 1.f / kk - 2.f / expm1f(2.f * kk) + (mdw - 1.f);
                const float raw = yl[5 * k + 4];
                const float sig = 1.f / (1.f + expf(-raw));
                const bool free_k = softplus(raw) + kKappaMin < kKappaMax;
                dl[5 * k + 4] = free_k ? g * resp * dlogk * sig : 0.f;
                const float vx = yl[5 * k + 1], vy = yl[5 * k + 2], vz = yl[5 * k + 3];
                const float vn = fmaxf(sqrtf(vx * vx + vy * vy + vz * vz), 1e-30f);
                const float sc = g * resp * kk / vn;
                dl[5 * k + 1] = sc * (wx - mdw * mu[k][0]);
                dl[5 * k + 2] = sc * (wy - mdw * mu[k][1]);
                dl[5 * k + 3] = sc * (wz - mdw * mu[k][2]);
            }
            if (!owner) {
#pragma unroll
                for (int i = 0; i < 20; ++i) xr[30 + i] = dl[i];
            }
            __syncthreads();
            if (owner) {
                float dy[kOut];
    #pragma unroll
                for (int i = 0; i < 20; ++i) {
                    dy[i] = dl[i];
                    dy[20 + i] = xr[30 + i];
                }
    #pragma unroll
                for (int i = 5 * kLobes; i < kOut; ++i) dy[i] = 0.f;
                if (row < n) loss_acc += g * logf(qs);
    #pragma unroll
                for (int kc = 0; kc < kOut / 8; ++kc)
                    *reinterpret_cast<uint4*>(smem + kTrOffDY + core_offset(tid, kc * 8, kOut)) =
                        make_uint4(pack_bf16x2(dy[8 * kc], dy[8 * kc + 1]), pack_bf16x2(dy[8 * kc + 2], dy[8 * kc + 3]),
                                   pack_bf16x2(dy[8 * kc + 4], dy[8 * kc + 5]), pack_bf16x2(dy[8 * kc + 6], dy[8 * kc + 7]));
                // warp sums of the 48 outputs' dY by recursive halving (padded to 64): at the step with lane offset o
                // a lane keeps the half of its partial sums that its lane bit o selects and adds the partner's copy of
                // it, so that lane l ends with the sums of outputs 2l and 2l + 1
                {
                    float t[64];
    #pragma unroll
                    for (int i = 0; i < 64; ++i) t[i] = i < kOut ? dy[i] : 0.f;
    #pragma unroll
                    for (int h = 32, o = 16; h >= 2; h >>= 1, o >>= 1) {
                        const bool up = (lane & o) != 0;
    #pragma unroll
                        for (int i = 0; i < h; ++i) {
                            const float send = up ? t[i] : t[i + h];
                            const float keep = up ? t[i + h] : t[i];
                            t[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, o);
                        }
                    }
                    if (2 * lane < kOut) {
                        if (t[0] != 0.f) atomicAdd(&gb4[2 * lane], t[0]);
                        if (t[1] != 0.f) atomicAdd(&gb4[2 * lane + 1], t[1]);
                    }
                }
            }
        }
        publish();
        // ---- backward ----
        for (int l = kLayers - 1; l >= 0; --l) {
            const uint32_t in = layer_in(l), outd = layer_out(l);
            // dZ_l: dY for the output layer, else written over a_{l+1}
            const unsigned char* dz = l == kLayers - 1 ? smem + kTrOffDY : act(smem, l + 1);
            const uint32_t dz_dim = l == kLayers - 1 ? (uint32_t)kOut : (uint32_t)kActDim;
            stage = 16u + (uint32_t)l;
            if (tid == 0) {
                // dW_l^T (M = 128 feature rows, N = out_l) += a_l^T . dZ_l over this tile's 128 records (K)
                const uint32_t a0 = smem_u32(act(smem, l)), z0 = smem_u32(dz);
                const uint32_t adim = act_dim(l);
                for (uint32_t s = 0; s < kTcRows / 16; ++s)
                    mma_bf16(tmem + dw_col(l), smem_desc(a0 + s * 2 * adim * 16, adim * 16, 128),
                             smem_desc(z0 + s * 2 * dz_dim * 16, dz_dim * 16, 128), instr_desc_major(outd, 1u, 1u),
                             (first && s == 0) ? 0u : 1u);
                // dA_l (M = 128 records, N = in_l) = dZ_l . W_l, K = out_l; W_l read MN-major (N = in_l)
                if (l > 0) {
                    const uint32_t w0 = smem_u32(w_s + tc_w_offset(l));
                    for (uint32_t s = 0; s < outd / 16; ++s)
                        mma_bf16(tmem + kAccCol, smem_desc(z0 + 256 * s, 128, dz_dim * 16),
                                 smem_desc(w0 + s * 2 * in * 16, in * 16, 128), instr_desc_major(in, 0u, 1u),
                                 s > 0 ? 1u : 0u);
                }
            }
            if (!commit_wait()) {
                failed = true;
                break;
            }
            if (l > 0) {
                // dZ_{l-1} = bf16(dA_l) where a_l > 0, over a_l (this thread's row only)
                unsigned char* a = act(smem, l);
                for (uint32_t c0 = 16u * half; c0 < in; c0 += 32u) {
                    float v[16];
                    tmem_ld16(lane_base + kAccCol + c0, v);
                    tmem_wait_ld();
                    // a_l > 0 tested on the bf16 bits (a ReLU output: +0 or positive), two columns per word
                    uint4 w0 = *reinterpret_cast<const uint4*>(a + core_offset(rowt, c0, kActDim));
                    uint4 w1 = *reinterpret_cast<const uint4*>(a + core_offset(rowt, c0 + 8, kActDim));
                    uint32_t aw[8] = { w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w };
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        aw[i] = pack_bf16x2(bf16_positive(aw[i] & 0xFFFFu) ? v[2 * i] : 0.f,
                                            bf16_positive(aw[i] >> 16) ? v[2 * i + 1] : 0.f);
                    *reinterpret_cast<uint4*>(a + core_offset(rowt, c0, kActDim)) = make_uint4(aw[0], aw[1], aw[2], aw[3]);
                    *reinterpret_cast<uint4*>(a + core_offset(rowt, c0 + 8, kActDim)) =
                        make_uint4(aw[4], aw[5], aw[6], aw[7]);
                }
                publish();
            }
        }
        first = false;
    }
    if (failed && tid == 0) mbar_wait_timed(bar_addr, phase);  // let MMAs in flight finish before freeing
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xFFFFFFFFu, loss_acc, o);
    if (lane == 0 && loss_acc != 0.f) atomicAdd(loss, loss_acc);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- this CTA's partial gradient: dW_l^T row f (this thread's TMEM lane) -> W_l[:, f]; the constant
    // feature's row -> the bias of layers 0..3; the output bias from the fp32 sums ----
    float* out = partial + (size_t)blockIdx.x * kParams;
    const uint32_t f = (uint32_t)rowt;
    for (int l = 0; l < kLayers; ++l) {
        const uint32_t in = layer_in(l), outd = layer_out(l);
        const uint32_t bias_row = l == 0 ? 84u : 64u;
        for (uint32_t c0 = 16u * half; c0 < outd; c0 += 32u) {
            float v[16];
            tmem_ld16(lane_base + dw_col(l) + c0, v);
            tmem_wait_ld();
            if (first || failed) {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.f;  // no tile reached this CTA: nothing was accumulated
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const uint32_t o = c0 + i;
                if (f < in) out[param_offset(l) + o * in + f] = v[i];
                if (f == bias_row && l < kLayers - 1) out[param_offset(l) + outd * in + o] = v[i];
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < kOut; i += kTrThreads) out[param_offset(kLayers - 1) + kOut * kHid + i] = gb4[i];
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrTmemCols));
}

// The records' weight sum (the loss normalisation) in a fixed order, so that a batch always gets the same
// normalisation bit for bit: a float atomic sum would change its last bits from call to call, and through
// the bf16 rounding of the loss gradient that reaches the gradient.  Pass 1: block b sums its contiguous
// range with a fixed tree into part[b]; pass 2: one warp adds the blocks' sums in order into scalars[0].
constexpr int kWsBlocks = 128, kWsThreads = 256;
__global__ void __launch_bounds__(kWsThreads) k_weight_sum_part(const float* __restrict__ rec, uint32_t n,
                                                               float* __restrict__ part) {
    __shared__ float sh[kWsThreads];
    const uint32_t per = (n + kWsBlocks - 1) / kWsBlocks;
    const uint32_t begin = blockIdx.x * per, end = min(n, begin + per);
    float s = 0.f;
    for (uint32_t i = begin + threadIdx.x; i < end; i += kWsThreads) s += rec[16 * (size_t)i + 12];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = kWsThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_weight_sum_final(const float* __restrict__ part, float* scalars) {
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int b = 0; b < kWsBlocks; ++b) s += part[b];
        scalars[0] = s;
    }
}

// grad[i] += sum over CTAs of partial[cta][i], every parameter.
__global__ void k_grad_reduce_all(const float* __restrict__ partial, uint32_t blocks, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    float s = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) s += partial[(size_t)b * kParams + i];
    grad[i] += s;
}

}  // namespace
}  // namespace guide

cudaError_t guide_gradient_tc(const GuideView& gv, const float* records, uint32_t n, float* grad, float* scalars,
                              void* workspace, uint32_t* error, cudaStream_t stream) {
    using namespace guide;
    static std::atomic<int> attr[kMaxDevices];
    cudaError_t e = smem_attr_once((const void*)k_grad_tc, (size_t)kTrSmem, attr);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(scalars, 0, 2 * sizeof(float), stream))) return e;
    if (n == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)sms);
    float* partial = static_cast<float*>(workspace);
    float* wpart = partial + (size_t)grid * kParams;  // kWsBlocks floats after the CTAs' partial gradients
    k_weight_sum_part<<<kWsBlocks, kWsThreads, 0, stream>>>(records, n, wpart);
    k_weight_sum_final<<<1, 32, 0, stream>>>(wpart, scalars);
    // PB2_TEST_TRAIN_TIMEOUT=<stage> (failure-detection tests): the first tile's MMAs of that stage are committed
    // to nothing, so its bounded wait runs out and the step reports the time-out; read on every call
    const char* inject = std::getenv("PB2_TEST_TRAIN_TIMEOUT");
    const uint32_t skip = inject ? (uint32_t)std::strtoul(inject, nullptr, 10) : 0u;
    k_grad_tc<<<grid, kTrThreads, kTrSmem, stream>>>(gv, records, n, scalars, partial, scalars + 1, error, skip);
    k_grad_reduce_all<<<(kParams + 255) / 256, 256, 0, stream>>>(partial, grid, grad);
    return cudaGetLastError();
}

}  // namespace pb2
