// guiding.cuh -- the path-guiding model on the device: input encoding, the 96-64-64-64-64-48 MLP with BF16
// tensor-core tiles and FP32 accumulation, the von Mises-Fisher mixture (pdf, sampling, loss gradient).
//
// The reference renderer has no guiding; the method follows the float64 restatement the tests use
// (one-blob-style input encoding, an MLP predicting 8 vMF lobes, training by the Monte-Carlo KL
// divergence against the radiance samples the integrator produces, Adam).
//
// MLP tiles: one warp runs 16 rows through every layer with mma.sync m16n8k16 (BF16 in, FP32
// accumulate).  Operands are staged in shared memory; rows are padded by 8 elements so the eight
// 16-byte rows an ldmatrix reads fall in distinct banks.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pb2 {
namespace guide {

constexpr int kIn = 96, kHid = 64, kOut = 48, kLobes = 8, kLayers = 5;
constexpr float kKappaMin = 0.05f, kKappaMax = 2000.0f;
constexpr float kBeta1 = 0.9f, kBeta2 = 0.99f, kEps = 1e-8f;

__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int layer_out(int l) { return l == kLayers - 1 ? kOut : kHid; }
__host__ __device__ constexpr int layer_stride(int l) { return layer_in(l) + 8; }  // bf16 elements per W row
// offsets of each layer's W in the padded bf16 weight image and in the flat fp32 parameter vector
__host__ __device__ constexpr int w16_offset(int l) {
    return l == 0 ? 0 : w16_offset(l - 1) + layer_out(l - 1) * layer_stride(l - 1);
}
__host__ __device__ constexpr int param_offset(int l) {
    return l == 0 ? 0 : param_offset(l - 1) + layer_out(l - 1) * layer_in(l - 1) + layer_out(l - 1);
}
constexpr int kW16Elems = w16_offset(kLayers);      // 23936
constexpr int kParams = param_offset(kLayers);      // 21808
constexpr int kBiasElems = 4 * kHid + kOut;         // 304
__host__ __device__ constexpr int bias_offset(int l) { return l * kHid; }

// activation tiles (bf16, 16 rows)
constexpr int kXStride = kIn + 8;   // 104
constexpr int kHStride = kHid + 8;  // 72
constexpr int kYStride = kOut + 8;  // 56

// ---- warp-level tensor-core primitives -------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t (&r)[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t (&r)[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Y[16 x out] = X[16 x in] W^T (+ bias, ReLU) for one warp.  X: bf16, row stride xs; W: bf16 [out][in],
// row stride ws.  Writes bf16 to H (row stride hs) when relu, else fp32 to Yf (row stride yfs).
template <int kInDim, int kOutDim, bool kRelu>
__device__ __forceinline__ void dense_forward(const __nv_bfloat16* X, int xs, const __nv_bfloat16* W, int ws,
                                              const float* bias, __nv_bfloat16* H, int hs, float* Yf, int yfs) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    constexpr int KT = kInDim / 16;
    uint32_t a[KT][4];
#pragma unroll
    for (int k = 0; k < KT; ++k) ldsm_x4(a[k], X + (lane & 15) * xs + k * 16 + (lane >> 4) * 8);
#pragma unroll
    for (int nt = 0; nt < kOutDim / 8; ++nt) {
        float c[4] = { 0.f, 0.f, 0.f, 0.f };
#pragma unroll
        for (int k = 0; k < KT; ++k) {
            uint32_t b[2];
            ldsm_x2(b, W + (nt * 8 + (lane & 7)) * ws + k * 16 + ((lane >> 3) & 1) * 8);
            mma16816(c, a[k], b);
        }
        const int col = nt * 8 + 2 * t;
        const float b0 = bias[col], b1 = bias[col + 1];
        float v0 = c[0] + b0, v1 = c[1] + b1, v2 = c[2] + b0, v3 = c[3] + b1;
        if (kRelu) {
            v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); v2 = fmaxf(v2, 0.f); v3 = fmaxf(v3, 0.f);
            *reinterpret_cast<__nv_bfloat162*>(H + g * hs + col) = __floats2bfloat162_rn(v0, v1);
            *reinterpret_cast<__nv_bfloat162*>(H + (g + 8) * hs + col) = __floats2bfloat162_rn(v2, v3);
        } else {
            Yf[g * yfs + col] = v0;
            Yf[g * yfs + col + 1] = v1;
            Yf[(g + 8) * yfs + col] = v2;
            Yf[(g + 8) * yfs + col + 1] = v3;
        }
    }
}

// dX[16 x in] = dZ[16 x out] W  (W: [out][in]); optionally masked by (Hprev > 0); bf16 out.
template <int kInDim, int kOutDim>
__device__ __forceinline__ void dense_backward_data(const __nv_bfloat16* dZ, int dzs, const __nv_bfloat16* W, int ws,
                                                    const __nv_bfloat16* Hprev, int hps, __nv_bfloat16* dX, int dxs) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    constexpr int KT = kOutDim / 16;
    uint32_t a[KT][4];
#pragma unroll
    for (int k = 0; k < KT; ++k) ldsm_x4(a[k], dZ + (lane & 15) * dzs + k * 16 + (lane >> 4) * 8);
#pragma unroll
    for (int nt = 0; nt < kInDim / 8; ++nt) {
        float c[4] = { 0.f, 0.f, 0.f, 0.f };
#pragma unroll
        for (int k = 0; k < KT; ++k) {
            uint32_t b[2];
            // B[k = out][n = in] from W stored [out][in]: transposed 8x8 loads
            ldsm_x2_t(b, W + (k * 16 + (lane & 15)) * ws + nt * 8);
            mma16816(c, a[k], b);
        }
        const int col = nt * 8 + 2 * t;
        const __nv_bfloat162 h0 = *reinterpret_cast<const __nv_bfloat162*>(Hprev + g * hps + col);
        const __nv_bfloat162 h1 = *reinterpret_cast<const __nv_bfloat162*>(Hprev + (g + 8) * hps + col);
        const float m0 = __low2float(h0) > 0.f ? 1.f : 0.f, m1 = __high2float(h0) > 0.f ? 1.f : 0.f;
        const float m2 = __low2float(h1) > 0.f ? 1.f : 0.f, m3 = __high2float(h1) > 0.f ? 1.f : 0.f;
        *reinterpret_cast<__nv_bfloat162*>(dX + g * dxs + col) = __floats2bfloat162_rn(c[0] * m0, c[1] * m1);
        *reinterpret_cast<__nv_bfloat162*>(dX + (g + 8) * dxs + col) = __floats2bfloat162_rn(c[2] * m2, c[3] * m3);
    }
}

// dW[out][in] += dZ^T X over the warp's 16 rows, accumulated into shared fp32 (row stride = in).
template <int kInDim, int kOutDim>
__device__ __forceinline__ void dense_backward_weight(const __nv_bfloat16* dZ, int dzs, const __nv_bfloat16* X, int xs,
                                                      float* dW) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int j = lane >> 3, r = lane & 7;
#pragma unroll
    for (int mt = 0; mt < kOutDim / 16; ++mt) {
        uint32_t a[4];
        // A[m = out][k = row] = dZ^T: transposed loads of dZ[row][out]
        ldsm_x4_t(a, dZ + ((j >> 1) * 8 + r) * dzs + mt * 16 + (j & 1) * 8);
#pragma unroll
        for (int nt = 0; nt < kInDim / 8; ++nt) {
            uint32_t b[2];
            // B[k = row][n = in] from X[row][in]: transposed loads
            ldsm_x2_t(b, X + (lane & 15) * xs + nt * 8);
            float c[4] = { 0.f, 0.f, 0.f, 0.f };
            mma16816(c, a, b);
            const int o0 = mt * 16 + g, i0 = nt * 8 + 2 * t;
            atomicAdd(&dW[o0 * kInDim + i0], c[0]);
            atomicAdd(&dW[o0 * kInDim + i0 + 1], c[1]);
            atomicAdd(&dW[(o0 + 8) * kInDim + i0], c[2]);
            atomicAdd(&dW[(o0 + 8) * kInDim + i0 + 1], c[3]);
        }
    }
}

// ---- input encoding --------------------------------------------------------------------------------
__device__ __forceinline__ void blob12(float x, __nv_bfloat16* out) {
    x = fminf(fmaxf(x, 0.f), 1.f) * 12.f;
#pragma unroll
    for (int i = 0; i < 12; ++i) out[i] = __float2bfloat16_rn(fmaxf(0.f, 1.f - fabsf(x - ((float)i + 0.5f))));
}
__device__ __forceinline__ void dir_angles(float x, float y, float z, float& th, float& ph) {
    th = acosf(fminf(fmaxf(z, -1.f), 1.f)) * 0.318309886183790671538f;
    ph = (atan2f(y, x) + 3.14159265358979323846f) * 0.159154943091895335769f;
}
// f[0..8] = pos01 xyz, normal xyz, wo xyz
__device__ __forceinline__ void encode_row(const float* f, __nv_bfloat16* row) {
    blob12(f[0], row + 0);
    blob12(f[1], row + 12);
    blob12(f[2], row + 24);
    float th, ph;
    dir_angles(f[3], f[4], f[5], th, ph);
    blob12(th, row + 36);
    blob12(ph, row + 48);
    dir_angles(f[6], f[7], f[8], th, ph);
    blob12(th, row + 60);
    blob12(ph, row + 72);
    row[84] = __float2bfloat16_rn(1.f);
#pragma unroll
    for (int i = 85; i < 96; ++i) row[i] = __float2bfloat16_rn(0.f);
}

// ---- vMF mixture --------------------------------------------------------------------------------------
struct Mixture {
    float w[kLobes];      // weights (softmax)
    float mu[kLobes][3];  // unit means
    float kappa[kLobes];
};

__device__ __forceinline__ float softplus(float x) { return x > 20.f ? x : log1pf(expf(x)); }

__device__ __forceinline__ void mixture_from_raw(const float* y, Mixture& m) {
    float mx = -3.0e38f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, y[5 * k]);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        m.w[k] = expf(y[5 * k] - mx);
        s += m.w[k];
    }
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        m.w[k] /= s;
        const float vx = y[5 * k + 1], vy = y[5 * k + 2], vz = y[5 * k + 3];
        const float n = sqrtf(vx * vx + vy * vy + vz * vz);
        if (n > 1e-12f) { m.mu[k][0] = vx / n; m.mu[k][1] = vy / n; m.mu[k][2] = vz / n; }
        else { m.mu[k][0] = 0.f; m.mu[k][1] = 0.f; m.mu[k][2] = 1.f; }
        m.kappa[k] = fminf(softplus(y[5 * k + 4]) + kKappaMin, kKappaMax);
    }
}

__device__ __forceinline__ float vmf_eval(const float* mu, float kappa, float x, float y, float z) {
    const float c = kappa / (6.2831853071795864f * (-expm1f(-2.f * kappa)));
    return c * expf(kappa * (mu[0] * x + mu[1] * y + mu[2] * z - 1.f));
}

__device__ __forceinline__ float mixture_pdf(const Mixture& m, float x, float y, float z) {
    float p = 0.f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) p += m.w[k] * vmf_eval(m.mu[k], m.kappa[k], x, y, z);
    return p;
}

// Lobe chosen by the weights' CDF with u_lobe; direction by inverting the vMF in the lobe's frame.
__device__ __forceinline__ void mixture_sample(const Mixture& m, float u_lobe, float u1, float u2, float& x, float& y,
                                               float& z) {
    int k = kLobes - 1;
    float c = 0.f;
#pragma unroll
    for (int i = 0; i < kLobes; ++i) {
        c += m.w[i];
        if (u_lobe < c) { k = i; break; }
    }
    const float kk = m.kappa[k];
    const float wz = fminf(1.f, fmaxf(-1.f, 1.f + logf(u1 + (1.f - u1) * expf(-2.f * kk)) / kk));
    const float r = sqrtf(fmaxf(0.f, 1.f - wz * wz));
    float sp, cp;
    sincosf(6.2831853071795864f * u2, &sp, &cp);
    const float lx = r * cp, ly = r * sp;
    const float* mu = m.mu[k];
    const float sign = mu[2] >= 0.f ? 1.f : -1.f;
    const float a = -1.f / (sign + mu[2]);
    const float b = mu[0] * mu[1] * a;
    const float tx = 1.f + sign * mu[0] * mu[0] * a, ty = sign * b, tz = -sign * mu[0];
    const float bx = b, by = sign + mu[1] * mu[1] * a, bz = -mu[1];
    x = lx * tx + ly * bx + wz * mu[0];
    y = lx * ty + ly * by + wz * mu[1];
    z = lx * tz + ly * bz + wz * mu[2];
}

// d(-g log q(wi)) / d raw outputs for one sample (g = the sample's loss weight); returns log q.
__device__ __forceinline__ float mixture_loss_grad(const float* y, float wx, float wy, float wz, float g, float* dy) {
    Mixture m;
    mixture_from_raw(y, m);
    float comp[kLobes];
    float q = 0.f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        comp[k] = vmf_eval(m.mu[k], m.kappa[k], wx, wy, wz);
        q += m.w[k] * comp[k];
    }
    const float qs = fmaxf(q, 1e-30f);
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const float resp = m.w[k] * comp[k] / qs;
        dy[5 * k] = g * (resp - m.w[k]);
        const float kk = m.kappa[k];
        const float mdw = m.mu[k][0] * wx + m.mu[k][1] * wy + m.mu[k][2] * wz;
        const float dlogk = 1.f / kk - 2.f / expm1f(2.f * kk) + (mdw - 1.f);
        const float raw = y[5 * k + 4];
        const float sig = 1.f / (1.f + expf(-raw));
        const bool free_k = softplus(raw) + kKappaMin < kKappaMax;
        dy[5 * k + 4] = free_k ? g * resp * dlogk * sig : 0.f;
        const float vx = y[5 * k + 1], vy = y[5 * k + 2], vz = y[5 * k + 3];
        const float vn = fmaxf(sqrtf(vx * vx + vy * vy + vz * vz), 1e-30f);
        const float s = g * resp * kk / vn;
        dy[5 * k + 1] = s * (wx - mdw * m.mu[k][0]);
        dy[5 * k + 2] = s * (wy - mdw * m.mu[k][1]);
        dy[5 * k + 3] = s * (wz - mdw * m.mu[k][2]);
    }
#pragma unroll
    for (int i = 5 * kLobes; i < kOut; ++i) dy[i] = 0.f;
    return logf(qs);
}

constexpr int kWarps = 4;
constexpr int kThreads = kWarps * 32;

// shared-memory image: bf16 weights | fp32 biases | per-warp tiles
struct FwdTile {
    __nv_bfloat16 x[16 * kXStride];
    __nv_bfloat16 h[2][16 * kHStride];
    float y[16 * kOut];
};
struct TrainTile {
    __nv_bfloat16 x[16 * kXStride];
    __nv_bfloat16 h[4][16 * kHStride];
    __nv_bfloat16 dz[2][16 * kHStride];
    float y[16 * kOut];
    float feat[16 * 16];
};

template <typename View>
__device__ __forceinline__ void load_weights(const View& gv, __nv_bfloat16* w_s, float* b_s) {
    const int4* src = reinterpret_cast<const int4*>(gv.w16);
    int4* dst = reinterpret_cast<int4*>(w_s);
    for (int i = threadIdx.x; i < kW16Elems / 8; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < kBiasElems; i += blockDim.x) b_s[i] = gv.b32[i];
}

__device__ __forceinline__ void forward_tile(const __nv_bfloat16* w_s, const float* b_s, const __nv_bfloat16* x,
                                             __nv_bfloat16* h0, __nv_bfloat16* h1, float* y) {
    dense_forward<kIn, kHid, true>(x, kXStride, w_s + w16_offset(0), layer_stride(0), b_s + bias_offset(0), h0, kHStride,
                                   nullptr, 0);
    __syncwarp();
    dense_forward<kHid, kHid, true>(h0, kHStride, w_s + w16_offset(1), layer_stride(1), b_s + bias_offset(1), h1,
                                    kHStride, nullptr, 0);
    __syncwarp();
    dense_forward<kHid, kHid, true>(h1, kHStride, w_s + w16_offset(2), layer_stride(2), b_s + bias_offset(2), h0,
                                    kHStride, nullptr, 0);
    __syncwarp();
    dense_forward<kHid, kHid, true>(h0, kHStride, w_s + w16_offset(3), layer_stride(3), b_s + bias_offset(3), h1,
                                    kHStride, nullptr, 0);
    __syncwarp();
    dense_forward<kHid, kOut, false>(h1, kHStride, w_s + w16_offset(4), layer_stride(4), b_s + bias_offset(4), nullptr,
                                     0, y, kOut);
    __syncwarp();
}

}  // namespace guide
}  // namespace pb2
