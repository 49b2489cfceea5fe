// guiding_tc.cuh -- the guiding network's forward pass on the 5th-generation tensor cores (tcgen05).
//
// A CTA holds the weights of all five layers once in shared memory and runs G independent warp
// groups of 4 warps (TcLayout<G>); each group evaluates its own 128-row tiles, so while one group waits for its MMAs
// another encodes inputs or drains its accumulator (the tensor pipe is shared by the groups of the SM).
// The encoded inputs and each hidden layer's output are bf16 operands in shared memory in the canonical
// K-major, no-swizzle UMMA layout (8-row x 16-byte core matrices; within a tile, core matrices adjacent in
// K are 128 bytes apart (LBO) and 8-row groups are K x 16 bytes apart (SBO)); the weights use the same
// layout.  For each layer one thread of the group issues K/16 `tcgen05.mma.cta_group::1.kind::f16`
// (M = 128, N = 64 or 48, BF16 x BF16 -> FP32) into the group's 64 TMEM columns and commits them to the
// group's mbarrier; every warp of the group then reads its 32 rows back with `tcgen05.ld.32x32b`, adds the
// bias, and writes the next layer's bf16 operand (ReLU and rounding of two columns in one `cvt.rn.relu.bf16x2`)
// over the one the completed MMAs read (a group has one operand buffer), and after the last layer the buffer
// stages the fp32 outputs so that a row-major output is written with coalesced stores.  Each thread loads its
// next tile's input row while the current tile's layers run.  Shared-memory writes that
// an MMA reads are made visible to the tensor core's async proxy with `fence.proxy.async.shared::cta`
// before the group's named barrier.
//
// Every wait on an mbarrier is bounded: on time-out the group records an error, stops issuing work, gives
// the tensor core a bounded time to drain, and the CTA frees its TMEM and returns.
#pragma once
#include <cuda_bf16.h>

#include "guiding.cuh"
#include "pb2_internal.h"

namespace pb2 {
namespace guide {

constexpr int kTcRows = 128;
constexpr int kTcGroupThreads = 128;
constexpr uint32_t kTmemColsPerGroup = 64;
constexpr uint32_t kWaitLimit = 1u << 20;  // mbarrier polls before a wait counts as failed

__host__ __device__ constexpr int tc_w_offset(int l) {  // bytes of layer l's weights in the staged image
    return l == 0 ? 0 : tc_w_offset(l - 1) + layer_out(l - 1) * layer_in(l - 1) * 2;
}
constexpr int kTcWBytes = tc_w_offset(kLayers);                        // 43,008
constexpr int kTcABytes = kTcRows * kIn * 2;                           // 24,576: a group's one operand buffer (the
                                                                       // input tile, each hidden layer's output written
                                                                       // over the input its MMA has consumed, and the
                                                                       // fp32 output staging, 128 x 48)

// Shared-memory layout and sizes of a CTA of G warp groups.
template <int G>
struct TcLayout {
    static constexpr int kGroups = G;
    static constexpr int kThreads = kTcGroupThreads * G;
    static constexpr uint32_t kTmemCols = G * kTmemColsPerGroup <= 128 ? 128u : G * kTmemColsPerGroup <= 256 ? 256u : 512u;
    static constexpr int kOffW = 0;
    static constexpr int kOffGroups = kTcWBytes;                       // 1024-aligned
    static constexpr int kOffBias = kOffGroups + G * kTcABytes;
    static constexpr int kOffBar = kOffBias + kBiasElems * 4;          // G mbarriers
    static constexpr int kOffSlot = kOffBar + 8 * G;                   // TMEM base address
    static constexpr int kOffFail = kOffSlot + 4;                      // G failure flags
    static constexpr int kSmem = kOffFail + 4 * G;
    static_assert(kOffGroups % 1024 == 0 && kTcABytes % 1024 == 0, "operand alignment");
    static_assert(kTcABytes >= kTcRows * kOut * 4, "output staging fits the operand buffer");
    static_assert(kOffBar % 8 == 0, "mbarrier alignment");
    static_assert(kSmem <= 227 * 1024, "shared memory per CTA");
    static_assert(G * kTmemColsPerGroup <= 512, "tensor memory per SM");
};
// The batched forward (k_forward_tc): seven groups, as many 128-row tiles in flight as shared memory holds
// (7 x 24 KB of operands beside the 43 KB of weights).  The in-render inference keeps four (its epilogue holds
// a row's 48 outputs in registers for the mixture).
constexpr int kTcGroupsForward = 7;
constexpr int kTcGroupsInfer = 4;

// Byte offset of element (row, k) of a K-major operand with `kdim` columns in the core-matrix layout.
__host__ __device__ constexpr uint32_t core_offset(uint32_t row, uint32_t k, uint32_t kdim) {
    return (row >> 3) * (kdim * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
    return d;
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t instr_desc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Two floats rounded to bf16 and packed (lo in the low half), with and without ReLU; `cvt.rn.relu` clamps the
// rounded value at 0, which for any float equals rounding max(x, 0).
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ uint32_t pack_relu_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


// Barrier of one warp group (named barrier 1 + g; barrier 0 is __syncthreads).
__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(kTcGroupThreads) : "memory");
}

// The encoded input row written straight into the operand buffer, 8 bf16 (16 bytes) at a time, with encode_row's
// arithmetic: 7 blob features of 12 bins (position xyz, the normal's and the outgoing direction's angles), a
// constant 1 at 84, zeros to 96.  Only the 7 scaled features live in registers.
__device__ __forceinline__ void encode_row_tile(const float (&f)[9], unsigned char* tile, uint32_t row) {
    float s[7];
    s[0] = fminf(fmaxf(f[0], 0.f), 1.f) * 12.f;
    s[1] = fminf(fmaxf(f[1], 0.f), 1.f) * 12.f;
    s[2] = fminf(fmaxf(f[2], 0.f), 1.f) * 12.f;
    float th, ph;
    dir_angles(f[3], f[4], f[5], th, ph);
    s[3] = fminf(fmaxf(th, 0.f), 1.f) * 12.f;
    s[4] = fminf(fmaxf(ph, 0.f), 1.f) * 12.f;
    dir_angles(f[6], f[7], f[8], th, ph);
    s[5] = fminf(fmaxf(th, 0.f), 1.f) * 12.f;
    s[6] = fminf(fmaxf(ph, 0.f), 1.f) * 12.f;
#pragma unroll
    for (int kc = 0; kc < kIn / 8; ++kc) {
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = kc * 8 + i;
            x[i] = 0.f;
            if (e < 84) x[i] = fmaxf(0.f, 1.f - fabsf(s[e / 12] - ((float)(e % 12) + 0.5f)));
            else if (e == 84) x[i] = 1.f;
        }
        *reinterpret_cast<uint4*>(tile + core_offset(row, kc * 8, kIn)) =
            make_uint4(pack_bf16x2(x[0], x[1]), pack_bf16x2(x[2], x[3]), pack_bf16x2(x[4], x[5]), pack_bf16x2(x[6], x[7]));
    }
}

// The tile loop of the tensor-core forward pass, for a CTA of TcLayout<G>::kThreads threads with
// TcLayout<G>::kSmem bytes of dynamic shared memory.  Rows: thread t of a group handles row tile * 128 + t of the
// n rows; rows.features(row, f, key) fills the 9 input features and a key the thread keeps.  Outputs: with
// Rows::kStaged, rows.store_tile(row0, count, staged, t, threads) writes rows [row0, row0 + count) from the
// group's staged fp32 outputs (row-major, 48 per row) cooperatively; otherwise rows.output(key, y) receives
// the 48 raw outputs of a row below n.  error[0] is set when a tensor-core wait timed out.
//
// Each group has one operand buffer: layer l's MMAs read it, and once they have completed (the group waited on
// its mbarrier) the epilogue writes layer l + 1's operand over it; after the last layer it stages the outputs.
template <int G, class Rows>
__device__ __forceinline__ void forward_tc_tiles(const GuideView& gv, uint32_t n, const Rows& rows, uint32_t* error,
                                                 unsigned char* smem) {
    using L = TcLayout<G>;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = tid / kTcGroupThreads, gt = tid % kTcGroupThreads;  // group and thread within it
    unsigned char* w_s = smem + L::kOffW;
    unsigned char* buf = smem + L::kOffGroups + g * kTcABytes;
    float* b_s = reinterpret_cast<float*>(smem + L::kOffBias);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::kOffBar) + g;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L::kOffSlot);
    volatile uint32_t& s_fail = reinterpret_cast<uint32_t*>(smem + L::kOffFail)[g];
    // a CTA without a tile (the in-render queue is often empty or short) leaves before staging weights or
    // allocating tensor memory; the condition is the same for all its threads
    if ((uint64_t)blockIdx.x * G * kTcRows >= n) return;

    // weights: padded row-major bf16 image -> core-matrix layout, 16 bytes at a time (all groups)
    for (int l = 0; l < kLayers; ++l) {
        const int in = layer_in(l), outd = layer_out(l), chunks = outd * (in / 8);
        for (int c = tid; c < chunks; c += L::kThreads) {
            const int o = c / (in / 8), kc = c % (in / 8);
            const int4 v = *reinterpret_cast<const int4*>(gv.w16 + w16_offset(l) + o * layer_stride(l) + kc * 8);
            *reinterpret_cast<int4*>(w_s + tc_w_offset(l) + core_offset(o, kc * 8, in)) = v;
        }
    }
    for (int i = tid; i < kBiasElems; i += L::kThreads) b_s[i] = gv.b32[i];
    if (gt == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(L::kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + (uint32_t)g * kTmemColsPerGroup;  // this group's accumulator columns
    const uint32_t bar_addr = smem_u32(bar);
    uint32_t phase = 0;
    bool failed = false;

    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const uint32_t stride = gridDim.x * G;
    // the next tile's input row is loaded while this tile's layers run
    float fn[9] = { 0.5f, 0.5f, 0.5f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 1.0f };
    uint32_t key_next = 0;
    {
        const uint32_t row0 = (blockIdx.x * G + g) * kTcRows + gt;
        if (row0 < n) rows.features(row0, fn, key_next);
    }
    for (uint32_t tile = blockIdx.x * G + g; tile < tiles && !failed; tile += stride) {
        const uint32_t row = tile * kTcRows + gt;
        encode_row_tile(fn, buf, (uint32_t)gt);
        const uint32_t key = key_next;
        {
            const uint32_t nrow = (tile + stride) * kTcRows + gt;
            if (tile + stride < tiles && nrow < n) rows.features(nrow, fn, key_next);
        }
        fence_async_smem();
        tc_fence_before();
        group_sync(g);
        tc_fence_after();
        float y[Rows::kStaged ? 1 : kOut];
        for (int l = 0; l < kLayers; ++l) {
            const uint32_t kdim = layer_in(l), ndim = layer_out(l);
            if (gt == 0) {
                const uint32_t a0 = smem_u32(buf), b0 = smem_u32(w_s + tc_w_offset(l));
                for (uint32_t k = 0; k < kdim / 16; ++k)
                    mma_bf16(tmem, smem_desc(a0 + 256 * k, 128, kdim * 16), smem_desc(b0 + 256 * k, 128, kdim * 16),
                             instr_desc(ndim), k > 0 ? 1u : 0u);
                mma_commit(bar_addr);
            }
            if (!mbar_wait_bounded(bar_addr, phase)) {
                s_fail = 1u;
                atomicExch(error, 1u);
            }
            phase ^= 1u;
            tc_fence_after();
            // (a wait that gave up is agreed on at the group barrier after the epilogue, which every thread reaches)
            // epilogue: this warp's 32 rows (TMEM lanes 32 (warp % 4) ..), 16 columns at a time; the layer's MMAs
            // have completed, so the operand buffer is free for the next layer's operand (or the staged outputs)
            const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
            float* st = reinterpret_cast<float*>(buf);
            for (uint32_t c0 = 0; c0 < ndim; c0 += 16) {
                float v[16];
                tmem_ld16(lane_base + c0, v);
                tmem_wait_ld();
                const float* bias = b_s + bias_offset(l) + c0;
                if (l < kLayers - 1) {
                    // bias, ReLU and the bf16 rounding of two columns per instruction
                    uint32_t hw[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) hw[i] = pack_relu_bf16x2(v[2 * i] + bias[2 * i], v[2 * i + 1] + bias[2 * i + 1]);
                    *reinterpret_cast<uint4*>(buf + core_offset(gt, c0, kHid)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                    *reinterpret_cast<uint4*>(buf + core_offset(gt, c0 + 8, kHid)) = make_uint4(hw[4], hw[5], hw[6], hw[7]);
                } else if constexpr (Rows::kStaged) {
                    // fp32 outputs row-major over the consumed operand
#pragma unroll
                    for (int i = 0; i < 16; i += 4)
                        *reinterpret_cast<float4*>(st + gt * kOut + c0 + i) =
                            make_float4(v[i] + bias[i], v[i + 1] + bias[i + 1], v[i + 2] + bias[i + 2], v[i + 3] + bias[i + 3]);
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) y[c0 + i] = v[i] + bias[i];
                }
            }
            if (l == kLayers - 1) {
                if constexpr (Rows::kStaged) {
                    group_sync(g);
                    const uint32_t row0 = tile * kTcRows;
                    rows.store_tile(row0, min((uint32_t)kTcRows, n - row0), st, gt, kTcGroupThreads);
                } else if (row < n) {
                    rows.output(key, y);
                }
            }
            fence_async_smem();
            tc_fence_before();
            group_sync(g);
            tc_fence_after();
            if (s_fail) {
                failed = true;
                break;
            }
        }
    }
    if (failed && gt == 0) {
        // give any MMA still in flight a bounded time to finish before its TMEM is freed
        mbar_wait_bounded(bar_addr, phase);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(L::kTmemCols));
}

template <int G>
constexpr size_t forward_tc_smem() { return (size_t)TcLayout<G>::kSmem; }

}  // namespace guide
}  // namespace pb2
