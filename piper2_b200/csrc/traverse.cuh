// traverse.cuh -- closest-hit and any-hit traversal of the 8-wide quantised BVH.
//
// Traversal order and node groups follow Ylitie, Karras and Laine (HPG 2017): a node group is
// (child_base, hit bits 24..31 | imask), the highest hit bit is visited first, and the ray octant is
// XOR-ed into the internal-child bit positions so children are visited near to far.  Triangles of
// hit leaves are tested as soon as their node is opened.
//
// Box tests are conservative: each slab distance t = (p + q 2^e - o) / d is computed as
// fma(q, 2^e / d, (p - o) / d), whose rounding error is bounded per node and axis by
// 2 eps (255 |2^e/d| + 2 |(p-o)/d|); that bound (with a 2x margin) is subtracted from the near and added
// to the far plane, so rounding never culls a box that holds the true closest hit.  The triangle
// test is the watertight test shared with the CPU oracle, ties in t resolve to the lower primitive
// id, so the result does not depend on traversal order and equals the oracle's bit for bit.
#pragma once
#include "pb2_bvh.h"
#include "pb2_device.cuh"

namespace pb2 {

constexpr int kStackSize = 48;
#ifndef PB2_CHILD_UNROLL
#define PB2_CHILD_UNROLL 8
#endif
// Copies of the child-test body.  Measured on a B200 (1M-triangle soup): with the iteration loops rolled,
// the fully unrolled child loop is 16 % faster than the rolled one (692 -> 804 Mrays/s closest hit).
constexpr int kChildUnroll = PB2_CHILD_UNROLL;

struct TraceResult {
    float t, u, v;
    uint32_t prim;
};

__device__ __forceinline__ float safe_rcp(float d) {
    const float a = fmaxf(fabsf(d), 1e-18f);
    return copysignf(__frcp_rn(a), d);
}

// Intersects the eight children of `node`; returns the hit mask (internal children at bits
// 24 + (slot ^ oct_inv), leaf triangles at their offsets), and the node's child/tri bases and imask.
__device__ __forceinline__ uint32_t intersect_children(const WideNode* __restrict__ nodes, uint32_t node_index,
                                                       const RayPre& p, float ix, float iy, float iz,
                                                       uint32_t oct_inv, float tbest, uint32_t& child_base,
                                                       uint32_t& tri_base, uint32_t& imask) {
    const uint4* nw = reinterpret_cast<const uint4*>(nodes + node_index);
    const uint4 w0 = __ldg(nw + 0);
    const uint4 w1 = __ldg(nw + 1);
    const uint4 w2 = __ldg(nw + 2);
    const uint4 w3 = __ldg(nw + 3);
    const uint4 w4 = __ldg(nw + 4);
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t ex = w0.w & 0xFFu, ey = (w0.w >> 8) & 0xFFu, ez = (w0.w >> 16) & 0xFFu;
    imask = w0.w >> 24;
    child_base = w1.x;
    tri_base = w1.y;
    const float ax = __uint_as_float(ex << 23) * ix;
    const float ay = __uint_as_float(ey << 23) * iy;
    const float az = __uint_as_float(ez << 23) * iz;
    const float bx = (px - p.ox) * ix;
    const float by = (py - p.oy) * iy;
    const float bz = (pz - p.oz) * iz;
    const float kEps2 = 4.0f * 5.9604645e-8f;
    const float dx = kEps2 * __fmaf_rn(256.0f, fabsf(ax), 2.0f * fabsf(bx));
    const float dy = kEps2 * __fmaf_rn(256.0f, fabsf(ay), 2.0f * fabsf(by));
    const float dz = kEps2 * __fmaf_rn(256.0f, fabsf(az), 2.0f * fabsf(bz));
    const float bnx = bx - dx, bfx = bx + dx;
    const float bny = by - dy, bfy = by + dy;
    const float bnz = bz - dz, bfz = bz + dz;
    // near/far quantised planes per axis, chosen by the sign of the direction
    const uint32_t nx_lo = ix >= 0.0f ? w2.x : w3.z, nx_hi = ix >= 0.0f ? w2.y : w3.w;
    const uint32_t fx_lo = ix >= 0.0f ? w3.z : w2.x, fx_hi = ix >= 0.0f ? w3.w : w2.y;
    const uint32_t ny_lo = iy >= 0.0f ? w2.z : w4.x, ny_hi = iy >= 0.0f ? w2.w : w4.y;
    const uint32_t fy_lo = iy >= 0.0f ? w4.x : w2.z, fy_hi = iy >= 0.0f ? w4.y : w2.w;
    const uint32_t nz_lo = iz >= 0.0f ? w3.x : w4.z, nz_hi = iz >= 0.0f ? w3.y : w4.w;
    const uint32_t fz_lo = iz >= 0.0f ? w4.z : w3.x, fz_hi = iz >= 0.0f ? w4.w : w3.y;
    // The eight child tests (unrolled: see kChildUnroll).
    uint32_t hitmask = 0;
#pragma unroll kChildUnroll
    for (int j = 0; j < 8; ++j) {
        const bool hi = j >= 4;
        const uint32_t sel = 0x7540u | (uint32_t)(j & 3);
        const uint32_t meta = ((hi ? w1.w : w1.z) >> (8 * (j & 3))) & 0xFFu;
        const float qnx = __uint_as_float(__byte_perm(hi ? nx_hi : nx_lo, 0x4B000000u, sel)) - 8388608.0f;
        const float qfx = __uint_as_float(__byte_perm(hi ? fx_hi : fx_lo, 0x4B000000u, sel)) - 8388608.0f;
        const float qny = __uint_as_float(__byte_perm(hi ? ny_hi : ny_lo, 0x4B000000u, sel)) - 8388608.0f;
        const float qfy = __uint_as_float(__byte_perm(hi ? fy_hi : fy_lo, 0x4B000000u, sel)) - 8388608.0f;
        const float qnz = __uint_as_float(__byte_perm(hi ? nz_hi : nz_lo, 0x4B000000u, sel)) - 8388608.0f;
        const float qfz = __uint_as_float(__byte_perm(hi ? fz_hi : fz_lo, 0x4B000000u, sel)) - 8388608.0f;
        const float tn = fmaxf(fmaxf(__fmaf_rn(qnx, ax, bnx), __fmaf_rn(qny, ay, bny)),
                               fmaxf(__fmaf_rn(qnz, az, bnz), p.tmin));
        const float tf = fminf(fminf(__fmaf_rn(qfx, ax, bfx), __fmaf_rn(qfy, ay, bfy)),
                               fminf(__fmaf_rn(qfz, az, bfz), tbest));
        if (meta != 0u && tn <= tf) {
            const uint32_t inner = ((meta & (meta << 1)) & 0x10u) != 0u;
            const uint32_t bit_index = inner ? ((meta & 0x1Fu) ^ oct_inv) : (meta & 0x1Fu);
            hitmask |= (meta >> 5) << bit_index;
        }
    }
    return hitmask;
}

// Plane test of the area-light parallelograms, operation for operation as the oracle's
// (planeIntersect + calcTexCoord, Src/BuiltinComponent/Geometry/BasicShapes/Kernel.cpp:30-79).
__device__ __forceinline__ bool plane_test(const DevPlane& pl, const RayPre& p, float tnear, float tfar, float& t_out,
                                           float& u_out, float& v_out, bool& front) {
    const float ox = RN_SUB(p.ox, pl.translation[0]), oy = RN_SUB(p.oy, pl.translation[1]),
                oz = RN_SUB(p.oz, pl.translation[2]);
    const float len = sqrtf(fmaxf(RN_ADD(RN_ADD(RN_MUL(p.dx, p.dx), RN_MUL(p.dy, p.dy)), RN_MUL(p.dz, p.dz)), 0.0f));
    const float dx = RN_DIV(p.dx, len), dy = RN_DIV(p.dy, len), dz = RN_DIV(p.dz, len);
    const float ex = RN_SUB(pl.origin[0], ox), ey = RN_SUB(pl.origin[1], oy), ez = RN_SUB(pl.origin[2], oz);
    const float b = RN_ADD(RN_ADD(RN_MUL(ex, pl.normal[0]), RN_MUL(ey, pl.normal[1])), RN_MUL(ez, pl.normal[2]));
    const float k = RN_ADD(RN_ADD(RN_MUL(dx, pl.normal[0]), RN_MUL(dy, pl.normal[1])), RN_MUL(dz, pl.normal[2]));
    const float t = RN_DIV(b, k);
    if (!(tnear < t && t < tfar)) return false;
    const float hx = RN_SUB(RN_MUL(dx, t), ex), hy = RN_SUB(RN_MUL(dy, t), ey), hz = RN_SUB(RN_MUL(dz, t), ez);
    const float* u = pl.u;
    const float* v = pl.v;
    float inv_det, x, y;
    if (pl.max_det_comp == 0) {
        inv_det = RN_DIV(1.0f, RN_SUB(RN_MUL(u[1], v[2]), RN_MUL(v[1], u[2])));
        x = RN_SUB(RN_MUL(hy, v[2]), RN_MUL(v[1], hz));
        y = RN_SUB(RN_MUL(u[1], hz), RN_MUL(hy, u[2]));
    } else if (pl.max_det_comp == 1) {
        inv_det = RN_DIV(1.0f, RN_SUB(RN_MUL(u[2], v[0]), RN_MUL(v[2], u[0])));
        x = RN_SUB(RN_MUL(hz, v[0]), RN_MUL(v[2], hx));
        y = RN_SUB(RN_MUL(u[2], hx), RN_MUL(hz, u[0]));
    } else {
        inv_det = RN_DIV(1.0f, RN_SUB(RN_MUL(u[0], v[1]), RN_MUL(v[0], u[1])));
        x = RN_SUB(RN_MUL(hx, v[1]), RN_MUL(v[0], hy));
        y = RN_SUB(RN_MUL(u[0], hy), RN_MUL(hx, u[1]));
    }
    const float uu = RN_MUL(x, inv_det), vv = RN_MUL(y, inv_det);
    if (!(0.0f <= uu && uu <= 1.0f && 0.0f <= vv && vv <= 1.0f)) return false;
    t_out = t;
    u_out = uu;
    v_out = vv;
    front = k > 0.0f;
    return true;
}

// Traversal stack: the top kSharedStack entries live in shared memory, transposed so that consecutive
// lanes touch consecutive words ([depth][thread]); deeper entries spill to a small local array.
#ifndef PB2_SHARED_STACK
#define PB2_SHARED_STACK 12
#endif
constexpr int kSharedStack = PB2_SHARED_STACK;
constexpr int kLocalStack = 48 - PB2_SHARED_STACK;
static_assert(kSharedStack + kLocalStack == kStackSize, "stack depth");

// Per-lane traversal state.  kClosest selects closest-hit vs any-hit semantics.
template <bool kClosest, bool kCount, int kThreads>
struct Traverser {
    RayPre p;
    float ix, iy, iz;
    uint32_t oct_inv;
    float tbest, bu, bv;
    uint32_t best_prim;
    uint32_t best_slot;
    uint2 group;
    uint2 tgroup;
    uint2* sstack;  // this lane's column of the shared stack
    uint2 lstack[kLocalStack];
    int sp;
    bool done;
    bool overflow;
    uint32_t node_visits, tri_tests;

    __device__ __forceinline__ void bind_stack(uint2* shared_base) { sstack = shared_base + threadIdx.x; }

    __device__ __forceinline__ void push(uint2 g) {
        if (sp < kSharedStack) sstack[sp * kThreads] = g;
        else if (sp < kStackSize) lstack[sp - kSharedStack] = g;
        else { overflow = true; return; }
        ++sp;
    }
    __device__ __forceinline__ uint2 pop() {
        --sp;
        return sp < kSharedStack ? sstack[sp * kThreads] : lstack[sp - kSharedStack];
    }

    __device__ __forceinline__ void init(const BvhView& bvh, float ox, float oy, float oz, float tmin, float dx,
                                         float dy, float dz, float tmax) {
        ray_prepare(ox, oy, oz, tmin, dx, dy, dz, tmax, p);
        ix = safe_rcp(dx);
        iy = safe_rcp(dy);
        iz = safe_rcp(dz);
        const uint32_t oct = (dx < 0.0f ? 1u : 0u) | (dy < 0.0f ? 2u : 0u) | (dz < 0.0f ? 4u : 0u);
        oct_inv = 7u - oct;
        tbest = tmax;
        bu = bv = 0.0f;
        best_prim = kInvalidPrim;
        best_slot = 0;
        sp = 0;
        overflow = false;
        node_visits = tri_tests = 0;
        tgroup = make_uint2(0, 0);
        if (bvh.tri_count == 0) {
            group = make_uint2(0, 0);
            done = true;
        } else {
            // the root as the only internal "child", in slot 0
            group = make_uint2(0u, (1u << (24u + oct_inv)) | 1u);
            done = false;
        }
    }

    __device__ __forceinline__ void test_tri(const BvhView& bvh, uint32_t slot) {
        const float4* t4 = reinterpret_cast<const float4*>(bvh.tris + slot);
        const float4 a = __ldg(t4 + 0), b = __ldg(t4 + 1), c = __ldg(t4 + 2);
        const uint32_t prim = __float_as_uint(a.w);
        if (kCount) ++tri_tests;
        float t, u, v;
        if (tri_test(p, a, b, c, t, u, v)) {
            if (!kClosest) {
                best_prim = prim;
                tbest = t;
                done = true;
            } else if (t < tbest || (t == tbest && prim < best_prim)) {
                tbest = t;
                bu = u;
                bv = v;
                best_prim = prim;
                best_slot = slot;
            }
        }
    }

    // One iteration: open the nearest pending internal child (if any), then test the triangles of the
    // leaves it hit.  (Postponing sparse triangle groups onto the stack, as in Ylitie et al., did not
    // measure faster on this hardware and is not done.)
    __device__ __forceinline__ void iteration(const BvhView& bvh) {
        if (group.y > 0x00FFFFFFu) {
            const uint32_t hits = group.y;
            const uint32_t bit = 31u - __clz(hits);
            const uint32_t slot = (bit - 24u) ^ oct_inv;
            const uint32_t rel = __popc(hits & 0xFFu & ((1u << slot) - 1u));
            const uint32_t node = group.x + rel;
            group.y &= ~(1u << bit);
            if (group.y > 0x00FFFFFFu) push(group);
            if (kCount) ++node_visits;
            uint32_t child_base, tri_base, imask;
            const uint32_t hm = intersect_children(bvh.nodes, node, p, ix, iy, iz, oct_inv, kClosest ? tbest : p.tmax,
                                                   child_base, tri_base, imask);
            group = make_uint2(child_base, (hm & 0xFF000000u) | imask);
            tgroup = make_uint2(tri_base, hm & 0x00FFFFFFu);
        } else {
            tgroup = group;
            group = make_uint2(0, 0);
        }
        while (tgroup.y != 0u) {
            const uint32_t b = __ffs(tgroup.y) - 1u;
            tgroup.y &= tgroup.y - 1u;
            test_tri(bvh, tgroup.x + b);
            if (!kClosest && done) return;
        }
        if (group.y <= 0x00FFFFFFu) {
            if (sp == 0) done = true;
            else group = pop();
        }
    }

    __device__ __forceinline__ void finish_planes(const BvhView& bvh, bool& plane_front) {
        plane_front = false;
        if constexpr (!kClosest) return;
        for (uint32_t i = 0; i < bvh.plane_count; ++i) {
            float t, u, v;
            bool front;
            if (plane_test(bvh.planes[i], p, p.tmin, tbest, t, u, v, front)) {
                tbest = t;
                bu = u;
                bv = v;
                best_prim = kPlaneFlag | i;
                plane_front = front;
            }
        }
    }
};

}  // namespace pb2
