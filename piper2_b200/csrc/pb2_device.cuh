// pb2_device.cuh -- device-side building blocks shared by the traversal and integrator kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pb2_math.h"

// Non-contracted IEEE operations.  The library is built with -fmad=false, and the operations whose
// rounding must match the CPU oracle bit for bit (the watertight triangle test, the plane test) are in
// addition spelled with the _rn intrinsics, which nvcc never fuses whatever the flags.
#define RN_MUL(a, b) __fmul_rn((a), (b))
#define RN_ADD(a, b) __fadd_rn((a), (b))
#define RN_SUB(a, b) __fsub_rn((a), (b))
#define RN_DIV(a, b) __fdiv_rn((a), (b))

namespace pb2 {

constexpr uint32_t kInvalidPrim = 0xFFFFFFFFu;
constexpr uint32_t kPlaneFlag = 0x80000000u;

struct RayPre {
    float ox, oy, oz;
    float dx, dy, dz;
    float idx, idy, idz;  // 1/d (copysign(FLT_MAX) for zero components)
    float sx, sy, sz;     // watertight shear constants
    int kx, ky, kz;
    float tmin, tmax;
};

__device__ __forceinline__ float comp3(float a, float b, float c, int k) { return k == 0 ? a : (k == 1 ? b : c); }

// Ray set-up of the watertight test (Woop, Benthin, Wald, JCGT 2013, Sec. 3).
__device__ __forceinline__ void ray_prepare(float ox, float oy, float oz, float tmin, float dx, float dy, float dz,
                                            float tmax, RayPre& p) {
    p.ox = ox; p.oy = oy; p.oz = oz;
    p.dx = dx; p.dy = dy; p.dz = dz;
    p.tmin = tmin; p.tmax = tmax;
    p.idx = dx != 0.0f ? RN_DIV(1.0f, dx) : copysignf(3.402823466e38f, dx);
    p.idy = dy != 0.0f ? RN_DIV(1.0f, dy) : copysignf(3.402823466e38f, dy);
    p.idz = dz != 0.0f ? RN_DIV(1.0f, dz) : copysignf(3.402823466e38f, dz);
    int kz = 0;
    if (fabsf(dy) > fabsf(dx)) kz = 1;
    if (fabsf(dz) > fabsf(comp3(dx, dy, dz, kz))) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const float dkz = comp3(dx, dy, dz, kz);
    if (dkz < 0.0f) { const int t = kx; kx = ky; ky = t; }
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.sx = RN_DIV(comp3(dx, dy, dz, kx), dkz);
    p.sy = RN_DIV(comp3(dx, dy, dz, ky), dkz);
    p.sz = RN_DIV(1.0f, dkz);
}

// The paper's double-precision recomputation of U, V, W when one of them is exactly zero (an edge or
// vertex hit).  Rare, so kept out of line to keep the hot loop small.
static __device__ __noinline__ void edge_fallback(float Ax, float Ay, float Bx, float By, float Cx, float Cy, float& U,
                                                  float& V, float& W) {
    U = __double2float_rn(__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx)));
    V = __double2float_rn(__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx)));
    W = __double2float_rn(__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax)));
}

// Watertight ray/triangle test, identical operation for operation to the CPU oracle.  Returns true
// and writes t, (u, v) = weights of v1, v2 for a hit with tmin < t < tmax.
__device__ __forceinline__ bool tri_test(const RayPre& p, float4 a4, float4 b4, float4 c4, float& t_out, float& u_out,
                                         float& v_out) {
    const float Ax_ = RN_SUB(a4.x, p.ox), Ay_ = RN_SUB(a4.y, p.oy), Az_ = RN_SUB(a4.z, p.oz);
    const float Bx_ = RN_SUB(b4.x, p.ox), By_ = RN_SUB(b4.y, p.oy), Bz_ = RN_SUB(b4.z, p.oz);
    const float Cx_ = RN_SUB(c4.x, p.ox), Cy_ = RN_SUB(c4.y, p.oy), Cz_ = RN_SUB(c4.z, p.oz);
    const float Akz = comp3(Ax_, Ay_, Az_, p.kz), Bkz = comp3(Bx_, By_, Bz_, p.kz), Ckz = comp3(Cx_, Cy_, Cz_, p.kz);
    const float Ax = RN_SUB(comp3(Ax_, Ay_, Az_, p.kx), RN_MUL(p.sx, Akz));
    const float Ay = RN_SUB(comp3(Ax_, Ay_, Az_, p.ky), RN_MUL(p.sy, Akz));
    const float Bx = RN_SUB(comp3(Bx_, By_, Bz_, p.kx), RN_MUL(p.sx, Bkz));
    const float By = RN_SUB(comp3(Bx_, By_, Bz_, p.ky), RN_MUL(p.sy, Bkz));
    const float Cx = RN_SUB(comp3(Cx_, Cy_, Cz_, p.kx), RN_MUL(p.sx, Ckz));
    const float Cy = RN_SUB(comp3(Cx_, Cy_, Cz_, p.ky), RN_MUL(p.sy, Ckz));
    float U = RN_SUB(RN_MUL(Cx, By), RN_MUL(Cy, Bx));
    float V = RN_SUB(RN_MUL(Ax, Cy), RN_MUL(Ay, Cx));
    float W = RN_SUB(RN_MUL(Bx, Ay), RN_MUL(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) edge_fallback(Ax, Ay, Bx, By, Cx, Cy, U, V, W);
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = RN_ADD(RN_ADD(U, V), W);
    if (det == 0.0f) return false;
    const float Az = RN_MUL(p.sz, Akz), Bz = RN_MUL(p.sz, Bkz), Cz = RN_MUL(p.sz, Ckz);
    const float T = RN_ADD(RN_ADD(RN_MUL(U, Az), RN_MUL(V, Bz)), RN_MUL(W, Cz));
    const float t = RN_DIV(T, det);
    if (!(t > p.tmin && t < p.tmax)) return false;
    t_out = t;
    u_out = RN_DIV(V, det);
    v_out = RN_DIV(W, det);
    return true;
}

}  // namespace pb2
