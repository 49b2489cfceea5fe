// shading.cuh -- device restatement of the reference's per-sample math: Sobol sampling, camera,
// BxDFs, lights.  Every expression keeps the reference's operation order (the library is compiled
// with -fmad=false, so no operation is fused unless written as an explicit fma), which makes each
// path bit-identical to the CPU oracle's.  File:line citations refer to the reference's tree.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pb2_math.h"

namespace pb2 {

struct v3 {
    float x, y, z;
};
__device__ __forceinline__ v3 mk3(float x, float y, float z) { return v3{ x, y, z }; }
__device__ __forceinline__ v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 mul3s(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ v3 div3s(v3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ v3 neg3(v3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross3(v3 a, v3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float sqrt_safe(float v) { return sqrtf(fmaxf(v, 0.0f)); }
__device__ __forceinline__ float len2_3(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__device__ __forceinline__ v3 normalize3(v3 a) { return div3s(a, sqrt_safe(len2_3(a))); }

struct spec {
    float r, g, b;
};
__device__ __forceinline__ spec mksp(float r, float g, float b) { return spec{ r, g, b }; }
__device__ __forceinline__ spec sp_add(spec a, spec b) { return mksp(a.r + b.r, a.g + b.g, a.b + b.b); }
__device__ __forceinline__ spec sp_mul(spec a, spec b) { return mksp(a.r * b.r, a.g * b.g, a.b * b.b); }
__device__ __forceinline__ spec sp_muls(spec a, float s) { return mksp(a.r * s, a.g * s, a.b * s); }
__device__ __forceinline__ spec sp_divs(spec a, float s) { return mksp(a.r / s, a.g / s, a.b / s); }
__device__ __forceinline__ bool sp_valid(spec a) { return a.r > 0.0f || a.g > 0.0f || a.b > 0.0f; }
__device__ __forceinline__ spec sp_zero() { return mksp(0.0f, 0.0f, 0.0f); }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.2831853071796f;
constexpr float kHalfPi = 1.57079632679489661923f;
constexpr float kQuarterPi = 0.785398163397448309616f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kSqrPi = 9.869604401089358f;

enum : int {
    kPartR = 1, kPartT = 2, kPartDiffuse = 4, kPartSpecular = 8, kPartGlossy = 16, kPartAll = 31,
    kPartNoSpecular = 31 ^ 8
};
__device__ __forceinline__ bool part_match(int provide, int require) { return (provide & require) == provide; }

// Material after host-side set-up: constant textures resolved, roughness remapped
// (MicrofacetDistribution::remapRoughness, Classic/Kernel.cpp:378-381, evaluated once per material).
struct DevMaterial {
    uint32_t type;
    float c0[3];
    float c1[3];
    float ax, ay;   // microfacet alphas
    float on_a, on_b;  // Oren-Nayar A, B (Classic/Kernel.cpp:103-109)
    uint32_t valid0, valid1;
    float roughness0, roughness1;
    uint32_t tex[4];  // color0, color1, roughness0, roughness1: 0 constant, k > 0 samples DevTexture k - 1
};

// A texture on the device: pb2_texture with the texels moved to device memory.
struct DevTexture {
    uint32_t kind, channel, wrap, width, height;
    const uint8_t* texels;
    float scale;
    float black[4], white[4];
};

__device__ __forceinline__ void texture_sample(const DevTexture& t, float tu, float tv, float* out) {
    if (t.kind == PB2_TEXTURE_IMAGE) {
        pb2_tex_sample(t.texels, t.width, t.height, t.channel, t.wrap, tu, tv, out);
    } else {
        const float* arr = pb2_checker_white(tu, tv, t.scale) ? t.white : t.black;
        for (uint32_t i = 0; i < t.channel; ++i) out[i] = arr[i];
    }
}

// The material's textured parameters at texture coordinate (tu, tv), then what the surface init derives from them
// per point (Classic/Kernel.cpp: the remapped roughness of plastic :459-462, glass :636-639 and substrate :770-772,
// Oren-Nayar's A and B :103-109); parameters without a texture keep the values set up once on the host.
__device__ __forceinline__ void apply_textures(DevMaterial& m, const DevTexture* tex, float tu, float tv) {
    float v[4] = { 0.0f, 0.0f, 0.0f, 0.0f };
    if (m.tex[0]) {
        texture_sample(tex[m.tex[0] - 1], tu, tv, v);
        m.c0[0] = v[0]; m.c0[1] = v[1]; m.c0[2] = v[2];
        m.valid0 = v[0] > 0.0f || v[1] > 0.0f || v[2] > 0.0f;
    }
    if (m.tex[1]) {
        texture_sample(tex[m.tex[1] - 1], tu, tv, v);
        m.c1[0] = v[0]; m.c1[1] = v[1]; m.c1[2] = v[2];
        m.valid1 = v[0] > 0.0f || v[1] > 0.0f || v[2] > 0.0f;
    }
    if (m.tex[2]) {
        texture_sample(tex[m.tex[2] - 1], tu, tv, v);
        m.roughness0 = v[0];
        if (m.type == PB2_SURFACE_CONDUCTOR) {
            m.ax = m.ay = v[0];
        } else if (m.type == PB2_SURFACE_PLASTIC) {
            m.ax = m.ay = pb2_remap_roughness(v[0]);
        } else {
            m.ax = pb2_remap_roughness(v[0]);
        }
        const float sigma = v[0] * 3.14159265358979323846f;
        const float sigma2 = sigma * sigma;
        m.on_a = 1.0f - (sigma2 / (2.0f * (sigma2 + 0.33f)));
        m.on_b = 0.45f * sigma2 / (sigma2 + 0.09f);
    }
    if (m.tex[3]) {
        texture_sample(tex[m.tex[3] - 1], tu, tv, v);
        m.roughness1 = v[0];
        if (m.type != PB2_SURFACE_CONDUCTOR && m.type != PB2_SURFACE_PLASTIC) m.ay = pb2_remap_roughness(v[0]);
    }
}

// LOBE_GGX_VNDF is the conductor extension's lobe (no reference counterpart): the same GGX reflection
// value as LOBE_MF_REFL, sampled with exact visible-normal sampling (Heitz 2018, "Sampling the GGX
// Distribution of Visible Normals", JCGT 7(4)) and reporting that sampler's density,
// pdf(wi) = G1(wo) D(wh) / (4 wo.z).  (The reference's MicrofacetReflection::pdf, Classic/Kernel.cpp:405-412,
// is not the density of its sampler, which one-sample MIS with a guide cannot tolerate.)
enum LobeType : int { LOBE_LAMBERT, LOBE_OREN_NAYAR, LOBE_MF_REFL, LOBE_FRESNEL_SPEC, LOBE_MF_TRANS, LOBE_BLEND, LOBE_GGX_VNDF };
enum FresnelType : int { FRESNEL_DIELECTRIC, FRESNEL_SCHLICK };

struct Lobe {
    int type, part;
    spec color, color2;
    float a, b, ax, ay, eta_i, eta_t, eta, correct;
    int fresnel;
};

struct Bsdf {
    int n;
    Lobe l[3];
    bool no_specular;
    bool mirror;
};

struct BsdfSample {
    v3 wi;
    spec f;
    float pdf;
    int part;
};

// FresnelDielectric (Classic/Kernel.cpp:271-286)
__device__ __forceinline__ float fresnel_dielectric(float eta_i, float eta_t, float cos_i) {
    cos_i = fmaxf(0.0f, fminf(1.0f, fabsf(cos_i)));
    const float sin_i = sqrt_safe(1.0f - cos_i * cos_i);
    const float sin_t = eta_i / eta_t * sin_i;
    if (sin_t >= 1.0f) return 1.0f;
    const float cos_t = sqrt_safe(1.0f - sin_t * sin_t);
    const float p1 = eta_t * cos_i, p2 = eta_i * cos_t;
    const float par = (p1 - p2) / (p1 + p2);
    const float p3 = eta_i * cos_i, p4 = eta_t * cos_t;
    const float perp = (p3 - p4) / (p3 + p4);
    return 0.5f * (par * par + perp * perp);
}

__device__ __forceinline__ spec lobe_fresnel(const Lobe& L, float c) {
    if (L.fresnel == FRESNEL_SCHLICK) {
        const float m = 1.0f - fminf(1.0f, fabsf(c));
        const float m5 = (m * m) * (m * m) * m;
        return mksp(L.color2.r + (1.0f - L.color2.r) * m5, L.color2.g + (1.0f - L.color2.g) * m5,
                    L.color2.b + (1.0f - L.color2.b) * m5);
    }
    const float f = fresnel_dielectric(L.eta_i, L.eta_t, c);
    return mksp(f, f, f);
}

// MicrofacetDistribution (Classic/Kernel.cpp:289-382)
__device__ __forceinline__ float mf_lambda(float ax, float ay, v3 w) {
    const float cos2 = w.z * w.z;
    const float sin2 = fmaxf(0.0f, 1.0f - cos2);
    const float tan2 = sin2 / cos2;
    if (isinf(tan2)) return 0.0f;
    const float sin_t = sqrtf(sin2);
    const float cos_phi = sin_t == 0.0f ? 1.0f : fminf(1.0f, fmaxf(-1.0f, w.x / sin_t));
    const float p1 = cos_phi * ax;
    const float sin_phi = sin_t == 0.0f ? 0.0f : fminf(1.0f, fmaxf(-1.0f, w.y / sin_t));
    const float p2 = sin_phi * ay;
    const float sqr = (p1 * p1 + p2 * p2) * tan2;
    return (-1.0f + sqrtf(1.0f + sqr)) * 0.5f;
}

__device__ __forceinline__ float mf_d(float ax, float ay, v3 wh) {
    const float cos2 = wh.z * wh.z;
    const float sin2 = fmaxf(0.0f, 1.0f - cos2);
    const float tan2 = sin2 / cos2;
    if (isinf(tan2)) return 0.0f;
    const float sin_t = sqrtf(sin2);
    const float cos_phi = sin_t == 0.0f ? 1.0f : fminf(1.0f, fmaxf(-1.0f, wh.x / sin_t));
    const float p1 = cos_phi / ax;
    const float sin_phi = sin_t == 0.0f ? 0.0f : fminf(1.0f, fmaxf(-1.0f, wh.y / sin_t));
    const float p2 = sin_phi / ay;
    const float e = cos2 * (1.0f + (p1 * p1 + p2 * p2) * tan2);
    return kInvPi / (ax * ay * e * e);
}

__device__ __forceinline__ void mf_sample11(float cos_theta, float u1, float u2, float& sx, float& sy) {
    if (cos_theta > 1.0f - 1e-5f) {
        const float r = sqrtf(u1 / (1.0f - u1));
        const float phi = kTwoPi * u2;
        float s, c;
        pb2_sincosf(phi, &s, &c);
        sx = r * c;
        sy = r * s;
        return;
    }
    const float sin_t = sqrt_safe(1.0f - cos_theta * cos_theta);
    const float tan_t = sin_t / cos_theta;
    const float tan2 = tan_t * tan_t;
    const float g1 = 2.0f / (1.0f + sqrtf(1.0f + tan2));
    const float a = 2.0f * u1 / g1 - 1.0f;
    const float a2 = a * a;
    const float v = fminf(1e10f, 1.0f / (a2 - 1.0f));
    const float d = sqrt_safe(tan2 * v * v - (a2 - tan2) * v);
    const float p = tan_t * v;
    const float p1 = p - d;
    const float p2 = p + d;
    const float x = (a < 0.0f || p2 > 1.0f / tan_t) ? p1 : p2;
    const float s = u2 > 0.5f ? 1.0f : -1.0f;
    const float nu2 = (u2 > 0.5f ? 2.0f : -2.0f) * (u2 - 0.5f);
    const float z = (nu2 * (nu2 * (nu2 * 0.27385f - 0.73369f) + 0.46341f)) /
                    (nu2 * (nu2 * (nu2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
    sx = x;
    sy = s * z * sqrtf(1.0f + x * x);
}

__device__ __forceinline__ v3 mf_sample_wh(float ax, float ay, v3 wi, float u1, float u2) {
    const v3 st = normalize3(mk3(ax * wi.x, ay * wi.y, wi.z));
    float sx, sy;
    mf_sample11(st.z, u1, u2, sx, sy);
    const float sin_t = sqrt_safe(1.0f - st.z * st.z);
    const float cos_phi = sin_t == 0.0f ? 1.0f : fminf(1.0f, fmaxf(-1.0f, st.x / sin_t));
    const float sin_phi = sin_t == 0.0f ? 0.0f : fminf(1.0f, fmaxf(-1.0f, st.y / sin_t));
    const float rx = cos_phi * sx - sin_phi * sy;
    const float ry = sin_phi * sx + cos_phi * sy;
    return normalize3(mk3(-rx * ax, -ry * ay, 1.0f));
}

__device__ __forceinline__ v3 half_vector(v3 a, v3 b) { return normalize3(mk3(a.x + b.x, a.y + b.y, a.z + b.z)); }

// Heitz 2018, listing 1: a visible normal of the GGX distribution (ax, ay) seen from wo (wo.z > 0).
__device__ __forceinline__ v3 ggx_sample_vndf(float ax, float ay, v3 wo, float u1, float u2) {
    const v3 vh = normalize3(mk3(ax * wo.x, ay * wo.y, wo.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    v3 t1 = mk3(1.0f, 0.0f, 0.0f);
    if (lensq > 0.0f) {
        const float inv = 1.0f / sqrtf(lensq);
        t1 = mk3(-vh.y * inv, vh.x * inv, 0.0f);
    }
    const v3 t2 = cross3(vh, t1);
    const float r = sqrtf(u1);
    float sp, cp;
    pb2_sincosf(kTwoPi * u2, &sp, &cp);
    const float p1 = r * cp;
    const float s = 0.5f * (1.0f + vh.z);
    const float p2 = (1.0f - s) * sqrt_safe(1.0f - p1 * p1) + s * (r * sp);
    const float pz = sqrt_safe(1.0f - p1 * p1 - p2 * p2);
    const v3 nh = mk3(p1 * t1.x + p2 * t2.x + pz * vh.x, p1 * t1.y + p2 * t2.y + pz * vh.y,
                      p1 * t1.z + p2 * t2.z + pz * vh.z);
    return normalize3(mk3(ax * nh.x, ay * nh.y, fmaxf(0.0f, nh.z)));
}
__device__ __forceinline__ v3 reflect3(v3 wo, v3 n) { return sub3(mul3s(n, 2.0f * dot3(wo, n)), wo); }
__device__ __forceinline__ bool refract3(v3 wi, v3 n, float eta, v3& wt) {
    const float cos_i = dot3(n, wi);
    const float sin2_i = fmaxf(0.0f, 1.0f - cos_i * cos_i);
    const float sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return false;
    const float cos_t = sqrt_safe(1.0f - sin2_t);
    wt = normalize3(sub3(mul3s(n, eta * cos_i - cos_t), mul3s(wi, eta)));
    return true;
}

// sampleConcentricDisk + sampleCosineHemisphere (Src/Kernel/Sampling.hpp:31-50)
__device__ __forceinline__ v3 sample_cosine_hemisphere(float u1, float u2) {
    u1 = 2.0f * u1 - 1.0f;
    u2 = 2.0f * u2 - 1.0f;
    const float au1 = fabsf(u1), au2 = fabsf(u2);
    float cx, cy;
    if (fminf(au1, au2) < 1e-4f) {
        cx = 0.0f;
        cy = 0.0f;
    } else {
        const float rad = au1 > au2 ? u1 : u2;
        const float theta = au1 > au2 ? kQuarterPi * (u2 / u1) : kHalfPi - kQuarterPi * (u1 / u2);
        float s, c;
        pb2_sincosf(theta, &s, &c);
        cx = c * rad;
        cy = s * rad;
    }
    const float z = sqrt_safe(1.0f - (cx * cx + cy * cy));
    return mk3(cx, cy, z);
}

__device__ __forceinline__ spec lobe_eval(const Lobe& L, v3 wo, v3 wi) {
    switch (L.type) {
        case LOBE_LAMBERT:
            return sp_muls(L.color, kInvPi);
        case LOBE_OREN_NAYAR: {
            const float sin_i = sqrt_safe(1.0f - wi.z * wi.z);
            const float sin_o = sqrt_safe(1.0f - wo.z * wo.z);
            if (sin_i < 1e-4f || sin_o < 1e-4f) return sp_zero();
            const float cos_phi_i = sin_i == 0.0f ? 1.0f : fminf(1.0f, fmaxf(-1.0f, wi.x / sin_i));
            const float sin_phi_i = sin_i == 0.0f ? 0.0f : fminf(1.0f, fmaxf(-1.0f, wi.y / sin_i));
            const float cos_phi_o = sin_o == 0.0f ? 1.0f : fminf(1.0f, fmaxf(-1.0f, wo.x / sin_o));
            const float sin_phi_o = sin_o == 0.0f ? 0.0f : fminf(1.0f, fmaxf(-1.0f, wo.y / sin_o));
            const float max_cos = fmaxf(0.0f, cos_phi_i * cos_phi_o + sin_phi_i * sin_phi_o);
            float sin_alpha, tan_beta;
            if (fabsf(wi.z) > fabsf(wo.z)) { sin_alpha = sin_o; tan_beta = sin_i / fabsf(wi.z); }
            else { sin_alpha = sin_i; tan_beta = sin_o / fabsf(wo.z); }
            return sp_muls(L.color, kInvPi * (L.a + L.b * max_cos * sin_alpha * tan_beta));
        }
        case LOBE_MF_REFL: {
            const v3 wh = half_vector(wo, wi);
            const spec F = lobe_fresnel(L, dot3(wi, wh));
            const float q = mf_d(L.ax, L.ay, wh) /
                            (4.0f * (1.0f + mf_lambda(L.ax, L.ay, wo) + mf_lambda(L.ax, L.ay, wi)) * fabsf(wo.z * wi.z));
            return sp_mul(L.color, mksp(F.r * q, F.g * q, F.b * q));
        }
        case LOBE_GGX_VNDF: {
            if (wo.z <= 0.0f || wi.z <= 0.0f) return sp_zero();
            const v3 wh = half_vector(wo, wi);
            const spec F = lobe_fresnel(L, dot3(wi, wh));
            const float q = mf_d(L.ax, L.ay, wh) /
                            (4.0f * (1.0f + mf_lambda(L.ax, L.ay, wo) + mf_lambda(L.ax, L.ay, wi)) * (wo.z * wi.z));
            return sp_mul(L.color, mksp(F.r * q, F.g * q, F.b * q));
        }
        case LOBE_MF_TRANS: {
            if (wi.z >= 0.0f) return sp_zero();
            v3 wh = normalize3(add3(wo, mul3s(wi, L.eta)));
            if (wh.z < 0.0f) wh = neg3(wh);
            if (dot3(wo, wh) * dot3(wi, wh) > 0.0f) return sp_zero();
            const float f = fresnel_dielectric(L.eta_i, L.eta_t, dot3(wo, wh));
            const float sd = dot3(wo, wh) + L.eta * dot3(wi, wh);
            const float num = (1.0f - f) * mf_d(L.ax, L.ay, wh) * fabsf(dot3(wi, wh)) * fabsf(dot3(wo, wh)) * L.correct;
            const float den = (1.0f + mf_lambda(L.ax, L.ay, wo) + mf_lambda(L.ax, L.ay, wi)) * wo.z * wi.z * (sd * sd);
            return sp_muls(L.color, fabsf(num / den));
        }
        case LOBE_BLEND: {
            const spec nrs = sp_add(L.color2, mksp(-1.0f, -1.0f, -1.0f));
            const float pi5 = 1.0f - 0.5f * fabsf(wi.z), po5 = 1.0f - 0.5f * fabsf(wo.z);
            const float pw_i = (pi5 * pi5) * (pi5 * pi5) * pi5, pw_o = (po5 * po5) * (po5 * po5) * po5;
            const float k = -28.f / (23.f * kPi) * (1.0f - pw_i) * (1.0f - pw_o);
            const spec diffuse = sp_muls(sp_mul(L.color, nrs), k);
            const v3 wh = half_vector(wo, wi);
            const float cm1 = dot3(wi, wh) - 1.0f;
            const float p5 = (cm1 * cm1) * (cm1 * cm1) * cm1;
            const spec schlick = sp_add(L.color2, sp_muls(nrs, p5));
            const float denom = 4.0f * fmaxf(fabsf(wi.z), fabsf(wo.z)) * fabsf(dot3(wi, wh));
            const spec specular = sp_muls(schlick, mf_d(L.ax, L.ay, wh) / denom);
            return sp_add(diffuse, specular);
        }
        default:
            return sp_zero();
    }
}

__device__ __forceinline__ float lobe_pdf(const Lobe& L, v3 wo, v3 wi) {
    switch (L.type) {
        case LOBE_LAMBERT:
        case LOBE_OREN_NAYAR:
            return wi.z > 0.0f ? fabsf(wi.z) * kInvPi : 0.0f;
        case LOBE_MF_REFL: {
            if (wi.z <= 0.0f) return 0.0f;
            const v3 wh = half_vector(wo, wi);
            const float p1 = 1.0f + mf_lambda(L.ax, L.ay, wo);
            const float p2 = mf_lambda(L.ax, L.ay, wh);
            return fabsf(0.25f / (wo.z * p1 * (p1 + p2)));
        }
        case LOBE_GGX_VNDF: {
            if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
            const v3 wh = half_vector(wo, wi);
            if (dot3(wo, wh) <= 0.0f) return 0.0f;
            return mf_d(L.ax, L.ay, wh) / (4.0f * wo.z * (1.0f + mf_lambda(L.ax, L.ay, wo)));
        }
        case LOBE_MF_TRANS: {
            if (wi.z >= 0.0f) return 0.0f;
            const v3 wh = normalize3(add3(wo, mul3s(wi, L.eta)));
            if (dot3(wo, wh) * dot3(wi, wh) > 0.0f) return 0.0f;
            const float sd = dot3(wo, wh) + L.eta * dot3(wi, wh);
            const float q = L.eta / sd;
            const float delta = fabsf((q * q) * dot3(wi, wh));
            return mf_d(L.ax, L.ay, wh) * fabsf(dot3(wo, wh)) * delta / ((1.0f + mf_lambda(L.ax, L.ay, wo)) * fabsf(wo.z));
        }
        case LOBE_BLEND: {
            if (wi.z <= 0.0f) return 0.0f;
            const v3 wh = half_vector(wo, wi);
            return 0.5f * (fabsf(wi.z) * kInvPi +
                           mf_d(L.ax, L.ay, wh) /
                               (4.0f * fabsf(wo.z) * (1.0f + mf_lambda(L.ax, L.ay, wo) + mf_lambda(L.ax, L.ay, wh))));
        }
        default:
            return 0.0f;
    }
}

__device__ __forceinline__ void lobe_sample(const Lobe& L, float u1, float u2, v3 wo, BsdfSample& res) {
    switch (L.type) {
        case LOBE_LAMBERT:
        case LOBE_OREN_NAYAR:
            res.wi = sample_cosine_hemisphere(u1, u2);
            res.f = lobe_eval(L, wo, res.wi);
            res.pdf = lobe_pdf(L, wo, res.wi);
            res.part = L.part;
            return;
        case LOBE_MF_REFL: {
            if (wo.z == 0.0f) return;
            const v3 wh = mf_sample_wh(L.ax, L.ay, wo, u1, u2);
            if (dot3(wo, wh) < 0.0f) return;
            res.wi = reflect3(wo, wh);
            if (res.wi.z <= 0.0f) return;
            const float p1 = 1.0f + mf_lambda(L.ax, L.ay, wo);
            const spec F = lobe_fresnel(L, dot3(res.wi, wh));
            const float q = mf_d(L.ax, L.ay, wh) / (4.0f * (p1 + mf_lambda(L.ax, L.ay, res.wi)) * fabsf(wo.z * res.wi.z));
            res.f = sp_mul(L.color, mksp(F.r * q, F.g * q, F.b * q));
            res.part = L.part;
            const float p2 = mf_lambda(L.ax, L.ay, wh);
            res.pdf = fabsf(0.25f / (wo.z * p1 * (p1 + p2)));
            return;
        }
        case LOBE_GGX_VNDF: {
            if (wo.z <= 0.0f) return;
            const v3 wh = ggx_sample_vndf(L.ax, L.ay, wo, u1, u2);
            res.wi = reflect3(wo, wh);
            if (res.wi.z <= 0.0f) return;
            res.f = lobe_eval(L, wo, res.wi);
            res.pdf = lobe_pdf(L, wo, res.wi);
            res.part = L.part;
            return;
        }
        case LOBE_FRESNEL_SPEC: {
            const float f = fresnel_dielectric(L.eta_i, L.eta_t, wo.z);
            if (u1 < f) {
                res.wi = mk3(-wo.x, -wo.y, wo.z);
                res.part = kPartR | kPartSpecular;
                res.pdf = f;
                res.f = sp_muls(L.color, f / fabsf(res.wi.z));
            } else {
                v3 wt;
                if (!refract3(wo, mk3(0.0f, 0.0f, 1.0f), L.eta, wt)) return;
                res.wi = wt;
                res.part = kPartT | kPartSpecular;
                res.pdf = 1.0f - f;
                res.f = sp_muls(L.color2, L.correct * res.pdf / fabsf(res.wi.z));
            }
            return;
        }
        case LOBE_MF_TRANS: {
            if (wo.z == 0.0f) return;
            const v3 wh = mf_sample_wh(L.ax, L.ay, wo, u1, u2);
            if (dot3(wo, wh) < 0.0f) return;
            v3 wt;
            if (!refract3(wo, wh, L.eta, wt)) return;
            res.wi = wt;
            res.part = L.part;
            res.f = lobe_eval(L, wo, wt);
            res.pdf = lobe_pdf(L, wo, wt);
            return;
        }
        case LOBE_BLEND: {
            if (u1 < 0.5f) {
                u1 = fminf(2.0f * u1, 1.0f);
                res.wi = sample_cosine_hemisphere(u1, u2);
            } else {
                u1 = fminf(2.0f * (u1 - 0.5f), 1.0f);
                const v3 wh = mf_sample_wh(L.ax, L.ay, wo, u1, u2);
                res.wi = reflect3(wo, wh);
                if (res.wi.z <= 0.0f) return;
            }
            res.part = L.part;
            res.pdf = lobe_pdf(L, wo, res.wi);
            res.f = lobe_eval(L, wo, res.wi);
            return;
        }
        default:
            return;
    }
}

// Surface init of the Classic module (Classic/Kernel.cpp: matte :249-268, plastic :441-470,
// glass :613-656, mirror :668-677, substrate :755-778, black body :45-48).
// kType >= 0 is the material's surface type known at compile time (the per-type shading kernels): the
// lobe count then folds to a constant and the lobes stay in registers.
template <int kType = -1>
__device__ __forceinline__ void bsdf_init(const DevMaterial& m, bool front, Bsdf& b) {
    b.n = 0;
    b.mirror = false;
    b.no_specular = false;
    const spec c0 = mksp(m.c0[0], m.c0[1], m.c0[2]);
    const spec c1 = mksp(m.c1[0], m.c1[1], m.c1[2]);
    switch (kType >= 0 ? (uint32_t)kType : m.type) {
        case PB2_SURFACE_MATTE: {
            Lobe& L = b.l[b.n++];
            L.part = kPartDiffuse | kPartR;
            L.color = c0;
            L.type = m.roughness0 > 0.0f ? LOBE_OREN_NAYAR : LOBE_LAMBERT;
            L.a = m.on_a;
            L.b = m.on_b;
            b.no_specular = true;
            break;
        }
        case PB2_SURFACE_PLASTIC: {
            if (m.valid0) {
                Lobe& L = b.l[b.n++];
                L.type = LOBE_LAMBERT; L.part = kPartDiffuse | kPartR; L.color = c0;
            }
            if (m.valid1) {
                Lobe& L = b.l[b.n++];
                L.type = LOBE_MF_REFL; L.part = kPartGlossy | kPartR; L.color = c1;
                L.fresnel = FRESNEL_DIELECTRIC;
                L.eta_i = front ? 1.0f : 1.46f;
                L.eta_t = front ? 1.46f : 1.0f;
                L.ax = m.ax; L.ay = m.ax;
            }
            b.no_specular = true;
            break;
        }
        case PB2_SURFACE_CONDUCTOR: {
            Lobe& L = b.l[b.n++];
            L.type = LOBE_GGX_VNDF; L.part = kPartGlossy | kPartR;
            L.color = mksp(1.0f, 1.0f, 1.0f);
            L.color2 = c1;
            L.fresnel = FRESNEL_SCHLICK;
            L.ax = m.ax; L.ay = m.ay;
            b.no_specular = true;
            break;
        }
        case PB2_SURFACE_GLASS: {
            if (!m.valid0 && !m.valid1) break;
            const float eta_i = front ? 1.0f : 1.5f, eta_t = front ? 1.5f : 1.0f;
            if (m.roughness0 == 0.0f && m.roughness1 == 0.0f) {
                Lobe& L = b.l[b.n++];
                L.type = LOBE_FRESNEL_SPEC; L.part = kPartR | kPartT | kPartSpecular;
                L.color = c0; L.color2 = c1;
                L.eta_i = eta_i; L.eta_t = eta_t;
                L.eta = eta_i / eta_t;
                L.correct = L.eta * L.eta;
            } else {
                if (m.valid0) {
                    Lobe& L = b.l[b.n++];
                    L.type = LOBE_MF_REFL; L.part = kPartGlossy | kPartR; L.color = c0;
                    L.fresnel = FRESNEL_DIELECTRIC; L.eta_i = eta_i; L.eta_t = eta_t; L.ax = m.ax; L.ay = m.ay;
                }
                if (m.valid1) {
                    Lobe& L = b.l[b.n++];
                    L.type = LOBE_MF_TRANS; L.part = kPartGlossy | kPartT; L.color = c1;
                    L.eta_i = eta_i; L.eta_t = eta_t; L.ax = m.ax; L.ay = m.ay;
                    L.eta = eta_t / eta_i;
                    L.correct = 1.0f;
                }
                b.no_specular = true;
            }
            break;
        }
        case PB2_SURFACE_MIRROR: {
            Lobe& L = b.l[b.n++];
            L.type = LOBE_FRESNEL_SPEC; L.part = kPartR | kPartSpecular; L.color = c0;
            b.mirror = true;
            break;
        }
        case PB2_SURFACE_SUBSTRATE: {
            if (!m.valid0 && !m.valid1) break;
            Lobe& L = b.l[b.n++];
            L.type = LOBE_BLEND; L.part = kPartGlossy | kPartR; L.color = c0; L.color2 = c1;
            L.ax = m.ax; L.ay = m.ay;
            b.no_specular = true;
            break;
        }
        default:
            break;
    }
}

__device__ __forceinline__ uint32_t bsdf_count(const Bsdf& b, int require) {
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (i < b.n) c += part_match(b.l[i].part, require) ? 1u : 0u;
    return c;
}

// sample() of KERNEL_FUNCTION_GROUP (Classic/Kernel.cpp:186-206), mirrorSample (:680-692)
__device__ __forceinline__ void bsdf_sample(const Bsdf& b, float u1, float u2, v3 wo, v3 ng, int require,
                                            BsdfSample& out) {
    out.pdf = 0.0f;
    if (b.mirror) {
        const int part = kPartR | kPartSpecular;
        if (part_match(part, require)) {
            out.wi = mk3(-wo.x, -wo.y, wo.z);
            out.f = sp_divs(b.l[0].color, fabsf(out.wi.z));
            out.part = part;
            out.pdf = 1.0f;
        }
        return;
    }
    const uint32_t count = bsdf_count(b, require);
    if (count == 0) return;
    uint32_t sel = (uint32_t)floorf(u1 * (float)count);
    if (sel > count - 1) sel = count - 1;
    u1 = u1 * (float)count - (float)sel;
    int chosen = -1;
#pragma unroll
    for (int i = 0, k = 0; i < 3; ++i) {
        if (i >= b.n || chosen >= 0 || !part_match(b.l[i].part, require)) continue;
        if ((uint32_t)k == sel) chosen = i;
        ++k;
    }
    // the chosen lobe by register selects (a dynamic index would put the lobes in local memory)
    lobe_sample(chosen == 0 ? b.l[0] : (chosen == 1 ? b.l[1] : b.l[2]), u1, u2, wo, out);
    if (out.pdf <= 0.0f) return;
    if (!(out.part & kPartSpecular)) {
        const int addition = (dot3(wo, ng) * dot3(out.wi, ng)) > 0.0f ? kPartR : kPartT;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (i >= b.n || i == chosen || !part_match(b.l[i].part, require)) continue;
            if (addition & b.l[i].part) out.f = sp_add(out.f, lobe_eval(b.l[i], wo, out.wi));
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (i >= b.n || i == chosen || !part_match(b.l[i].part, require)) continue;
            out.pdf = out.pdf + lobe_pdf(b.l[i], wo, out.wi);
        }
    }
    if (count > 1) out.pdf = out.pdf / (float)count;
}

__device__ __forceinline__ spec bsdf_eval(const Bsdf& b, v3 wo, v3 wi, v3 ng, int require) {
    if (b.mirror) return sp_zero();
    const int addition = (dot3(wo, ng) * dot3(wi, ng)) > 0.0f ? kPartR : kPartT;
    spec f = sp_zero();
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (i < b.n && part_match(b.l[i].part, require) && (addition & b.l[i].part))
            f = sp_add(f, lobe_eval(b.l[i], wo, wi));
    return f;
}

__device__ __forceinline__ float bsdf_pdf(const Bsdf& b, v3 wo, v3 wi, int require) {
    if (b.mirror) return 0.0f;
    const uint32_t count = bsdf_count(b, require);
    if (count == 0) return 0.0f;
    float pdf = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (i < b.n && part_match(b.l[i].part, require)) pdf = pdf + lobe_pdf(b.l[i], wo, wi);
    if (count > 1) pdf = pdf / (float)count;
    return pdf;
}

__device__ __forceinline__ float power_heuristic(float a, float b) {
    const float sp1 = a * a;
    const float sp2 = b * b;
    return sp1 / (sp1 + sp2);
}

}  // namespace pb2
