/*
 * pb2_math.h -- elementary functions with one definition on the host and on sm_100a.
 *
 * The render path calls cos/sin (camera lens disk, cosine hemisphere, GGX slope sampling, environment
 * sampling), acos (environment pdf) and exp (Gaussian film filter).  The reference calls the C library
 * (Src/Kernel/PhysicalQuantitySI.hpp:162-175, Src/Kernel/Sampling.hpp:24-43,
 * Src/BuiltinComponent/RenderDriver/FixedSampler/Kernel.cpp:65-69).  CUDA's and glibc's versions of
 * those functions can differ in the last bit, which would let a single path diverge between the GPU
 * and the CPU oracle.  These functions are written once here, from textbook methods, using only IEEE
 * add/mul/div/sqrt and explicitly fused multiply-adds, so a host build with -ffp-contract=off and a
 * device build give bit-identical results:
 *
 *   sin/cos : Cody-Waite reduction by pi/2 (three-part constant, fused), then the Taylor series of sin
 *             (to x^9) and cos (to x^10) on |r| <= pi/4 -- truncation error < 3e-9 relative.
 *   exp     : reduction by ln 2 (two-part constant), Taylor series to r^7 on |r| <= ln2/2, then an
 *             exact power-of-two scale.
 *   acos    : the binomial (arcsine) series on |x| <= 1/2, and acos(x) = 2 asin(sqrt((1-x)/2)) above.
 *
 * Accuracy is checked against the C library in the CPU tests (within 4 ulp).  The device runs these same
 * definitions, so the GPU parity tests, which compare whole paths bit for bit with the CPU oracle, cover
 * their device builds.
 */
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define PB2_HD static __host__ __device__ __forceinline__
#else
#define PB2_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define PB2_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#define PB2_RINT(x) rintf(x)
#else
#define PB2_FMA(a, b, c) fmaf((a), (b), (c))
#define PB2_RINT(x) rintf(x)
#endif

/* pi/2 split into three floats: hi = nearest float, mid/lo = successive remainders. */
#define PB2_PIO2_HI 1.57079637050628662109375f
#define PB2_PIO2_MID (-4.37113882867379289e-08f)
#define PB2_PIO2_LO (-1.71512451000588187e-15f)
#define PB2_TWO_OVER_PI 0.636619772367581343076f

PB2_HD float pb2_ldexp_int(float x, int k) {
    /* x * 2^k for k in [-252, 254] using exact power-of-two factors. */
    while (k > 127) { x = x * 1.7014118346046923e38f; k -= 127; }
    while (k < -126) { x = x * 1.1754943508222875e-38f; k += 126; }
    union { uint32_t u; float f; } s;
    s.u = (uint32_t)(k + 127) << 23;
    return x * s.f;
}

PB2_HD void pb2_sincosf(float x, float* s_out, float* c_out) {
    const float q = PB2_RINT(x * PB2_TWO_OVER_PI);
    float r = PB2_FMA(-q, PB2_PIO2_HI, x);
    r = PB2_FMA(-q, PB2_PIO2_MID, r);
    r = PB2_FMA(-q, PB2_PIO2_LO, r);
    const float r2 = r * r;
    /* sin(r) = r + r^3 (-1/6 + r^2 (1/120 + r^2 (-1/5040 + r^2 / 362880))) */
    float ps = PB2_FMA(r2, 2.75573192239858906526e-6f, -1.98412698412698412698e-4f);
    ps = PB2_FMA(r2, ps, 8.33333333333333333333e-3f);
    ps = PB2_FMA(r2, ps, -1.66666666666666666667e-1f);
    const float s = PB2_FMA(r * r2, ps, r);
    /* cos(r) = 1 + r^2 (-1/2 + r^2 (1/24 + r^2 (-1/720 + r^2 (1/40320 - r^2/3628800)))) */
    float pc = PB2_FMA(r2, -2.75573192239858906526e-7f, 2.48015873015873015873e-5f);
    pc = PB2_FMA(r2, pc, -1.38888888888888888889e-3f);
    pc = PB2_FMA(r2, pc, 4.16666666666666666667e-2f);
    pc = PB2_FMA(r2, pc, -0.5f);
    const float c = PB2_FMA(r2, pc, 1.0f);
    const int quadrant = ((int)q) & 3;
    float so, co;
    switch (quadrant) {
        case 0: so = s; co = c; break;
        case 1: so = c; co = -s; break;
        case 2: so = -s; co = -c; break;
        default: so = -c; co = s; break;
    }
    *s_out = so;
    *c_out = co;
}

PB2_HD float pb2_sinf(float x) {
    float s, c;
    pb2_sincosf(x, &s, &c);
    return s;
}

PB2_HD float pb2_cosf(float x) {
    float s, c;
    pb2_sincosf(x, &s, &c);
    return c;
}

#define PB2_LN2_HI 0.693145751953125f
#define PB2_LN2_LO 1.42860676533018705e-06f
#define PB2_LOG2E 1.44269504088896340736f

PB2_HD float pb2_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283935546875f) return INFINITY;
    if (x < -103.97208404541015625f) return 0.0f;
    const float k = PB2_RINT(x * PB2_LOG2E);
    float r = PB2_FMA(-k, PB2_LN2_HI, x);
    r = PB2_FMA(-k, PB2_LN2_LO, r);
    /* e^r = sum r^n / n!, n <= 7 */
    float p = PB2_FMA(r, 1.98412698412698412698e-4f, 1.38888888888888888889e-3f);
    p = PB2_FMA(r, p, 8.33333333333333333333e-3f);
    p = PB2_FMA(r, p, 4.16666666666666666667e-2f);
    p = PB2_FMA(r, p, 1.66666666666666666667e-1f);
    p = PB2_FMA(r, p, 0.5f);
    p = PB2_FMA(r, p, 1.0f);
    p = PB2_FMA(r, p, 1.0f);
    return pb2_ldexp_int(p, (int)k);
}

/* asin on |x| <= 1/2 by the binomial series x + sum_{n=1..11} c_n x^(2n+1),
 * c_n = (2n)! / (4^n (n!)^2 (2n+1)); the first omitted term is below 4e-10 relative. */
PB2_HD float pb2_asin_small(float x) {
    const float z = x * x;
    float p = 7.31252587359884544810e-03f;     /* c_11 = 88179/12058624 */
    p = PB2_FMA(z, p, 8.39033580961681506316e-03f); /* c_10 = 46189/5505024 */
    p = PB2_FMA(z, p, 9.76160952919407839956e-03f); /* c_9  = 12155/1245184 */
    p = PB2_FMA(z, p, 1.15518008961397050660e-02f); /* c_8  = 6435/557056 */
    p = PB2_FMA(z, p, 1.39648437500000006939e-02f); /* c_7  = 143/10240 */
    p = PB2_FMA(z, p, 1.73527644230769238776e-02f); /* c_6  = 231/13312 */
    p = PB2_FMA(z, p, 2.23721590909090918553e-02f); /* c_5  = 63/2816 */
    p = PB2_FMA(z, p, 3.03819444444444440590e-02f); /* c_4  = 35/1152 */
    p = PB2_FMA(z, p, 4.46428571428571438484e-02f); /* c_3  = 5/112 */
    p = PB2_FMA(z, p, 7.49999999999999972244e-02f); /* c_2  = 3/40 */
    p = PB2_FMA(z, p, 1.66666666666666657415e-01f); /* c_1  = 1/6 */
    return PB2_FMA(x * z, p, x);
}

PB2_HD float pb2_acosf(float x) {
    const float pio2 = 1.57079632679489661923f;
    const float pi = 3.14159265358979323846f;
    const float a = fabsf(x);
    float r;
    if (a <= 0.5f) {
        r = pio2 - pb2_asin_small(x);
    } else {
        const float h = sqrtf((1.0f - a) * 0.5f);
        const float t = 2.0f * pb2_asin_small(h);
        r = x > 0.0f ? t : pi - t;
    }
    return r;
}

/* ---- Owen scrambling of Sobol values (an extension: the reference's "Scramble" is notImplemented,
 * ScrambledSobolSampler.cpp:51-53) -----------------------------------------------------------------
 * Nested uniform scrambling by hashing (Burley, "Practical Hash-based Owen Scrambling", JCGT 9(4), 2020):
 * reverse the bits, apply the Laine-Karras style permutation (an added seed, then x ^= x * c with even
 * constants -- each output bit depends only on the same and lower bits of the reversed value), reverse
 * back.  Every elementary interval of the input maps to one of the output, so a Sobol dimension stays
 * stratified.  The per-dimension seed is the MurmurHash3 finaliser of (seed, dimension). */
PB2_HD uint32_t pb2_reverse_bits(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
#endif
}

PB2_HD uint32_t pb2_owen_dim_seed(uint32_t seed, uint32_t dim) {
    uint32_t h = seed ^ (dim * 0x9E3779B9u + 0x632BE5ABu);
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

PB2_HD uint32_t pb2_owen_scramble(uint32_t v, uint32_t seed) {
    uint32_t x = pb2_reverse_bits(v);
    x += seed;
    x ^= x * 0x6C50B47Cu;
    x ^= x * 0xB82F1E52u;
    x ^= x * 0xC7AFE638u;
    x ^= x * 0x8D22F6E6u;
    return pb2_reverse_bits(x);
}


/* ---- instance transforms -------------------------------------------------------------------------------
 * An instance's local-to-world transform in the reference's TransformSRT layout (Src/Kernel/Transform.hpp:390-393):
 * 16 floats -- scale x y z, skew xy xz yz, shift x y z, quaternion w x y z, translation x y z.  The reference hands
 * it to Embree 3 unchanged as an RTCQuaternionDecomposition (Src/BuiltinComponent/Tracer/Embree/Embree.cpp:699-703),
 * whose published meaning is local-to-world = T * R * S with
 *     S = [ sx kxy kxz hx ]      R = rotation of the unit quaternion (w, x, y, z)     T = translation
 *         [  0  sy kyz hy ]
 *         [  0   0  sz hz ]
 * pb2_srt_matrix_hd writes the row-major 3x4 matrix [L | t], L = R * S(3x3), t = R * h + translation, normalising the
 * quaternion first (the caller rejects a zero quaternion).  Points map as ((m0 x + m1 y) + m2 z) + m3 per row, every
 * operation a single IEEE operation, so the host flattening and a device evaluation agree bit for bit. */
PB2_HD void pb2_srt_matrix_hd(const float* srt, float* m) {
    const float sx = srt[0], sy = srt[1], sz = srt[2], kxy = srt[3], kxz = srt[4], kyz = srt[5];
    const float hx = srt[6], hy = srt[7], hz = srt[8];
    const float n2 = ((srt[9] * srt[9] + srt[10] * srt[10]) + srt[11] * srt[11]) + srt[12] * srt[12];
    const float inv = 1.0f / sqrtf(n2);
    const float w = srt[9] * inv, x = srt[10] * inv, y = srt[11] * inv, z = srt[12] * inv;
    float r[9];
    r[0] = 1.0f - 2.0f * (y * y + z * z);
    r[1] = 2.0f * (x * y - w * z);
    r[2] = 2.0f * (x * z + w * y);
    r[3] = 2.0f * (x * y + w * z);
    r[4] = 1.0f - 2.0f * (x * x + z * z);
    r[5] = 2.0f * (y * z - w * x);
    r[6] = 2.0f * (x * z - w * y);
    r[7] = 2.0f * (y * z + w * x);
    r[8] = 1.0f - 2.0f * (x * x + y * y);
    for (int i = 0; i < 3; ++i) {
        const float a = r[3 * i], b = r[3 * i + 1], c = r[3 * i + 2];
        m[4 * i + 0] = a * sx;
        m[4 * i + 1] = a * kxy + b * sy;
        m[4 * i + 2] = (a * kxz + b * kyz) + c * sz;
        m[4 * i + 3] = ((a * hx + b * hy) + c * hz) + srt[13 + i];
    }
}

PB2_HD void pb2_xform_point(const float* m, const float* p, float* out) {
    for (int i = 0; i < 3; ++i) out[i] = ((m[4 * i] * p[0] + m[4 * i + 1] * p[1]) + m[4 * i + 2] * p[2]) + m[4 * i + 3];
}

PB2_HD void pb2_xform_vector(const float* m, const float* v, float* out) {
    for (int i = 0; i < 3; ++i) out[i] = (m[4 * i] * v[0] + m[4 * i + 1] * v[1]) + m[4 * i + 2] * v[2];
}

/* A mesh vertex in world space: the instance matrix (if any), then the node translation. */
PB2_HD void pb2_mesh_vertex(const float* matrix, const float* translation, const float* p, float* out) {
    if (matrix) {
        float q[3];
        pb2_xform_point(matrix, p, q);
        for (int i = 0; i < 3; ++i) out[i] = q[i] + translation[i];
    } else {
        for (int i = 0; i < 3; ++i) out[i] = p[i] + translation[i];
    }
}

/* ---- natural logarithm ------------------------------------------------------------------------------------
 * For finite x > 0: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log(m) = 2 atanh(s), s = (m - 1) / (m + 1)
 * (|s| <= 0.1716), atanh(s) = s + s^3/3 + s^5/5 + ... to s^15 (truncation < 1e-13 relative), then
 * e ln2 with ln2 in two parts (the constants of pb2_expf).  Used where a logarithm is evaluated per shading point (the roughness remap of a
 * textured material) so that the device and the oracle agree bit for bit. */
PB2_HD float pb2_logf(float x) {
    union { float f; uint32_t u; } b;
    b.f = x;
    int e = 0;
    if (b.u < 0x00800000u) { /* subnormal (x > 0 assumed): scale into the normal range */
        b.f = x * 8388608.0f;
        e = -23;
    }
    e += (int)(b.u >> 23) - 127;
    b.u = (b.u & 0x007FFFFFu) | 0x3F800000u; /* m in [1, 2) */
    float m = b.f;
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = 0.0666666667f;               /* 1/15 */
    p = PB2_FMA(p, s2, 0.0769230769f);     /* 1/13 */
    p = PB2_FMA(p, s2, 0.0909090909f);     /* 1/11 */
    p = PB2_FMA(p, s2, 0.111111111f);      /* 1/9 */
    p = PB2_FMA(p, s2, 0.142857143f);      /* 1/7 */
    p = PB2_FMA(p, s2, 0.2f);              /* 1/5 */
    p = PB2_FMA(p, s2, 0.333333333f);      /* 1/3 */
    const float lm = 2.0f * PB2_FMA(s * s2, p, s);
    const float fe = (float)e;
    return PB2_FMA(fe, PB2_LN2_HI, PB2_FMA(fe, PB2_LN2_LO, lm));
}

/* MicrofacetDistribution::remapRoughness (Src/BuiltinComponent/Surface/Classic/Kernel.cpp:378-381) with pb2_logf:
 * the per-point form for textured roughness (a constant roughness is remapped once on the host with the C
 * library's log, as the reference does). */
PB2_HD float pb2_remap_roughness(float roughness) {
    const float x = pb2_logf(fmaxf(1e-3f, roughness));
    return fmaxf(1e-3f, 1.62142f + (0.819955f + (0.1734f + (0.0171201f + 0.000640711f * x) * x) * x) * x);
}

/* ---- textures ---------------------------------------------------------------------------------------------
 * CheckBoard (Src/BuiltinComponent/Texture/ProceduralTexture/Kernel.cpp:27-38) and the bilinear SampledTexture
 * (Texture/SampledTexture/Kernel.cpp:22-83), including its wrap arithmetic: IEEE remainder, "Mirror" folding into
 * [0, size/2] (fabs of the remainder), the last texel repeated at the edge of a mirrored axis, 8-bit texels scaled
 * by 0.003921568f.  remainderf is exact on both sides. */
PB2_HD float pb2_checker_mod(float x, float scale) {
    const float r = remainderf(x * scale, 2.0f);
    return r < 0.0f ? r + 2.0f : r;
}

PB2_HD int pb2_checker_white(float u, float v, float scale) {
    return (pb2_checker_mod(u, scale) > 1.0f) == (pb2_checker_mod(v, scale) > 1.0f);
}

PB2_HD uint32_t pb2_tex_locate(float p, uint32_t size, uint32_t mirror) {
    const float mod = (float)size;
    float s = remainderf(p, mod);
    if (mirror) s = fabsf(s);
    else if (s < 0.0f) s = s + mod;
    if (!(s >= 0.0f)) s = 0.0f; /* a NaN coordinate */
    const uint32_t i = s < 4294967040.0f ? (uint32_t)s : 0xFFFFFFFFu;
    return i < size - 1u ? i : size - 1u;
}

PB2_HD uint32_t pb2_tex_next(uint32_t p, uint32_t size, uint32_t mirror) {
    const uint32_t s = p + 1u;
    return s == size ? (mirror ? p : 0u) : s;
}

PB2_HD float pb2_tex_left_weight(float u) { return (0.5f + floorf(u + 0.5f)) - u; }

/* Bilinear lookup of `channel` 8-bit channels at texture coordinate (tu, tv); out[0..channel). */
PB2_HD void pb2_tex_sample(const uint8_t* texels, uint32_t width, uint32_t height, uint32_t channel, uint32_t mirror,
                           float tu, float tv, float* out) {
    const uint32_t stride = width * channel;
    const float u = tu * (float)width, v = tv * (float)height;
    const uint32_t plu = pb2_tex_locate(u - 0.5f, width, mirror), pru = pb2_tex_next(plu, width, mirror);
    const uint32_t plv = pb2_tex_locate(v - 0.5f, height, mirror), prv = pb2_tex_next(plv, height, mirror);
    const float lwx = pb2_tex_left_weight(u), lwy = pb2_tex_left_weight(v);
    const float rwx = 1.0f - lwx, rwy = 1.0f - lwy;
    const uint32_t cu[4] = { plu, pru, plu, pru }, cv[4] = { plv, plv, prv, prv };
    const float w[4] = { lwx * lwy, rwx * lwy, lwx * rwy, rwx * rwy };
    for (uint32_t i = 0; i < channel; ++i) out[i] = 0.0f;
    for (int c = 0; c < 4; ++c) {
        const uint32_t idx = cv[c] * stride + cu[c] * channel;
        for (uint32_t i = 0; i < channel; ++i) out[i] = out[i] + w[c] * (float)texels[idx + i];
    }
    for (uint32_t i = 0; i < channel; ++i) out[i] = out[i] * 0.003921568f;
}
