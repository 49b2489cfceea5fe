/*
 * pb2_oracle.c -- CPU oracle for the Piper2 render path.  TEST INFRASTRUCTURE ONLY (see pb2_oracle.h).
 *
 * Build: gcc -std=c11 -O2 -ffp-contract=off -fopenmp -fPIC -shared (no -march=native, no -ffast-math),
 * so that every float operation is a single IEEE operation in the order written here, which is the
 * order of the reference's expressions.  File:line citations are relative to the reference's tree.
 */
#include "pb2_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../piper2_b200/csrc/pb2_math.h"
#include "sobol_tables.h"

/* ------------------------------------------------------------------------------------------------
 * Arithmetic type.  The oracle proper is single precision (real = float): every operation is the
 * reference's float operation.  Built with -DOR_FP64 the same source is the double-precision
 * restatement used as ground truth for error measurements (liboracle_fp64.so): the same estimator,
 * sample points and constants, with every intermediate in double and libm's elementary functions.
 * ---------------------------------------------------------------------------------------------- */
#ifdef OR_FP64
typedef double real;
#define R_SQRT sqrt
#define R_FABS fabs
#define R_FMAX fmax
#define R_FMIN fmin
#define R_FLOOR floor
#define R_CEIL ceil
#define R_LOG log
#define R_EXP exp
#define R_COPYSIGN copysign
#define R_PEXP exp
#define R_SIN sin
#define R_ACOS acos
static inline void R_SINCOS(double x, double* s, double* c) { *s = sin(x); *c = cos(x); }
#define R_MAX_VALUE DBL_MAX
#else
typedef float real;
#define R_SQRT sqrtf
#define R_FABS fabsf
#define R_FMAX fmaxf
#define R_FMIN fminf
#define R_FLOOR floorf
#define R_CEIL ceilf
#define R_LOG logf
#define R_EXP expf
#define R_COPYSIGN copysignf
#define R_PEXP pb2_expf
#define R_SIN pb2_sinf
#define R_ACOS pb2_acosf
#define R_SINCOS pb2_sincosf
#define R_MAX_VALUE FLT_MAX
#endif

/* ------------------------------------------------------------------------------------------------
 * Small vector helpers.  Each returns exactly the reference's operation order.
 * ---------------------------------------------------------------------------------------------- */
typedef struct v3 { real x, y, z; } v3;
static inline v3 mk3(real x, real y, real z) { v3 r = { x, y, z }; return r; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul3s(v3 a, real s) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline v3 div3s(v3 a, real s) { return mk3(a.x / s, a.y / s, a.z / s); }
static inline v3 neg3(v3 a) { return mk3(-a.x, -a.y, -a.z); }
/* dot of Vector/Normal: a.x*b.x + a.y*b.y + a.z*b.z (Src/Kernel/Transform.hpp:269-277) */
static inline real dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* cross (Transform.hpp:193-196, 262-267) */
static inline v3 cross3(v3 a, v3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* sqrtSafe (Src/Kernel/PhysicalQuantitySI.hpp:107-110) */
static inline real sqrt_safe(real v) { return R_SQRT(R_FMAX(v, 0.0f)); }
/* lengthSquared / length (Transform.hpp:178-186) */
static inline real len2_3(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
/* Normal(Vector) normalises: v / length(v) (Transform.hpp:244-248) */
static inline v3 normalize3(v3 a) { return div3s(a, sqrt_safe(len2_3(a))); }
static inline v3 ld3(const float* p) { return mk3(p[0], p[1], p[2]); }

typedef struct spec { real r, g, b; } spec;
static inline spec mksp(real r, real g, real b) { spec s = { r, g, b }; return s; }
static inline spec sp_add(spec a, spec b) { return mksp(a.r + b.r, a.g + b.g, a.b + b.b); }
static inline spec sp_mul(spec a, spec b) { return mksp(a.r * b.r, a.g * b.g, a.b * b.b); }
static inline spec sp_muls(spec a, real s) { return mksp(a.r * s, a.g * s, a.b * s); }
static inline spec sp_divs(spec a, real s) { return mksp(a.r / s, a.g / s, a.b / s); }
/* Spectrum::valid (Src/Kernel/Protocol.hpp:84-86) */
static inline int sp_valid(spec a) { return a.r > 0.0f || a.g > 0.0f || a.b > 0.0f; }
static const spec SP_ZERO = { 0.0f, 0.0f, 0.0f };

/* Constants (PhysicalQuantitySI.hpp:235-257), as real. */
#define K_PI 3.14159265358979323846f
#define K_TWO_PI 6.2831853071796f
#define K_HALF_PI 1.57079632679489661923f
#define K_QUARTER_PI 0.785398163397448309616f
#define K_INV_PI 0.318309886183790671538f
#define K_SQR_PI 9.869604401089358f

/* ------------------------------------------------------------------------------------------------
 * Sobol sampler (Src/BuiltinComponent/Sampler/ScrambledSobolSampler/Kernel.cpp)
 * ---------------------------------------------------------------------------------------------- */
/* sobolSampleImpl (:23-29), scramble = 0 */
float or_sobol_sample(uint64_t index, uint32_t dim) {
    uint32_t v = 0;
    for (uint32_t i = dim * PB2_SOBOL_MATRIX_SIZE; index; index >>= 1, i++)
        if (index & 1) v ^= pb2_sobol_matrices32[i];
    return (float)v * 0x1p-32f;
}

/* sobolIntervalToIndex (:31-50) */
uint64_t or_sobol_interval_to_index(uint32_t m, uint32_t sample, uint32_t px, uint32_t py) {
    if (m == 0) return 0;
    const uint32_t m2 = m << 1;
    uint64_t index = (uint64_t)sample << m2;
    uint64_t delta = 0;
    for (int c = 0; sample; sample >>= 1, ++c)
        if (sample & 1) delta ^= pb2_vdc_sobol_matrices[m - 1][c];
    uint64_t b = (((uint64_t)px << m) | py) ^ delta;
    for (int c = 0; b; b >>= 1, ++c)
        if (b & 1) index ^= pb2_vdc_sobol_matrices_inv[m - 1][c];
    return index;
}

/* sobolStart (:52-62) */
void or_sobol_start(uint32_t resolution, uint32_t log2_resolution, uint32_t px, uint32_t py, uint32_t sample,
                    uint64_t* index, float offset[2]) {
    const uint64_t idx = or_sobol_interval_to_index(log2_resolution, sample, px, py);
    *index = idx;
    offset[0] = fminf(fmaxf(or_sobol_sample(idx, 0) * (float)resolution - (float)px, 0.0f), 1.0f);
    offset[1] = fminf(fmaxf(or_sobol_sample(idx, 1) * (float)resolution - (float)py, 0.0f), 1.0f);
}

const char* or_sobol_digest(void) { return PB2_SOBOL_TABLE_SHA256; }

/* ------------------------------------------------------------------------------------------------
 * Host-side component setup
 * ---------------------------------------------------------------------------------------------- */
/* MicrofacetDistribution::remapRoughness (Src/BuiltinComponent/Surface/Classic/Kernel.cpp:378-381).
 * Roughness comes from constant textures, so the remap is done once per material on the host. */
static real remap_roughness(real roughness) {
    const real x = R_LOG(R_FMAX(1e-3f, roughness));
    return R_FMAX(1e-3f, 1.62142f + (0.819955f + (0.1734f + (0.0171201f + 0.000640711f * x) * x) * x) * x);
}
float or_remap_roughness(float roughness) { return (float)remap_roughness(roughness); }
float or_logf(float x) { return pb2_logf(x); }
float or_remap_roughness_point(float roughness) { return pb2_remap_roughness(roughness); }

/* Plane construction (Src/BuiltinComponent/Geometry/BasicShapes/BasicShapes.cpp:70-89) */
void or_plane_make(const float origin[3], const float u[3], const float v[3], pb2_plane* out) {
    const v3 uu = ld3(u), vv = ld3(v);
    const v3 det3 = cross3(uu, vv);
    const real area = sqrt_safe(len2_3(det3));
    const v3 n = div3s(det3, area);
    const v3 t = normalize3(uu);
    const real a0 = R_FABS(det3.x), a1 = R_FABS(det3.y), a2 = R_FABS(det3.z);
    uint32_t sel;
    if (a0 >= a1 && a0 >= a2) sel = 0;
    else sel = (a1 >= a0 && a1 >= a2) ? 1 : 2;
    memcpy(out->origin, origin, sizeof(float) * 3);
    memcpy(out->u, u, sizeof(float) * 3);
    memcpy(out->v, v, sizeof(float) * 3);
    out->normal[0] = n.x; out->normal[1] = n.y; out->normal[2] = n.z;
    out->tangent[0] = t.x; out->tangent[1] = t.y; out->tangent[2] = t.z;
    out->max_det_comp = sel;
}

/* calcRenderRECT (Src/Interface/BuiltinComponent/Sensor.hpp:38-75) */
void or_calc_render_rect(uint32_t width, uint32_t height, float device_aspect, uint32_t fit_mode,
                         pb2_ndc_transform* tr, pb2_rect* rect) {
    const float iar = (float)width / (float)height;
    const float iiar = 1.0f / iar;
    const float idar = 1.0f / device_aspect;
    if (fit_mode == PB2_FIT_FILL) {
        rect->left = 0; rect->top = 0; rect->width = width; rect->height = height;
        if (iar > device_aspect) {
            tr->ox = 0.0f; tr->oy = (idar - iiar) * 0.5f * device_aspect; tr->sx = 1.0f; tr->sy = iiar * device_aspect;
        } else {
            tr->ox = (device_aspect - iar) * 0.5f * idar; tr->oy = 0.0f; tr->sx = iar * idar; tr->sy = 1.0f;
        }
    } else {
        if (iar > device_aspect) {
            tr->ox = -(iar - device_aspect) * 0.5f * idar; tr->oy = 0.0f; tr->sx = iar * idar; tr->sy = 1.0f;
            rect->left = (uint32_t)floorf(fmaxf(0.0f, (float)width * (iar - device_aspect) * 0.5f * iiar));
            rect->top = 0;
            uint32_t r = (uint32_t)ceilf((float)width * (iar + device_aspect) * 0.5f * iiar);
            rect->width = (width < r ? width : r) - rect->left;
            rect->height = height;
        } else {
            tr->ox = 0.0f; tr->oy = -(iiar - idar) * 0.5f * device_aspect; tr->sx = 1.0f; tr->sy = device_aspect * iiar;
            rect->left = 0;
            rect->top = (uint32_t)floorf(fmaxf(0.0f, (float)height * (iiar - idar) * 0.5f * iar));
            rect->width = width;
            rect->height = (uint32_t)ceilf((float)height * (iiar + idar) * 0.5f * iar) - rect->top;
        }
    }
}

/* ------------------------------------------------------------------------------------------------
 * Camera (Src/BuiltinComponent/Sensor/PerspectiveCamera/Kernel.cpp:22-48)
 * ---------------------------------------------------------------------------------------------- */
static void camera_ray(const pb2_camera* cam, real ndc_x, real ndc_y, real u1, real u2, v3* org, v3* dir_out) {
    const v3 base = ld3(cam->position);
    const v3 look = ld3(cam->look_at);
    const v3 forward = normalize3(sub3(look, base));
    const v3 right = cross3(forward, ld3(cam->up));
    const v3 up = cross3(right, forward);
    const v3 film_hit = add3(add3(base, mul3s(right, cam->sensor_size[0] * (0.5f - ndc_x))),
                             mul3s(up, cam->sensor_size[1] * (ndc_y - 0.5f)));
    const real focal_distance = dot3(sub3(look, base), forward);
    const real film_distance = 1.0f / (1.0f / cam->focal_length - 1.0f / focal_distance);
    const v3 lens_center = add3(base, mul3s(forward, film_distance));
    /* sampleUniformDisk (Src/Kernel/Sampling.hpp:24-29) */
    const real ang = u1 * K_TWO_PI;
    const real rad = sqrt_safe(u2);
    real s, c;
    R_SINCOS(ang, &s, &c);
    const real lx = rad * c, ly = rad * s;
    const v3 lens_hit = add3(add3(lens_center, mul3s(right, cam->aperture_radius * lx)),
                             mul3s(up, cam->aperture_radius * ly));
    const v3 dir = sub3(lens_center, film_hit);
    const v3 focus_hit = add3(lens_center, mul3s(dir, focal_distance / dot3(dir, forward)));
    *org = lens_hit;
    *dir_out = normalize3(sub3(focus_hit, lens_hit));
}

void or_camera_ray(const pb2_camera* cam, float ndc_x, float ndc_y, float u1, float u2, pb2_ray* ray) {
    v3 o, d;
    camera_ray(cam, ndc_x, ndc_y, u1, u2, &o, &d);
    ray->org[0] = (float)o.x; ray->org[1] = (float)o.y; ray->org[2] = (float)o.z;
    ray->dir[0] = (float)d.x; ray->dir[1] = (float)d.y; ray->dir[2] = (float)d.z;
    ray->tmin = 1e-3f;
    ray->tmax = 1e5f;
}

/* ------------------------------------------------------------------------------------------------
 * Scene and traversal
 * ---------------------------------------------------------------------------------------------- */
typedef struct or_node {
    float bmin[3], bmax[3];
    uint32_t first; /* leaf: first triangle slot; internal: left child (right = first + 1) */
    uint32_t count; /* 0 = internal */
} or_node;

typedef struct or_light {
    spec radiance;
    uint32_t first_plane, plane_count;
    v3 translation;
    real area, inverse_area;
} or_light;

struct or_scene {
    uint32_t ntri;
    float* tri;         /* 9 floats per triangle, world space */
    uint32_t* tri_mat;   /* material per triangle */
    uint32_t nplane;
    pb2_plane* planes;
    uint32_t* plane_light; /* area light of each plane */
    real* plane_cdf;
    real* plane_pdf;
    uint32_t nlight;     /* area lights */
    or_light* lights;
    uint32_t nmat;
    pb2_material* mats;
    real* alpha;        /* remapped roughness x, y per material */
    uint32_t ntex;
    pb2_texture* tex;   /* texels copied */
    float* tri_uv;      /* 6 floats per triangle: the texcoords of its vertices in index order, or NULL */
    spec env;
    /* BVH */
    or_node* nodes;
    uint32_t nnodes;
    uint32_t* order;     /* triangle slot -> triangle index */
};

uint32_t or_scene_triangle_count(const or_scene* s) { return s->ntri; }

typedef struct ray_pre {
    v3 o, d, id;
    int kx, ky, kz;
    real sx, sy, sz;
    real tmin, tmax;
} ray_pre;

static void ray_prepare_v(v3 o, v3 d, real tmin, real tmax, ray_pre* p) {
    p->o = o;
    p->d = d;
    const real dd[3] = { d.x, d.y, d.z };
    real inv[3];
    for (int i = 0; i < 3; ++i) inv[i] = dd[i] != 0.0f ? 1.0f / dd[i] : R_COPYSIGN(R_MAX_VALUE, dd[i]);
    p->id = mk3(inv[0], inv[1], inv[2]);
    /* Woop et al. 2013, Sec. 3: kz = dominant axis, swap kx/ky to keep winding when dir[kz] < 0 */
    int kz = 0;
    if (R_FABS(dd[1]) > R_FABS(dd[kz])) kz = 1;
    if (R_FABS(dd[2]) > R_FABS(dd[kz])) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (dd[kz] < 0.0f) { int t = kx; kx = ky; ky = t; }
    p->kx = kx; p->ky = ky; p->kz = kz;
    p->sx = dd[kx] / dd[kz];
    p->sy = dd[ky] / dd[kz];
    p->sz = 1.0f / dd[kz];
    p->tmin = tmin;
    p->tmax = tmax;
}

static void ray_prepare(const pb2_ray* r, ray_pre* p) { ray_prepare_v(ld3(r->org), ld3(r->dir), r->tmin, r->tmax, p); }

static inline real comp(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

/* Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2(1), 2013), single precision with the
 * paper's double-precision fallback for edge hits.  t = T / det; barycentrics (U, V, W) / det weight
 * (v0, v1, v2); the returned (u, v) weight v1 and v2 (Embree's convention). */
static int tri_test(const ray_pre* p, const float* tri, real* t_out, real* u_out, real* v_out) {
    const v3 A = sub3(ld3(tri + 0), p->o);
    const v3 B = sub3(ld3(tri + 3), p->o);
    const v3 C = sub3(ld3(tri + 6), p->o);
    const real Az_ = comp(A, p->kz), Bz_ = comp(B, p->kz), Cz_ = comp(C, p->kz);
    const real Ax = comp(A, p->kx) - p->sx * Az_;
    const real Ay = comp(A, p->ky) - p->sy * Az_;
    const real Bx = comp(B, p->kx) - p->sx * Bz_;
    const real By = comp(B, p->ky) - p->sy * Bz_;
    const real Cx = comp(C, p->kx) - p->sx * Cz_;
    const real Cy = comp(C, p->ky) - p->sy * Cz_;
    real U = Cx * By - Cy * Bx;
    real V = Ax * Cy - Ay * Cx;
    real W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (real)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (real)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (real)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
    const real det = U + V + W;
    if (det == 0.0f) return 0;
    const real Az = p->sz * Az_, Bz = p->sz * Bz_, Cz = p->sz * Cz_;
    const real T = U * Az + V * Bz + W * Cz;
    const real t = T / det;
    if (!(t > p->tmin && t < p->tmax)) return 0;
    *t_out = t;
    *u_out = V / det;
    *v_out = W / det;
    return 1;
}

int or_intersect_triangle(const float ray[8], const float v0[3], const float v1[3], const float v2[3], float* t,
                          float* u, float* v) {
    pb2_ray r;
    memcpy(&r, ray, sizeof(r));
    ray_pre p;
    ray_prepare(&r, &p);
    float tri[9];
    memcpy(tri, v0, 12); memcpy(tri + 3, v1, 12); memcpy(tri + 6, v2, 12);
    real tt, uu, vv;
    const int hit = tri_test(&p, tri, &tt, &uu, &vv);
    if (hit) { *t = (float)tt; *u = (float)uu; *v = (float)vv; }
    return hit;
}

/* planeIntersect + calcTexCoord (Src/BuiltinComponent/Geometry/BasicShapes/Kernel.cpp:30-79), in the
 * plane's local frame; Embree hands the callback a re-normalised direction (Embree.cpp:569-577). */
static int plane_test(const pb2_plane* pl, v3 org_local, v3 dir, real tnear, real tfar, real* t_out,
                      int* front, real uv[2]) {
    const v3 d = normalize3(dir);
    const v3 delta = sub3(ld3(pl->origin), org_local);
    const v3 n = ld3(pl->normal);
    const real b = dot3(delta, n);
    const real k = dot3(d, n);
    const real t = b / k;
    if (!(tnear < t && t < tfar)) return 0;
    const v3 pos = sub3(mul3s(d, t), delta);
    const v3 u = ld3(pl->u), v = ld3(pl->v);
    real inv_det, x, y;
    switch (pl->max_det_comp) {
        case 0:
            inv_det = 1.0f / (u.y * v.z - v.y * u.z);
            x = pos.y * v.z - v.y * pos.z;
            y = u.y * pos.z - pos.y * u.z;
            break;
        case 1:
            inv_det = 1.0f / (u.z * v.x - v.z * u.x);
            x = pos.z * v.x - v.z * pos.x;
            y = u.z * pos.x - pos.z * u.x;
            break;
        default:
            inv_det = 1.0f / (u.x * v.y - v.x * u.y);
            x = pos.x * v.y - v.x * pos.y;
            y = u.x * pos.y - pos.x * u.y;
            break;
    }
    const real uu = x * inv_det, vv = y * inv_det;
    if (!(0.0f <= uu && uu <= 1.0f && 0.0f <= vv && vv <= 1.0f)) return 0;
    *t_out = t;
    *front = k > 0.0f;
    uv[0] = uu; uv[1] = vv;
    return 1;
}

/* Conservative slab test: the far distance is widened by 3 ulp-scale (Ize 2013, "Robust BVH Ray
 * Traversal"), so rounding never culls a box holding the true closest hit.  The current best distance
 * is widened the same way: a triangle's t (watertight test arithmetic) can round a few ulp below the
 * slab entry of the flat box that holds it, and a box holding a tie at exactly the best t must still
 * be opened for the lowest-primitive tie rule (coplanar floors and box bottoms). */
static inline int box_test(const ray_pre* p, const float* bmin, const float* bmax, real tbest, real* tnear_out) {
    const real tx0 = (bmin[0] - p->o.x) * p->id.x, tx1 = (bmax[0] - p->o.x) * p->id.x;
    const real ty0 = (bmin[1] - p->o.y) * p->id.y, ty1 = (bmax[1] - p->o.y) * p->id.y;
    const real tz0 = (bmin[2] - p->o.z) * p->id.z, tz1 = (bmax[2] - p->o.z) * p->id.z;
    const real tn = R_FMAX(R_FMAX(R_FMIN(tx0, tx1), R_FMIN(ty0, ty1)), R_FMAX(R_FMIN(tz0, tz1), p->tmin));
    const real tf = R_FMIN(R_FMIN(R_FMAX(tx0, tx1), R_FMAX(ty0, ty1)), R_FMAX(tz0, tz1)) * 1.0000004f;
    *tnear_out = tn;
    return tn <= R_FMIN(tf, tbest * 1.0000004f);
}

typedef struct or_hit_rec {
    real t, u, v;
    uint32_t prim; /* triangle index or PB2_PLANE_FLAG | plane */
    int front;     /* planes only */
} or_hit_rec;

static inline void consider_tri(const or_scene* s, const ray_pre* p, uint32_t prim, or_hit_rec* h) {
    real t, u, v;
    if (tri_test(p, s->tri + 9 * (size_t)prim, &t, &u, &v)) {
        if (t < h->t || (t == h->t && prim < h->prim)) {
            h->t = t; h->u = u; h->v = v; h->prim = prim;
        }
    }
}

static void closest_tris(const or_scene* s, const ray_pre* p, or_hit_rec* h, uint64_t* nv, uint64_t* nt) {
    if (!s->nodes) {
        for (uint32_t i = 0; i < s->ntri; ++i) consider_tri(s, p, i, h);
        if (nt) *nt += s->ntri;
        return;
    }
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const or_node* n = &s->nodes[stack[--sp]];
        real tn;
        if (nv) (*nv)++;
        if (!box_test(p, n->bmin, n->bmax, h->t, &tn)) continue;
        if (n->count) {
            for (uint32_t i = 0; i < n->count; ++i) consider_tri(s, p, s->order[n->first + i], h);
            if (nt) *nt += n->count;
        } else {
            const or_node* l = &s->nodes[n->first];
            const or_node* r = &s->nodes[n->first + 1];
            real tl, tr;
            const int hl = box_test(p, l->bmin, l->bmax, h->t, &tl);
            const int hr = box_test(p, r->bmin, r->bmax, h->t, &tr);
            if (hl && hr) {
                if (tl <= tr) { stack[sp++] = n->first + 1; stack[sp++] = n->first; }
                else { stack[sp++] = n->first; stack[sp++] = n->first + 1; }
            } else if (hl) stack[sp++] = n->first;
            else if (hr) stack[sp++] = n->first + 1;
        }
    }
}

static int any_tris(const or_scene* s, const ray_pre* p, uint64_t* nv, uint64_t* nt) {
    real t, u, v;
    if (!s->nodes) {
        for (uint32_t i = 0; i < s->ntri; ++i) {
            if (nt) (*nt)++;
            if (tri_test(p, s->tri + 9 * (size_t)i, &t, &u, &v)) return 1;
        }
        return 0;
    }
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const or_node* n = &s->nodes[stack[--sp]];
        real tn;
        if (nv) (*nv)++;
        if (!box_test(p, n->bmin, n->bmax, p->tmax, &tn)) continue;
        if (n->count) {
            for (uint32_t i = 0; i < n->count; ++i) {
                if (nt) (*nt)++;
                if (tri_test(p, s->tri + 9 * (size_t)s->order[n->first + i], &t, &u, &v)) return 1;
            }
        } else {
            stack[sp++] = n->first + 1;
            stack[sp++] = n->first;
        }
    }
    return 0;
}

/* Closest hit of one ray over triangles then planes (planes lose ties: a plane is accepted only
 * strictly before the current closest t, as the callback sees tFar, BasicShapes/Kernel.cpp:69). */
static void closest_one(const or_scene* s, const ray_pre* pp, or_hit_rec* h) {
    const ray_pre p = *pp;
    h->t = p.tmax;
    h->prim = PB2_INVALID_PRIM;
    h->u = h->v = 0.0f;
    h->front = 0;
    closest_tris(s, &p, h, NULL, NULL);
    for (uint32_t i = 0; i < s->nplane; ++i) {
        const or_light* L = &s->lights[s->plane_light[i]];
        const v3 ol = sub3(p.o, L->translation);
        real t, uv[2];
        int front;
        if (plane_test(&s->planes[i], ol, p.d, p.tmin, h->t, &t, &front, uv)) {
            h->t = t; h->prim = PB2_PLANE_FLAG | i; h->front = front; h->u = uv[0]; h->v = uv[1];
        }
    }
}

void or_trace_closest(const or_scene* s, const pb2_ray* rays, uint32_t n, pb2_hit* hits, int threads) {
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        or_hit_rec h;
        ray_pre p;
        ray_prepare(&rays[i], &p);
        closest_one(s, &p, &h);
        hits[i].t = h.prim == PB2_INVALID_PRIM ? rays[i].tmax : h.t;
        hits[i].prim = h.prim;
        hits[i].u = h.u;
        hits[i].v = h.v;
    }
}

void or_trace_any(const or_scene* s, const pb2_ray* rays, uint32_t n, uint32_t* occluded, int threads) {
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        ray_pre p;
        ray_prepare(&rays[i], &p);
        occluded[i] = (uint32_t)any_tris(s, &p, NULL, NULL);
    }
}

int or_closest_triangle(const or_scene* s, const pb2_ray* ray, pb2_hit* hit) {
    ray_pre p;
    ray_prepare(ray, &p);
    or_hit_rec h;
    h.t = ray->tmax; h.prim = PB2_INVALID_PRIM; h.u = h.v = 0.0f; h.front = 0;
    closest_tris(s, &p, &h, NULL, NULL);
    hit->t = h.t; hit->prim = h.prim; hit->u = h.u; hit->v = h.v;
    return h.prim != PB2_INVALID_PRIM;
}

int or_any_triangle(const or_scene* s, const pb2_ray* ray) {
    ray_pre p;
    ray_prepare(ray, &p);
    return any_tris(s, &p, NULL, NULL);
}

const float* or_triangle_vertices(const or_scene* s, uint32_t prim) { return s->tri + 9 * (size_t)prim; }

void or_trace_counters(const or_scene* s, const pb2_ray* rays, uint32_t n, int closest, uint64_t* node_visits,
                       uint64_t* tri_tests) {
    uint64_t nv = 0, nt = 0;
    for (uint32_t i = 0; i < n; ++i) {
        ray_pre p;
        ray_prepare(&rays[i], &p);
        if (closest) {
            or_hit_rec h;
            h.t = rays[i].tmax; h.prim = PB2_INVALID_PRIM;
            closest_tris(s, &p, &h, &nv, &nt);
        } else {
            any_tris(s, &p, &nv, &nt);
        }
    }
    *node_visits = nv;
    *tri_tests = nt;
}

/* ---- binned SAH BVH over triangle centroids --------------------------------------------------- */
typedef struct build_ctx {
    const float* tri;
    float* cen;       /* 3 per triangle */
    float* tbmin;     /* 3 per triangle */
    float* tbmax;
    uint32_t* order;
    or_node* nodes;
    uint32_t nnodes;
} build_ctx;

static float area_of(const float* mn, const float* mx) {
    const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    if (dx < 0.0f) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

#define OR_BINS 16
static void build_rec(build_ctx* c, uint32_t node, uint32_t first, uint32_t count) {
    or_node* n = &c->nodes[node];
    float mn[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, mx[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
    float cmn[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, cmx[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
    for (uint32_t i = first; i < first + count; ++i) {
        const uint32_t t = c->order[i];
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], c->tbmin[3 * t + k]);
            mx[k] = fmaxf(mx[k], c->tbmax[3 * t + k]);
            cmn[k] = fminf(cmn[k], c->cen[3 * t + k]);
            cmx[k] = fmaxf(cmx[k], c->cen[3 * t + k]);
        }
    }
    memcpy(n->bmin, mn, 12);
    memcpy(n->bmax, mx, 12);
    if (count <= 4) {
        n->first = first; n->count = count;
        return;
    }
    int best_axis = -1, best_split = 0;
    float best_cost = FLT_MAX;
    for (int axis = 0; axis < 3; ++axis) {
        const float ext = cmx[axis] - cmn[axis];
        if (!(ext > 0.0f)) continue;
        uint32_t bcnt[OR_BINS] = { 0 };
        float bmn[OR_BINS][3], bmx[OR_BINS][3];
        for (int b = 0; b < OR_BINS; ++b)
            for (int k = 0; k < 3; ++k) { bmn[b][k] = FLT_MAX; bmx[b][k] = -FLT_MAX; }
        const float scale = (float)OR_BINS / ext;
        for (uint32_t i = first; i < first + count; ++i) {
            const uint32_t t = c->order[i];
            int b = (int)((c->cen[3 * t + axis] - cmn[axis]) * scale);
            if (b >= OR_BINS) b = OR_BINS - 1;
            if (b < 0) b = 0;
            bcnt[b]++;
            for (int k = 0; k < 3; ++k) {
                bmn[b][k] = fminf(bmn[b][k], c->tbmin[3 * t + k]);
                bmx[b][k] = fmaxf(bmx[b][k], c->tbmax[3 * t + k]);
            }
        }
        float lmn[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, lmx[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
        float larea[OR_BINS];
        uint32_t lcnt[OR_BINS];
        uint32_t acc = 0;
        for (int b = 0; b < OR_BINS - 1; ++b) {
            for (int k = 0; k < 3; ++k) { lmn[k] = fminf(lmn[k], bmn[b][k]); lmx[k] = fmaxf(lmx[k], bmx[b][k]); }
            acc += bcnt[b];
            larea[b] = area_of(lmn, lmx);
            lcnt[b] = acc;
        }
        float rmn[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, rmx[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
        uint32_t racc = 0;
        for (int b = OR_BINS - 1; b > 0; --b) {
            for (int k = 0; k < 3; ++k) { rmn[k] = fminf(rmn[k], bmn[b][k]); rmx[k] = fmaxf(rmx[k], bmx[b][k]); }
            racc += bcnt[b];
            const uint32_t l = lcnt[b - 1];
            if (l == 0 || racc == 0) continue;
            const float cost = larea[b - 1] * (float)l + area_of(rmn, rmx) * (float)racc;
            if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = b; }
        }
    }
    uint32_t mid;
    if (best_axis < 0) {
        mid = first + count / 2; /* all centroids equal: median split by index */
    } else {
        const float ext = cmx[best_axis] - cmn[best_axis];
        const float scale = (float)OR_BINS / ext;
        uint32_t i = first, j = first + count;
        while (i < j) {
            const uint32_t t = c->order[i];
            int b = (int)((c->cen[3 * t + best_axis] - cmn[best_axis]) * scale);
            if (b >= OR_BINS) b = OR_BINS - 1;
            if (b < 0) b = 0;
            if (b < best_split) ++i;
            else { --j; const uint32_t tmp = c->order[i]; c->order[i] = c->order[j]; c->order[j] = tmp; }
        }
        mid = i;
        if (mid == first || mid == first + count) mid = first + count / 2;
    }
    const uint32_t left = c->nnodes;
    c->nnodes += 2;
    n = &c->nodes[node];
    n->first = left;
    n->count = 0;
    build_rec(c, left, first, mid - first);
    build_rec(c, left + 1, mid, first + count - mid);
}

static void build_bvh(or_scene* s) {
    build_ctx c;
    const uint32_t nt = s->ntri;
    c.tri = s->tri;
    c.cen = (float*)malloc(sizeof(float) * 3 * nt);
    c.tbmin = (float*)malloc(sizeof(float) * 3 * nt);
    c.tbmax = (float*)malloc(sizeof(float) * 3 * nt);
    c.order = (uint32_t*)malloc(sizeof(uint32_t) * nt);
    c.nodes = (or_node*)malloc(sizeof(or_node) * (2 * (size_t)nt + 1));
    c.nnodes = 1;
    for (uint32_t i = 0; i < nt; ++i) {
        const float* t = s->tri + 9 * (size_t)i;
        for (int k = 0; k < 3; ++k) {
            const float a = t[k], b = t[3 + k], d = t[6 + k];
            c.tbmin[3 * i + k] = fminf(a, fminf(b, d));
            c.tbmax[3 * i + k] = fmaxf(a, fmaxf(b, d));
            c.cen[3 * i + k] = 0.5f * (c.tbmin[3 * i + k] + c.tbmax[3 * i + k]);
        }
        c.order[i] = i;
    }
    build_rec(&c, 0, 0, nt);
    free(c.cen);
    free(c.tbmin);
    free(c.tbmax);
    s->nodes = c.nodes;
    s->nnodes = c.nnodes;
    s->order = c.order;
}

or_scene* or_scene_create(const pb2_scene* d, int use_bvh) {
    or_scene* s = (or_scene*)calloc(1, sizeof(or_scene));
    uint64_t nt = 0;
    for (uint32_t m = 0; m < d->mesh_count; ++m) nt += d->meshes[m].tri_count;
    s->ntri = (uint32_t)nt;
    s->tri = (float*)malloc(sizeof(float) * 9 * (nt ? nt : 1));
    s->tri_mat = (uint32_t*)malloc(sizeof(uint32_t) * (nt ? nt : 1));
    uint64_t k = 0;
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        const pb2_mesh* mesh = &d->meshes[m];
        for (uint32_t i = 0; i < mesh->tri_count; ++i, ++k) {
            for (int j = 0; j < 3; ++j) {
                const uint32_t vi = mesh->indices[3 * i + j];
                pb2_mesh_vertex(mesh->transform, mesh->translation, mesh->vertices + 3 * vi, s->tri + 9 * k + 3 * j);
            }
            s->tri_mat[k] = mesh->material;
        }
    }
    s->nplane = d->plane_count;
    s->planes = (pb2_plane*)malloc(sizeof(pb2_plane) * (d->plane_count ? d->plane_count : 1));
    s->plane_light = (uint32_t*)calloc(d->plane_count ? d->plane_count : 1, sizeof(uint32_t));
    s->plane_cdf = (real*)calloc(d->plane_count ? d->plane_count : 1, sizeof(real));
    s->plane_pdf = (real*)calloc(d->plane_count ? d->plane_count : 1, sizeof(real));
    if (d->plane_count) memcpy(s->planes, d->planes, sizeof(pb2_plane) * d->plane_count);
    s->nlight = d->area_light_count;
    s->lights = (or_light*)calloc(d->area_light_count ? d->area_light_count : 1, sizeof(or_light));
    for (uint32_t l = 0; l < d->area_light_count; ++l) {
        const pb2_area_light* al = &d->area_lights[l];
        or_light* L = &s->lights[l];
        L->radiance = mksp(al->radiance[0], al->radiance[1], al->radiance[2]);
        L->first_plane = al->first_plane;
        L->plane_count = al->plane_count;
        L->translation = ld3(al->translation);
        /* BasicShapes.cpp:76-94: running area -> cdf, per-plane area -> pdf, both / total */
        real total = 0.0f;
        for (uint32_t i = 0; i < al->plane_count; ++i) {
            const pb2_plane* pl = &d->planes[al->first_plane + i];
            const real area = sqrt_safe(len2_3(cross3(ld3(pl->u), ld3(pl->v))));
            total = total + area;
            s->plane_cdf[al->first_plane + i] = total;
            s->plane_pdf[al->first_plane + i] = area;
            s->plane_light[al->first_plane + i] = l;
        }
        for (uint32_t i = 0; i < al->plane_count; ++i) {
            s->plane_cdf[al->first_plane + i] = s->plane_cdf[al->first_plane + i] / total;
            s->plane_pdf[al->first_plane + i] = s->plane_pdf[al->first_plane + i] / total;
        }
        L->area = total;
        L->inverse_area = 1.0f / total;
    }
    s->nmat = d->material_count;
    s->mats = (pb2_material*)malloc(sizeof(pb2_material) * (d->material_count ? d->material_count : 1));
    s->alpha = (real*)malloc(sizeof(real) * 2 * (d->material_count ? d->material_count : 1));
    if (d->material_count) memcpy(s->mats, d->materials, sizeof(pb2_material) * d->material_count);
    for (uint32_t m = 0; m < d->material_count; ++m) {
        const pb2_material* mt = &d->materials[m];
        if (mt->type == PB2_SURFACE_CONDUCTOR) {
            s->alpha[2 * m] = mt->roughness[0];
            s->alpha[2 * m + 1] = mt->roughness[0];
        } else if (mt->type == PB2_SURFACE_PLASTIC) {
            s->alpha[2 * m] = remap_roughness(mt->roughness[0]);
            s->alpha[2 * m + 1] = s->alpha[2 * m];
        } else {
            s->alpha[2 * m] = remap_roughness(mt->roughness[0]);
            s->alpha[2 * m + 1] = remap_roughness(mt->roughness[1]);
        }
    }
    s->ntex = d->texture_count;
    s->tex = (pb2_texture*)calloc(d->texture_count ? d->texture_count : 1, sizeof(pb2_texture));
    for (uint32_t i = 0; i < d->texture_count; ++i) {
        s->tex[i] = d->textures[i];
        if (d->textures[i].kind == PB2_TEXTURE_IMAGE) {
            const size_t n = (size_t)d->textures[i].width * d->textures[i].height * d->textures[i].channel;
            uint8_t* copy = (uint8_t*)malloc(n ? n : 1);
            memcpy(copy, d->textures[i].texels, n);
            s->tex[i].texels = copy;
        }
    }
    s->tri_uv = NULL;
    int textured = 0;
    for (uint32_t m = 0; m < d->material_count; ++m)
        for (int k = 0; k < 4; ++k) textured |= d->materials[m].texture[k] != 0;
    if (textured) {
        s->tri_uv = (float*)calloc(6 * (nt ? nt : 1), sizeof(float));
        uint64_t q = 0;
        for (uint32_t m = 0; m < d->mesh_count; ++m) {
            const pb2_mesh* mesh = &d->meshes[m];
            for (uint32_t i = 0; i < mesh->tri_count; ++i, ++q)
                if (mesh->texcoords)
                    for (int j = 0; j < 3; ++j) {
                        const uint32_t vi = mesh->indices[3 * i + j];
                        s->tri_uv[6 * q + 2 * j] = mesh->texcoords[2 * vi];
                        s->tri_uv[6 * q + 2 * j + 1] = mesh->texcoords[2 * vi + 1];
                    }
        }
    }
    s->env = mksp(d->env_radiance[0], d->env_radiance[1], d->env_radiance[2]);
    if (use_bvh && s->ntri > 0) build_bvh(s);
    return s;
}

void or_scene_destroy(or_scene* s) {
    if (!s) return;
    free(s->tri); free(s->tri_mat); free(s->planes); free(s->plane_light); free(s->plane_cdf);
    free(s->plane_pdf); free(s->lights); free(s->mats); free(s->alpha); free(s->nodes); free(s->order);
    for (uint32_t i = 0; i < s->ntex; ++i)
        if (s->tex[i].kind == PB2_TEXTURE_IMAGE) free((void*)s->tex[i].texels);
    free(s->tex); free(s->tri_uv);
    free(s);
}

/* ------------------------------------------------------------------------------------------------
 * Surface geometry at a hit
 * ---------------------------------------------------------------------------------------------- */
enum { KIND_SURFACE = 0, KIND_AREA_LIGHT = 1, KIND_MISSING = 2 };

typedef struct surf_info {
    int kind;
    real t;
    v3 T, B, N, Ng; /* local frame == world frame (translation-only instances) */
    int front;
    uint32_t material;
    uint32_t light; /* area light index */
    float tu, tv;   /* texture coordinate (triangles of a textured scene) */
} surf_info;

/* piperEmbreeTrace (Src/BuiltinComponent/Tracer/Embree/Embree.cpp:267-355) with
 * calcTriangleMeshSurface (Tracer/Embree/Kernel.cpp:170-192) and planeSurface
 * (BasicShapes/Kernel.cpp:101-111). */
static void trace_surface(const or_scene* s, v3 o, v3 d, real tmin, real tmax, surf_info* si, uint64_t* nrays) {
    ray_pre r;
    ray_prepare_v(o, d, tmin, tmax, &r);
    or_hit_rec h;
    closest_one(s, &r, &h);
    if (nrays) (*nrays)++;
    if (h.prim == PB2_INVALID_PRIM) {
        si->kind = KIND_MISSING;
        return;
    }
    si->t = h.t;
    if (h.prim & PB2_PLANE_FLAG) {
        const uint32_t pi = h.prim & ~PB2_PLANE_FLAG;
        const pb2_plane* pl = &s->planes[pi];
        si->kind = KIND_AREA_LIGHT;
        si->light = s->plane_light[pi];
        si->front = h.front;
        const v3 n = ld3(pl->normal);
        si->Ng = h.front ? neg3(n) : n;
        si->N = si->Ng;
        si->T = ld3(pl->tangent);
        si->B = cross3(si->N, si->T);
        return;
    }
    const float* tri = s->tri + 9 * (size_t)h.prim;
    const v3 p0 = ld3(tri), p1 = ld3(tri + 3), p2 = ld3(tri + 6);
    const v3 ng = normalize3(cross3(sub3(p1, p0), sub3(p2, p0)));
    const int front = dot3(d, ng) < 0.0f;
    si->kind = KIND_SURFACE;
    si->front = front;
    si->material = s->tri_mat[h.prim];
    si->N = si->Ng = front ? ng : neg3(ng);
    const v3 e1 = mk3(1.0f, 0.0f, 0.0f), e2 = mk3(0.0f, 1.0f, 0.0f);
    if (R_FABS(dot3(si->N, e1)) < R_FABS(dot3(si->N, e2)))
        si->T = cross3(si->N, e1);
    else
        si->T = cross3(si->N, e2);
    si->B = cross3(si->N, si->T);
    /* calcTriangleMeshSurface's texCoord (Tracer/Embree/Kernel.cpp:181-190): tc[i1] u + tc[i2] v + tc[i0] w */
    si->tu = si->tv = 0.0f;
    if (s->tri_uv) {
        const float* q = s->tri_uv + 6 * (size_t)h.prim;
        const real w = (1.0f - h.u) - h.v;
        si->tu = (float)((q[2] * h.u + q[4] * h.v) + q[0] * w);
        si->tv = (float)((q[3] * h.u + q[5] * h.v) + q[1] * w);
    }
}

static int occluded(const or_scene* s, v3 o, v3 d, real tmin, real tmax, uint64_t* nrays) {
    ray_pre p;
    ray_prepare_v(o, d, tmin, tmax, &p);
    if (nrays) (*nrays)++;
    return any_tris(s, &p, NULL, NULL);
}

/* SurfaceIntersectionInfo::local2Shading / shading2Local (Src/Kernel/Protocol.hpp:55-66) */
static inline v3 to_shading(const surf_info* si, v3 v) { return mk3(dot3(si->T, v), dot3(si->B, v), dot3(si->N, v)); }
static inline v3 to_local(const surf_info* si, v3 v) {
    return mk3(si->T.x * v.x + si->B.x * v.y + si->N.x * v.z, si->T.y * v.x + si->B.y * v.y + si->N.y * v.z,
               si->T.z * v.x + si->B.z * v.y + si->N.z * v.z);
}

/* ------------------------------------------------------------------------------------------------
 * BxDFs (Src/BuiltinComponent/Surface/Classic/Kernel.cpp)
 * ---------------------------------------------------------------------------------------------- */
enum {
    PART_R = 1, PART_T = 2, PART_DIFFUSE = 4, PART_SPECULAR = 8, PART_GLOSSY = 16, PART_ALL = 31,
    PART_NO_SPECULAR = 31 ^ 8
};
/* match (Protocol.hpp:143-145) */
static inline int part_match(int provide, int require) { return (provide & require) == provide; }

typedef struct bsdf_sample { v3 wi; spec f; real pdf; int part; } bsdf_sample;

/* LOBE_GGX_VNDF: the conductor extension (no reference counterpart), GGX reflection sampled with exact
 * visible-normal sampling (Heitz 2018, JCGT 7(4), listing 1) and its density G1(wo) D(wh) / (4 wo.z). */
enum { LOBE_LAMBERT, LOBE_OREN_NAYAR, LOBE_MF_REFL, LOBE_FRESNEL_SPEC, LOBE_MF_TRANS, LOBE_MIRROR, LOBE_BLEND,
       LOBE_GGX_VNDF };
enum { FRESNEL_DIELECTRIC, FRESNEL_SCHLICK };

typedef struct lobe {
    int type;
    int part;
    spec color;   /* reflection / transmission */
    spec color2;  /* FresnelBlend specular, Schlick F0 */
    real a, b;   /* Oren-Nayar A, B */
    real ax, ay; /* microfacet alphas */
    real eta_i, eta_t;
    real eta, correct;
    int fresnel;
} lobe;

typedef struct bsdf {
    int n;
    lobe l[3];
    int no_specular;
    int mirror; /* Mirror surface: sample only, evaluate/pdf are the black body's (Classic.cpp:163-166) */
} bsdf;

/* FresnelDielectric (Kernel.cpp:271-286) */
static real fresnel_dielectric(real eta_i, real eta_t, real cos_i) {
    cos_i = R_FMAX(0.0f, R_FMIN(1.0f, R_FABS(cos_i)));
    const real sin_i = sqrt_safe(1.0f - cos_i * cos_i);
    const real sin_t = eta_i / eta_t * sin_i;
    if (sin_t >= 1.0f) return 1.0f;
    const real cos_t = sqrt_safe(1.0f - sin_t * sin_t);
    const real p1 = eta_t * cos_i, p2 = eta_i * cos_t;
    const real par = (p1 - p2) / (p1 + p2);
    const real p3 = eta_i * cos_i, p4 = eta_t * cos_t;
    const real perp = (p3 - p4) / (p3 + p4);
    return 0.5f * (par * par + perp * perp);
}

static spec lobe_fresnel(const lobe* L, real c) {
    if (L->fresnel == FRESNEL_SCHLICK) {
        /* extension: Schlick's approximation F0 + (1 - F0)(1 - cos)^5 */
        const real m = 1.0f - R_FMIN(1.0f, R_FABS(c));
        const real m5 = (m * m) * (m * m) * m;
        return mksp(L->color2.r + (1.0f - L->color2.r) * m5, L->color2.g + (1.0f - L->color2.g) * m5,
                    L->color2.b + (1.0f - L->color2.b) * m5);
    }
    const real f = fresnel_dielectric(L->eta_i, L->eta_t, c);
    return mksp(f, f, f);
}

/* MicrofacetDistribution (Kernel.cpp:289-382) */
static real mf_lambda(real ax, real ay, v3 w) {
    const real cos2 = w.z * w.z;
    const real sin2 = R_FMAX(0.0f, 1.0f - cos2);
    const real tan2 = sin2 / cos2;
    if (isinf(tan2)) return 0.0f;
    const real sin_t = R_SQRT(sin2);
    const real cos_phi = sin_t == 0.0f ? 1.0f : R_FMIN(1.0f, R_FMAX(-1.0f, w.x / sin_t));
    const real p1 = cos_phi * ax;
    const real sin_phi = sin_t == 0.0f ? 0.0f : R_FMIN(1.0f, R_FMAX(-1.0f, w.y / sin_t));
    const real p2 = sin_phi * ay;
    const real sqr = (p1 * p1 + p2 * p2) * tan2;
    return (-1.0f + R_SQRT(1.0f + sqr)) * 0.5f;
}

static real mf_d(real ax, real ay, v3 wh) {
    const real cos2 = wh.z * wh.z;
    const real sin2 = R_FMAX(0.0f, 1.0f - cos2);
    const real tan2 = sin2 / cos2;
    if (isinf(tan2)) return 0.0f;
    const real sin_t = R_SQRT(sin2);
    const real cos_phi = sin_t == 0.0f ? 1.0f : R_FMIN(1.0f, R_FMAX(-1.0f, wh.x / sin_t));
    const real p1 = cos_phi / ax;
    const real sin_phi = sin_t == 0.0f ? 0.0f : R_FMIN(1.0f, R_FMAX(-1.0f, wh.y / sin_t));
    const real p2 = sin_phi / ay;
    const real e = cos2 * (1.0f + (p1 * p1 + p2 * p2) * tan2);
    return K_INV_PI / (ax * ay * e * e);
}

static void mf_sample11(real cos_theta, real u1, real u2, real* sx, real* sy) {
    if (cos_theta > 1.0f - 1e-5f) {
        const real r = R_SQRT(u1 / (1.0f - u1));
        const real phi = K_TWO_PI * u2;
        real s, c;
        R_SINCOS(phi, &s, &c);
        *sx = r * c;
        *sy = r * s;
        return;
    }
    const real sin_t = sqrt_safe(1.0f - cos_theta * cos_theta);
    const real tan_t = sin_t / cos_theta;
    const real tan2 = tan_t * tan_t;
    const real g1 = 2.0f / (1.0f + R_SQRT(1.0f + tan2));
    const real a = 2.0f * u1 / g1 - 1.0f;
    const real a2 = a * a;
    const real v = R_FMIN(1e10f, 1.0f / (a2 - 1.0f));
    const real d = sqrt_safe(tan2 * v * v - (a2 - tan2) * v);
    const real p = tan_t * v;
    const real p1 = p - d;
    const real p2 = p + d;
    const real x = (a < 0.0f || p2 > 1.0f / tan_t) ? p1 : p2;
    const real s = u2 > 0.5f ? 1.0f : -1.0f;
    const real nu2 = (u2 > 0.5f ? 2.0f : -2.0f) * (u2 - 0.5f);
    const real z = (nu2 * (nu2 * (nu2 * 0.27385f - 0.73369f) + 0.46341f)) /
                    (nu2 * (nu2 * (nu2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
    *sx = x;
    *sy = s * z * R_SQRT(1.0f + x * x);
}

static v3 mf_sample_wh(real ax, real ay, v3 wi, real u1, real u2) {
    const v3 st = normalize3(mk3(ax * wi.x, ay * wi.y, wi.z));
    real sx, sy;
    mf_sample11(st.z, u1, u2, &sx, &sy);
    const real sin_t = sqrt_safe(1.0f - st.z * st.z);
    const real cos_phi = sin_t == 0.0f ? 1.0f : R_FMIN(1.0f, R_FMAX(-1.0f, st.x / sin_t));
    const real sin_phi = sin_t == 0.0f ? 0.0f : R_FMIN(1.0f, R_FMAX(-1.0f, st.y / sin_t));
    const real rx = cos_phi * sx - sin_phi * sy;
    const real ry = sin_phi * sx + cos_phi * sy;
    return normalize3(mk3(-rx * ax, -ry * ay, 1.0f));
}

/* halfVector (Transform.hpp:279-282) */
static inline v3 half_vector(v3 a, v3 b) { return normalize3(mk3(a.x + b.x, a.y + b.y, a.z + b.z)); }

/* Heitz 2018, listing 1: a visible normal of the GGX distribution (ax, ay) seen from wo (wo.z > 0). */
static v3 ggx_sample_vndf(real ax, real ay, v3 wo, real u1, real u2) {
    const v3 vh = normalize3(mk3(ax * wo.x, ay * wo.y, wo.z));
    const real lensq = vh.x * vh.x + vh.y * vh.y;
    v3 t1 = mk3(1.0f, 0.0f, 0.0f);
    if (lensq > 0.0f) {
        const real inv = 1.0f / R_SQRT(lensq);
        t1 = mk3(-vh.y * inv, vh.x * inv, 0.0f);
    }
    const v3 t2 = cross3(vh, t1);
    const real r = R_SQRT(u1);
    real sp, cp;
    R_SINCOS(K_TWO_PI * u2, &sp, &cp);
    const real p1 = r * cp;
    const real s = 0.5f * (1.0f + vh.z);
    const real p2 = (1.0f - s) * sqrt_safe(1.0f - p1 * p1) + s * (r * sp);
    const real pz = sqrt_safe(1.0f - p1 * p1 - p2 * p2);
    const v3 nh = mk3(p1 * t1.x + p2 * t2.x + pz * vh.x, p1 * t1.y + p2 * t2.y + pz * vh.y,
                      p1 * t1.z + p2 * t2.z + pz * vh.z);
    return normalize3(mk3(ax * nh.x, ay * nh.y, R_FMAX(0.0f, nh.z)));
}
/* reflect (Transform.hpp:405-408) */
static inline v3 reflect3(v3 wo, v3 n) { return sub3(mul3s(n, 2.0f * dot3(wo, n)), wo); }
/* refract (Transform.hpp:410-421) */
static int refract3(v3 wi, v3 n, real eta, v3* wt) {
    const real cos_i = dot3(n, wi);
    const real sin2_i = R_FMAX(0.0f, 1.0f - cos_i * cos_i);
    const real sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return 0;
    const real cos_t = sqrt_safe(1.0f - sin2_t);
    *wt = normalize3(sub3(mul3s(n, eta * cos_i - cos_t), mul3s(wi, eta)));
    return 1;
}

/* sampleConcentricDisk / sampleCosineHemisphere (Src/Kernel/Sampling.hpp:31-50) */
static v3 sample_cosine_hemisphere(real u1, real u2) {
    u1 = 2.0f * u1 - 1.0f;
    u2 = 2.0f * u2 - 1.0f;
    const real au1 = R_FABS(u1), au2 = R_FABS(u2);
    real cx, cy;
    if (R_FMIN(au1, au2) < 1e-4f) {
        cx = 0.0f; cy = 0.0f;
    } else {
        const real rad = au1 > au2 ? u1 : u2;
        const real theta = au1 > au2 ? K_QUARTER_PI * (u2 / u1) : K_HALF_PI - K_QUARTER_PI * (u1 / u2);
        real s, c;
        R_SINCOS(theta, &s, &c);
        cx = c * rad; cy = s * rad;
    }
    const real z = sqrt_safe(1.0f - (cx * cx + cy * cy));
    return mk3(cx, cy, z);
}

static spec lobe_eval(const lobe* L, v3 wo, v3 wi) {
    switch (L->type) {
        case LOBE_LAMBERT: /* Kernel.cpp:89-91 */
            return sp_muls(L->color, K_INV_PI);
        case LOBE_OREN_NAYAR: { /* Kernel.cpp:111-139 */
            const real sin_i = sqrt_safe(1.0f - wi.z * wi.z);
            const real sin_o = sqrt_safe(1.0f - wo.z * wo.z);
            if (sin_i < 1e-4f || sin_o < 1e-4f) return SP_ZERO;
            const real cos_phi_i = sin_i == 0.0f ? 1.0f : R_FMIN(1.0f, R_FMAX(-1.0f, wi.x / sin_i));
            const real sin_phi_i = sin_i == 0.0f ? 0.0f : R_FMIN(1.0f, R_FMAX(-1.0f, wi.y / sin_i));
            const real cos_phi_o = sin_o == 0.0f ? 1.0f : R_FMIN(1.0f, R_FMAX(-1.0f, wo.x / sin_o));
            const real sin_phi_o = sin_o == 0.0f ? 0.0f : R_FMIN(1.0f, R_FMAX(-1.0f, wo.y / sin_o));
            const real max_cos = R_FMAX(0.0f, cos_phi_i * cos_phi_o + sin_phi_i * sin_phi_o);
            real sin_alpha, tan_beta;
            if (R_FABS(wi.z) > R_FABS(wo.z)) { sin_alpha = sin_o; tan_beta = sin_i / R_FABS(wi.z); }
            else { sin_alpha = sin_i; tan_beta = sin_o / R_FABS(wo.z); }
            return sp_muls(L->color, K_INV_PI * (L->a + L->b * max_cos * sin_alpha * tan_beta));
        }
        case LOBE_MF_REFL: { /* Kernel.cpp:397-404 */
            const v3 wh = half_vector(wo, wi);
            const spec F = lobe_fresnel(L, dot3(wi, wh));
            const real q = mf_d(L->ax, L->ay, wh) /
                            (4.0f * (1.0f + mf_lambda(L->ax, L->ay, wo) + mf_lambda(L->ax, L->ay, wi)) * R_FABS(wo.z * wi.z));
            return sp_mul(L->color, mksp(F.r * q, F.g * q, F.b * q));
        }
        case LOBE_GGX_VNDF: {
            if (wo.z <= 0.0f || wi.z <= 0.0f) return SP_ZERO;
            const v3 wh = half_vector(wo, wi);
            const spec F = lobe_fresnel(L, dot3(wi, wh));
            const real q = mf_d(L->ax, L->ay, wh) /
                            (4.0f * (1.0f + mf_lambda(L->ax, L->ay, wo) + mf_lambda(L->ax, L->ay, wi)) * (wo.z * wi.z));
            return sp_mul(L->color, mksp(F.r * q, F.g * q, F.b * q));
        }
        case LOBE_MF_TRANS: { /* Kernel.cpp:553-573 */
            if (wi.z >= 0.0f) return SP_ZERO;
            v3 wh = normalize3(add3(wo, mul3s(wi, L->eta)));
            if (wh.z < 0.0f) wh = neg3(wh);
            if (dot3(wo, wh) * dot3(wi, wh) > 0.0f) return SP_ZERO;
            const real f = fresnel_dielectric(L->eta_i, L->eta_t, dot3(wo, wh));
            const real sd = dot3(wo, wh) + L->eta * dot3(wi, wh);
            const real num = (1.0f - f) * mf_d(L->ax, L->ay, wh) * R_FABS(dot3(wi, wh)) * R_FABS(dot3(wo, wh)) * L->correct;
            const real den = (1.0f + mf_lambda(L->ax, L->ay, wo) + mf_lambda(L->ax, L->ay, wi)) * wo.z * wi.z * (sd * sd);
            return sp_muls(L->color, R_FABS(num / den));
        }
        case LOBE_BLEND: { /* FresnelBlend::evaluate (Kernel.cpp:706-722) */
            const spec nrs = sp_add(L->color2, mksp(-1.0f, -1.0f, -1.0f));
            const real pi5 = 1.0f - 0.5f * R_FABS(wi.z), po5 = 1.0f - 0.5f * R_FABS(wo.z);
            const real pw_i = (pi5 * pi5) * (pi5 * pi5) * pi5, pw_o = (po5 * po5) * (po5 * po5) * po5;
            const real k = -28.f / (23.f * K_PI) * (1.0f - pw_i) * (1.0f - pw_o);
            const spec diffuse = sp_muls(sp_mul(L->color, nrs), k);
            const v3 wh = half_vector(wo, wi);
            const real cm1 = dot3(wi, wh) - 1.0f;
            const real p5 = (cm1 * cm1) * (cm1 * cm1) * cm1;
            const spec schlick = sp_add(L->color2, sp_muls(nrs, p5));
            const real denom = 4.0f * R_FMAX(R_FABS(wi.z), R_FABS(wo.z)) * R_FABS(dot3(wi, wh));
            const spec specular = sp_muls(schlick, mf_d(L->ax, L->ay, wh) / denom);
            return sp_add(diffuse, specular);
        }
        default: /* specular lobes: delta, evaluate = 0 */
            return SP_ZERO;
    }
}

static real lobe_pdf(const lobe* L, v3 wo, v3 wi) {
    switch (L->type) {
        case LOBE_LAMBERT:
        case LOBE_OREN_NAYAR: /* DefaultBxDFHelper::pdf (Kernel.cpp:76-78) */
            return wi.z > 0.0f ? R_FABS(wi.z) * K_INV_PI : 0.0f;
        case LOBE_MF_REFL: { /* Kernel.cpp:405-412 */
            if (wi.z <= 0.0f) return 0.0f;
            const v3 wh = half_vector(wo, wi);
            const real p1 = 1.0f + mf_lambda(L->ax, L->ay, wo);
            const real p2 = mf_lambda(L->ax, L->ay, wh);
            return R_FABS(0.25f / (wo.z * p1 * (p1 + p2)));
        }
        case LOBE_GGX_VNDF: {
            if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
            const v3 wh = half_vector(wo, wi);
            if (dot3(wo, wh) <= 0.0f) return 0.0f;
            return mf_d(L->ax, L->ay, wh) / (4.0f * wo.z * (1.0f + mf_lambda(L->ax, L->ay, wo)));
        }
        case LOBE_MF_TRANS: { /* Kernel.cpp:574-586 */
            if (wi.z >= 0.0f) return 0.0f;
            const v3 wh = normalize3(add3(wo, mul3s(wi, L->eta)));
            if (dot3(wo, wh) * dot3(wi, wh) > 0.0f) return 0.0f;
            const real sd = dot3(wo, wh) + L->eta * dot3(wi, wh);
            const real q = L->eta / sd;
            const real delta = R_FABS((q * q) * dot3(wi, wh));
            return mf_d(L->ax, L->ay, wh) * R_FABS(dot3(wo, wh)) * delta /
                   ((1.0f + mf_lambda(L->ax, L->ay, wo)) * R_FABS(wo.z));
        }
        case LOBE_BLEND: { /* Kernel.cpp:723-732 */
            if (wi.z <= 0.0f) return 0.0f;
            const v3 wh = half_vector(wo, wi);
            return 0.5f * (R_FABS(wi.z) * K_INV_PI +
                           mf_d(L->ax, L->ay, wh) /
                               (4.0f * R_FABS(wo.z) * (1.0f + mf_lambda(L->ax, L->ay, wo) + mf_lambda(L->ax, L->ay, wh))));
        }
        default:
            return 0.0f;
    }
}

/* Per-lobe sample; leaves res->pdf untouched when it rejects (the caller preset it to 0). */
static void lobe_sample(const lobe* L, real u1, real u2, v3 wo, bsdf_sample* res) {
    switch (L->type) {
        case LOBE_LAMBERT:
        case LOBE_OREN_NAYAR: /* DefaultBxDFHelper::sample (Kernel.cpp:68-74) */
            res->wi = sample_cosine_hemisphere(u1, u2);
            res->f = lobe_eval(L, wo, res->wi);
            res->pdf = lobe_pdf(L, wo, res->wi);
            res->part = L->part;
            return;
        case LOBE_MF_REFL: { /* Kernel.cpp:413-432 */
            if (wo.z == 0.0f) return;
            const v3 wh = mf_sample_wh(L->ax, L->ay, wo, u1, u2);
            if (dot3(wo, wh) < 0.0f) return;
            res->wi = reflect3(wo, wh);
            if (res->wi.z <= 0.0f) return;
            const real p1 = 1.0f + mf_lambda(L->ax, L->ay, wo);
            const spec F = lobe_fresnel(L, dot3(res->wi, wh));
            const real q = mf_d(L->ax, L->ay, wh) / (4.0f * (p1 + mf_lambda(L->ax, L->ay, res->wi)) * R_FABS(wo.z * res->wi.z));
            res->f = sp_mul(L->color, mksp(F.r * q, F.g * q, F.b * q));
            res->part = L->part;
            const real p2 = mf_lambda(L->ax, L->ay, wh);
            res->pdf = R_FABS(0.25f / (wo.z * p1 * (p1 + p2)));
            return;
        }
        case LOBE_GGX_VNDF: {
            if (wo.z <= 0.0f) return;
            const v3 wh = ggx_sample_vndf(L->ax, L->ay, wo, u1, u2);
            res->wi = reflect3(wo, wh);
            if (res->wi.z <= 0.0f) return;
            res->f = lobe_eval(L, wo, res->wi);
            res->pdf = lobe_pdf(L, wo, res->wi);
            res->part = L->part;
            return;
        }
        case LOBE_FRESNEL_SPEC: { /* FresnelSpecular::sample (Kernel.cpp:519-536) */
            const real f = fresnel_dielectric(L->eta_i, L->eta_t, wo.z);
            if (u1 < f) {
                res->wi = mk3(-wo.x, -wo.y, wo.z);
                res->part = PART_R | PART_SPECULAR;
                res->pdf = f;
                res->f = sp_muls(L->color, f / R_FABS(res->wi.z));
            } else {
                v3 wt;
                if (!refract3(wo, mk3(0.0f, 0.0f, 1.0f), L->eta, &wt)) return;
                res->wi = wt;
                res->part = PART_T | PART_SPECULAR;
                res->pdf = 1.0f - f;
                res->f = sp_muls(L->color2, L->correct * res->pdf / R_FABS(res->wi.z));
            }
            return;
        }
        case LOBE_MF_TRANS: { /* Kernel.cpp:587-599 */
            if (wo.z == 0.0f) return;
            const v3 wh = mf_sample_wh(L->ax, L->ay, wo, u1, u2);
            if (dot3(wo, wh) < 0.0f) return;
            v3 wt;
            if (!refract3(wo, wh, L->eta, &wt)) return;
            res->wi = wt;
            res->part = L->part;
            res->f = lobe_eval(L, wo, wt);
            res->pdf = lobe_pdf(L, wo, wt);
            return;
        }
        case LOBE_BLEND: { /* FresnelBlend::sample (Kernel.cpp:733-747) */
            if (u1 < 0.5f) {
                u1 = R_FMIN(2.0f * u1, 1.0f);
                res->wi = sample_cosine_hemisphere(u1, u2);
            } else {
                u1 = R_FMIN(2.0f * (u1 - 0.5f), 1.0f);
                const v3 wh = mf_sample_wh(L->ax, L->ay, wo, u1, u2);
                res->wi = reflect3(wo, wh);
                if (res->wi.z <= 0.0f) return;
            }
            res->part = L->part;
            res->pdf = lobe_pdf(L, wo, res->wi);
            res->f = lobe_eval(L, wo, res->wi);
            return;
        }
        default:
            return;
    }
}

/* Surface init (matteInit :249-268, plasticInit :441-470, glassInit :613-656, mirrorInit :668-677,
 * substrateInit :755-778, blackBodyInit :45-48).  Lobe order = the KERNEL_FUNCTION_GROUP order. */
/* The material's textured parameters at (tu, tv) (CheckBoard, ProceduralTexture/Kernel.cpp:27-38; SampledTexture,
 * SampledTexture/Kernel.cpp:59-83); a textured roughness is remapped per point with pb2_logf. */
static void texture_value(const pb2_texture* t, float tu, float tv, float* out) {
    if (t->kind == PB2_TEXTURE_IMAGE) {
        pb2_tex_sample(t->texels, t->width, t->height, t->channel, t->wrap, tu, tv, out);
    } else {
        const float* arr = pb2_checker_white(tu, tv, t->scale) ? t->white : t->black;
        for (uint32_t i = 0; i < t->channel; ++i) out[i] = arr[i];
    }
}

void or_texture_sample(const pb2_texture* t, float tu, float tv, float* out) { texture_value(t, tu, tv, out); }

static void bsdf_init(const or_scene* s, uint32_t mat, int front, float tu, float tv, bsdf* b) {
    pb2_material mm = s->mats[mat];
    const pb2_material* m = &mm;
    real ax = s->alpha[2 * mat], ay = s->alpha[2 * mat + 1];
    for (int k = 0; k < 4; ++k) {
        if (!mm.texture[k]) continue;
        float v[4] = { 0.0f, 0.0f, 0.0f, 0.0f };
        texture_value(&s->tex[mm.texture[k] - 1], tu, tv, v);
        if (k == 0) { mm.color0[0] = v[0]; mm.color0[1] = v[1]; mm.color0[2] = v[2]; }
        if (k == 1) { mm.color1[0] = v[0]; mm.color1[1] = v[1]; mm.color1[2] = v[2]; }
        if (k == 2) {
            mm.roughness[0] = v[0];
            if (mm.type == PB2_SURFACE_CONDUCTOR) ax = ay = v[0];
            else if (mm.type == PB2_SURFACE_PLASTIC) ax = ay = pb2_remap_roughness(v[0]);
            else ax = pb2_remap_roughness(v[0]);
        }
        if (k == 3) {
            mm.roughness[1] = v[0];
            if (mm.type != PB2_SURFACE_CONDUCTOR && mm.type != PB2_SURFACE_PLASTIC) ay = pb2_remap_roughness(v[0]);
        }
    }
    const spec c0 = mksp(m->color0[0], m->color0[1], m->color0[2]);
    const spec c1 = mksp(m->color1[0], m->color1[1], m->color1[2]);
    memset(b, 0, sizeof(*b));
    switch (m->type) {
        case PB2_SURFACE_MATTE: {
            lobe* L = &b->l[b->n++];
            L->part = PART_DIFFUSE | PART_R;
            L->color = c0;
            if (m->roughness[0] > 0.0f) {
                L->type = LOBE_OREN_NAYAR;
                const real sigma = m->roughness[0] * K_PI;
                const real sigma2 = sigma * sigma;
                L->a = 1.0f - (sigma2 / (2.0f * (sigma2 + 0.33f)));
                L->b = 0.45f * sigma2 / (sigma2 + 0.09f);
            } else {
                L->type = LOBE_LAMBERT;
            }
            b->no_specular = 1;
            break;
        }
        case PB2_SURFACE_PLASTIC: {
            if (sp_valid(c0)) {
                lobe* L = &b->l[b->n++];
                L->type = LOBE_LAMBERT; L->part = PART_DIFFUSE | PART_R; L->color = c0;
            }
            if (sp_valid(c1)) {
                lobe* L = &b->l[b->n++];
                L->type = LOBE_MF_REFL; L->part = PART_GLOSSY | PART_R; L->color = c1;
                L->fresnel = FRESNEL_DIELECTRIC;
                L->eta_i = front ? 1.0f : 1.46f;
                L->eta_t = front ? 1.46f : 1.0f;
                L->ax = ax; L->ay = ax;
            }
            b->no_specular = 1;
            break;
        }
        case PB2_SURFACE_CONDUCTOR: {
            lobe* L = &b->l[b->n++];
            L->type = LOBE_GGX_VNDF; L->part = PART_GLOSSY | PART_R;
            L->color = mksp(1.0f, 1.0f, 1.0f);
            L->color2 = c1;
            L->fresnel = FRESNEL_SCHLICK;
            L->ax = ax; L->ay = ay;
            b->no_specular = 1;
            break;
        }
        case PB2_SURFACE_GLASS: {
            if (!sp_valid(c0) && !sp_valid(c1)) { b->no_specular = 0; break; }
            const real eta_i = front ? 1.0f : 1.5f, eta_t = front ? 1.5f : 1.0f;
            if (m->roughness[0] == 0.0f && m->roughness[1] == 0.0f) {
                lobe* L = &b->l[b->n++];
                L->type = LOBE_FRESNEL_SPEC; L->part = PART_R | PART_T | PART_SPECULAR;
                L->color = c0; L->color2 = c1;
                L->eta_i = eta_i; L->eta_t = eta_t;
                L->eta = eta_i / eta_t;
                L->correct = L->eta * L->eta; /* TransportMode::Radiance */
                b->no_specular = 0;
            } else {
                if (sp_valid(c0)) {
                    lobe* L = &b->l[b->n++];
                    L->type = LOBE_MF_REFL; L->part = PART_GLOSSY | PART_R; L->color = c0;
                    L->fresnel = FRESNEL_DIELECTRIC; L->eta_i = eta_i; L->eta_t = eta_t; L->ax = ax; L->ay = ay;
                }
                if (sp_valid(c1)) {
                    lobe* L = &b->l[b->n++];
                    L->type = LOBE_MF_TRANS; L->part = PART_GLOSSY | PART_T; L->color = c1;
                    L->eta_i = eta_i; L->eta_t = eta_t; L->ax = ax; L->ay = ay;
                    L->eta = eta_t / eta_i;
                    L->correct = 1.0f; /* TransportMode::Radiance */
                }
                b->no_specular = 1;
            }
            break;
        }
        case PB2_SURFACE_MIRROR: {
            lobe* L = &b->l[b->n++];
            L->type = LOBE_MIRROR; L->part = PART_R | PART_SPECULAR; L->color = c0;
            b->mirror = 1;
            b->no_specular = 0;
            break;
        }
        case PB2_SURFACE_SUBSTRATE: {
            if (!sp_valid(c0) && !sp_valid(c1)) { b->no_specular = 0; break; }
            lobe* L = &b->l[b->n++];
            L->type = LOBE_BLEND; L->part = PART_GLOSSY | PART_R; L->color = c0; L->color2 = c1;
            L->ax = ax; L->ay = ay;
            b->no_specular = 1;
            break;
        }
        default: /* black body */
            b->no_specular = 0;
            break;
    }
}

static uint32_t bsdf_count(const bsdf* b, int require) {
    uint32_t c = 0;
    for (int i = 0; i < b->n; ++i) c += part_match(b->l[i].part, require);
    return c;
}

/* sample() of KERNEL_FUNCTION_GROUP (Kernel.cpp:186-206) */
static void bsdf_sample_fn(const bsdf* b, real u1, real u2, v3 wo, v3 ng, int require, bsdf_sample* out) {
    out->pdf = 0.0f;
    if (b->mirror) { /* mirrorSample (Kernel.cpp:680-692) */
        const int part = PART_R | PART_SPECULAR;
        if (part_match(part, require)) {
            out->wi = mk3(-wo.x, -wo.y, wo.z);
            out->f = sp_divs(b->l[0].color, R_FABS(out->wi.z));
            out->part = part;
            out->pdf = 1.0f;
        }
        return;
    }
    const uint32_t count = bsdf_count(b, require);
    if (count == 0) return;
    uint32_t sel = (uint32_t)R_FLOOR(u1 * (real)count);
    if (sel > count - 1) sel = count - 1;
    u1 = u1 * (real)count - (real)sel;
    int chosen = -1;
    for (int i = 0, k = 0; i < b->n; ++i) {
        if (!part_match(b->l[i].part, require)) continue;
        if ((uint32_t)k == sel) { chosen = i; break; }
        ++k;
    }
    lobe_sample(&b->l[chosen], u1, u2, wo, out);
    if (out->pdf <= 0.0f) return;
    if (!(out->part & PART_SPECULAR)) {
        const int addition = (dot3(wo, ng) * dot3(out->wi, ng)) > 0.0f ? PART_R : PART_T;
        for (int i = 0; i < b->n; ++i) { /* evaluateN (:168-176) */
            if (i == chosen || !part_match(b->l[i].part, require)) continue;
            if (addition & b->l[i].part) out->f = sp_add(out->f, lobe_eval(&b->l[i], wo, out->wi));
        }
        for (int i = 0; i < b->n; ++i) { /* pdfN (:158-166) */
            if (i == chosen || !part_match(b->l[i].part, require)) continue;
            out->pdf = out->pdf + lobe_pdf(&b->l[i], wo, out->wi);
        }
    }
    if (count > 1) out->pdf = out->pdf / (real)count;
}

/* PREFIX##Evaluate (Kernel.cpp:217-224) */
static spec bsdf_eval(const bsdf* b, v3 wo, v3 wi, v3 ng, int require) {
    if (b->mirror) return SP_ZERO;
    const int addition = (dot3(wo, ng) * dot3(wi, ng)) > 0.0f ? PART_R : PART_T;
    spec f = SP_ZERO;
    for (int i = 0; i < b->n; ++i)
        if (part_match(b->l[i].part, require) && (addition & b->l[i].part)) f = sp_add(f, lobe_eval(&b->l[i], wo, wi));
    return f;
}

/* PREFIX##Pdf (Kernel.cpp:226-236) */
static real bsdf_pdf(const bsdf* b, v3 wo, v3 wi, int require) {
    if (b->mirror) return 0.0f;
    const uint32_t count = bsdf_count(b, require);
    if (count == 0) return 0.0f;
    real pdf = 0.0f;
    for (int i = 0; i < b->n; ++i)
        if (part_match(b->l[i].part, require)) pdf = pdf + lobe_pdf(&b->l[i], wo, wi);
    if (count > 1) pdf = pdf / (real)count;
    return pdf;
}

/* ------------------------------------------------------------------------------------------------
 * Lights (Src/BuiltinComponent/Light/...)
 * ---------------------------------------------------------------------------------------------- */
typedef struct light_sample { v3 dir; spec rad; real pdf; real distance; } light_sample;

/* select() (Src/Kernel/Sampling.hpp:52-63): note u is remapped with cdf[r] itself. */
static uint32_t cdf_select(const real* cdf, const real* pdf, uint32_t size, real* u) {
    uint32_t l = 0, r = size;
    while (l < r) {
        const uint32_t mid = (l + r) >> 1;
        if (*u >= cdf[mid]) l = mid + 1;
        else r = mid;
    }
    /* u == 1.0f (a Sobol value whose real conversion rounds up to 2^32) makes the reference read one
     * entry past the end; the library and this restatement use the last entry instead */
    if (r >= size) r = size - 1;
    *u = (*u - cdf[r]) / pdf[r];
    return r;
}

/* diffuseSample (AreaLight/Kernel.cpp:24-41) over planeSample (BasicShapes/Kernel.cpp:113-134) */
static void area_sample(const or_scene* s, uint32_t li, v3 hit, real u1, real u2, light_sample* ls) {
    const or_light* L = &s->lights[li];
    const uint32_t idx = cdf_select(s->plane_cdf + L->first_plane, s->plane_pdf + L->first_plane, L->plane_count, &u1);
    const pb2_plane* pl = &s->planes[L->first_plane + idx];
    const v3 lp = add3(add3(ld3(pl->origin), mul3s(ld3(pl->u), u1)), mul3s(ld3(pl->v), u2));
    const v3 src = add3(lp, L->translation);
    v3 n = ld3(pl->normal);
    if (dot3(sub3(hit, src), n) <= 0.0f) n = neg3(n);
    real pdf = L->inverse_area;
    const v3 delta = sub3(src, hit);
    if (pdf == 0.0f || dot3(delta, n) >= 0.0f) {
        ls->pdf = 0.0f;
        return;
    }
    ls->rad = L->radiance;
    const real dis2 = len2_3(delta);
    ls->distance = R_SQRT(dis2);
    ls->dir = div3s(delta, ls->distance);
    ls->pdf = pdf * dis2 / R_FABS(dot3(n, ls->dir));
}

/* SESample (BasicLight/Kernel.cpp:61-73): phi covers [0, pi] only, as in the reference. */
static void env_sample(const or_scene* s, real u1, real u2, light_sample* ls) {
    ls->rad = s->env;
    const real theta = u1 * K_PI, phi = u2 * K_PI;
    real st, ct, sp, cp;
    R_SINCOS(theta, &st, &ct);
    R_SINCOS(phi, &sp, &cp);
    ls->dir = mk3(st * cp, st * sp, ct);
    ls->pdf = st == 0.0f ? 0.0f : 1.0f / ((2.0f * K_SQR_PI) * st);
    ls->distance = 1e5f;
}

/* SEPdf (BasicLight/Kernel.cpp:80-89) */
static real env_pdf(v3 dir) {
    const real theta = R_ACOS(R_FMAX(-1.0f, R_FMIN(1.0f, dir.z)));
    const real st = R_SIN(theta);
    return st == 0.0f ? 0.0f : 1.0f / ((2.0f * K_SQR_PI) * st);
}

/* ------------------------------------------------------------------------------------------------
 * Integrator (Src/BuiltinComponent/Integrator/PathTracing/Kernel.cpp:23-193)
 * ---------------------------------------------------------------------------------------------- */
typedef struct path_ctx {
    const or_scene* s;
    uint64_t index;
    uint32_t dim;
    uint32_t scramble, seed; /* Owen scrambling of dimensions >= 2 (extension, pb2_math.h) */
    int overflow;
    uint64_t closest_rays, shadow_rays;
} path_ctx;

/* piperSample (Tracer/Embree/Kernel.cpp:37-45); the mt19937_64 tail past dimension 1023 is not
 * reproduced (settings that could reach it are rejected up front). */
/* Dimension `dim` (>= 2) of a sample, Owen-scrambled when asked for (extension: the reference's Scramble
 * is notImplemented, ScrambledSobolSampler.cpp:51-53). */
float or_sobol_sample_scrambled(uint64_t index, uint32_t dim, uint32_t scramble, uint32_t seed) {
    uint32_t v = 0;
    for (uint32_t i = dim * PB2_SOBOL_MATRIX_SIZE; index; index >>= 1, i++)
        if (index & 1) v ^= pb2_sobol_matrices32[i];
    if (scramble) v = pb2_owen_scramble(v, pb2_owen_dim_seed(seed, dim));
    return (float)v * 0x1p-32f;
}

static inline real next_sample(path_ctx* c) {
    if (c->dim >= PB2_SOBOL_DIMS) { c->overflow = 1; return 0.5f; }
    const uint32_t d = c->dim++;
    return or_sobol_sample_scrambled(c->index, d, c->scramble, c->seed);
}

/* The two uniform numbers of piperSurfaceSample / piperLightSample are the two `piperSample(context)`
 * arguments of one call (Tracer/Embree/Kernel.cpp:117, 145); the compiler evaluates them right to left,
 * so u2 takes the lower dimension. */
static inline void next_pair(path_ctx* c, real* u1, real* u2) {
    *u2 = next_sample(c);
    *u1 = next_sample(c);
}

static inline real power_heuristic(real a, real b) {
    const real sp1 = a * a;
    const real sp2 = b * b;
    return sp1 / (sp1 + sp2);
}

static spec mis(path_ctx* c, v3 hit, const bsdf* b, v3 wo, const surf_info* si, v3 ng_sh) {
    const or_scene* s = c->s;
    /* uniformSelect (BasicLight/Kernel.cpp:91-98): lights[0] = environment, then the area lights */
    const uint32_t count = 1 + s->nlight;
    const real u = next_sample(c);
    uint32_t sel = (uint32_t)R_FLOOR(u * (real)count);
    if (sel > count - 1) sel = count - 1;
    const real sel_pdf = 1.0f / (real)count;
    const int delta = 0;
    if (sel_pdf <= 0.0f) return SP_ZERO;

    spec part_a = SP_ZERO;
    {
        light_sample ls;
        real u1, u2;
        next_pair(c, &u1, &u2);
        if (sel == 0) env_sample(s, u1, u2, &ls);
        else area_sample(s, sel - 1, hit, u1, u2, &ls);
        if (ls.pdf > 0.0f && sp_valid(ls.rad)) {
            const v3 wi = to_shading(si, ls.dir);
            const spec f = bsdf_eval(b, wo, wi, ng_sh, PART_NO_SPECULAR);
            if (sp_valid(f)) {
                if (!occluded(s, hit, ls.dir, R_FMIN(1e-3f, ls.distance), ls.distance, &c->shadow_rays)) {
                    real w = R_FABS(wi.z) / ls.pdf;
                    if (!delta) {
                        const real bp = bsdf_pdf(b, wo, wi, PART_NO_SPECULAR);
                        w = w * power_heuristic(ls.pdf, bp);
                    }
                    part_a = sp_muls(sp_mul(f, ls.rad), w);
                }
            }
        }
    }
    spec part_b = SP_ZERO;
    if (!delta) {
        bsdf_sample bs;
        real u1, u2;
        next_pair(c, &u1, &u2);
        bsdf_sample_fn(b, u1, u2, wo, ng_sh, PART_NO_SPECULAR, &bs);
        if (bs.pdf > 0.0f && sp_valid(bs.f)) {
            real weight = R_FABS(bs.wi.z) / bs.pdf;
            const v3 dir = to_local(si, bs.wi);
            surf_info hs;
            trace_surface(s, hit, dir, 1e-3f, 1e5f, &hs, &c->closest_rays);
            const int is_sel_light = hs.kind == KIND_AREA_LIGHT && sel != 0 && hs.light == sel - 1;
            if (is_sel_light || hs.kind == KIND_MISSING) {
                spec rad;
                real pdf;
                if (hs.kind == KIND_MISSING) {
                    rad = s->env;
                    pdf = sp_valid(rad) ? env_pdf(dir) : 0.0f;
                } else {
                    const or_light* L = &s->lights[hs.light];
                    /* diffuseEvaluate / diffusePdf (AreaLight/Kernel.cpp:43-55) */
                    rad = dot3(hs.N, dir) < 0.0f ? L->radiance : SP_ZERO;
                    pdf = hs.t * hs.t / (R_FABS(dot3(hs.N, dir)) * L->area);
                }
                if (sp_valid(rad) && pdf > 0.0f) {
                    weight = weight * power_heuristic(bs.pdf, pdf);
                    part_b = sp_muls(sp_mul(rad, bs.f), weight);
                }
            }
        }
    }
    return sp_divs(sp_add(part_a, part_b), sel_pdf);
}

static spec trace_path(path_ctx* c, const pb2_render_settings* st, v3 o, v3 d, uint32_t* depth_out) {
    const or_scene* s = c->s;
    spec pf = mksp(1.0f, 1.0f, 1.0f);
    spec sample = SP_ZERO;
    int specular = 1;
    uint32_t depth = 0;
    for (;;) {
        surf_info si;
        trace_surface(s, o, d, 1e-3f, 1e5f, &si, &c->closest_rays);
        if (specular && (si.kind == KIND_AREA_LIGHT || si.kind == KIND_MISSING)) {
            spec rad;
            if (si.kind == KIND_AREA_LIGHT) {
                const v3 delta = mul3s(d, si.t);
                const v3 wi = normalize3(delta);
                rad = dot3(si.N, wi) < 0.0f ? s->lights[si.light].radiance : SP_ZERO;
            } else {
                rad = s->env;
            }
            sample = sp_add(sample, sp_mul(pf, rad));
        }
        if (si.kind == KIND_AREA_LIGHT) {
            --depth;
            o = add3(o, mul3s(d, si.t + 0.001f));
            continue;
        }
        if (si.kind == KIND_MISSING || depth >= st->max_depth) break;

        const v3 wo = to_shading(&si, neg3(d));
        const v3 ng_sh = to_shading(&si, si.Ng);
        bsdf b;
        bsdf_init(s, si.material, si.front, si.tu, si.tv, &b);
        const v3 hit = add3(o, mul3s(d, si.t));
        if (b.no_specular) sample = sp_add(sample, sp_mul(pf, mis(c, hit, &b, wo, &si, ng_sh)));
        bsdf_sample ss;
        real u1, u2;
        next_pair(c, &u1, &u2);
        bsdf_sample_fn(&b, u1, u2, wo, ng_sh, PART_ALL, &ss);
        if (!(ss.pdf > 0.0f && sp_valid(ss.f))) break;
        pf = sp_muls(sp_mul(pf, ss.f), R_FABS(ss.wi.z) / ss.pdf);
        if (depth > st->min_rr_depth) {
            const real p = R_FMAX(0.05f, 1.0f - R_FMAX(pf.r, R_FMAX(pf.g, pf.b)));
            if (next_sample(c) < p) break;
            pf = sp_divs(pf, 1.0f - p);
        }
        d = to_local(&si, ss.wi);
        o = add3(hit, mul3s(si.Ng, (ss.part & PART_R) ? 0.001f : -0.001f));
        specular = (ss.part & PART_SPECULAR) != 0;
        ++depth;
    }
    *depth_out = depth;
    return sample;
}

/* accumulate + filters (Src/BuiltinComponent/RenderDriver/FixedSampler/Kernel.cpp:30-69) */
static real filter_weight(const pb2_render_settings* st, real dx, real dy) {
    switch (st->filter) {
        case PB2_FILTER_TRIANGLE:
            return R_FMAX(0.0f, 1.0f - R_FABS(dx)) * R_FMAX(0.0f, 1.0f - R_FABS(dy));
        case PB2_FILTER_GAUSSIAN: {
            const real neg_alpha = -st->gaussian_alpha;
            const real sub = R_EXP(-st->gaussian_alpha); /* host: FixedSampler.cpp:43 */
            const real wx = R_FMAX(R_PEXP(neg_alpha * dx * dx) - sub, 0.0f);
            const real wy = R_FMAX(R_PEXP(neg_alpha * dy * dy) - sub, 0.0f);
            return wx * wy;
        }
        default:
            return 1.0f;
    }
}

static void splat(const pb2_render_settings* st, float* rgbw, float px, float py, spec v) {
    const int32_t bx = (int32_t)(px - 0.5f), by = (int32_t)(py - 0.5f);
    const int32_t xs[4] = { bx, bx + 1, bx, bx + 1 };
    const int32_t ys[4] = { by, by, by + 1, by + 1 };
    for (int k = 0; k < 4; ++k) {
        const uint32_t x = (uint32_t)xs[k], y = (uint32_t)ys[k];
        if (!(x < st->width && y < st->height)) continue;
        const real w = filter_weight(st, px - ((float)x + 0.5f), py - ((float)y + 0.5f));
        float* p = rgbw + 4 * ((size_t)x + (size_t)y * st->width);
        p[0] += (float)(v.r * w);
        p[1] += (float)(v.g * w);
        p[2] += (float)(v.b * w);
        p[3] += (float)w;
    }
}

/* BxDF of scene material `mat` (shading frame, geometric normal +z) for checks of its sampler:
 * n samples (u pairs in u[2i], u[2i+1]) -> wi (3n), f (3n), pdf (n; 0 where the sample was rejected). */
void or_bsdf_sample(const or_scene* s, uint32_t mat, int front, const float wo_in[3], uint32_t n, const float* u,
                    float* wi, float* f, float* pdf) {
    bsdf b;
    bsdf_init(s, mat, front, 0.0f, 0.0f, &b);
    const v3 wo = mk3(wo_in[0], wo_in[1], wo_in[2]);
    const v3 ng = mk3(0.0f, 0.0f, 1.0f);
    for (uint32_t i = 0; i < n; ++i) {
        bsdf_sample r;
        memset(&r, 0, sizeof(r));
        bsdf_sample_fn(&b, u[2 * i], u[2 * i + 1], wo, ng, PART_ALL, &r);
        wi[3 * i] = r.wi.x; wi[3 * i + 1] = r.wi.y; wi[3 * i + 2] = r.wi.z;
        f[3 * i] = r.f.r; f[3 * i + 1] = r.f.g; f[3 * i + 2] = r.f.b;
        pdf[i] = r.pdf;
    }
}

/* The same BxDF's value and pdf at n given directions. */
void or_bsdf_eval(const or_scene* s, uint32_t mat, int front, const float wo_in[3], uint32_t n, const float* wi,
                  float* f, float* pdf) {
    bsdf b;
    bsdf_init(s, mat, front, 0.0f, 0.0f, &b);
    const v3 wo = mk3(wo_in[0], wo_in[1], wo_in[2]);
    const v3 ng = mk3(0.0f, 0.0f, 1.0f);
    for (uint32_t i = 0; i < n; ++i) {
        const v3 w = mk3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        const spec v = bsdf_eval(&b, wo, w, ng, PART_ALL);
        f[3 * i] = v.r; f[3 * i + 1] = v.g; f[3 * i + 2] = v.b;
        pdf[i] = bsdf_pdf(&b, wo, w, PART_ALL);
    }
}

/* Frame set-up shared by the render entry points: the render rect and NDC transform (calcRenderRECT)
 * and the Sobol resolution (ScrambledSobolSampler.cpp:66-72). */
typedef struct frame_ctx {
    pb2_ndc_transform tr;
    pb2_rect full;
    uint32_t res, log2res;
} frame_ctx;

static int frame_setup(const pb2_render_settings* st, frame_ctx* f) {
    if (st->scramble > 1) return -1;
    if (5u + 8u * (uint64_t)st->max_depth > PB2_SOBOL_DIMS) return -2;
    const float dev_aspect = st->camera.sensor_size[0] / st->camera.sensor_size[1];
    or_calc_render_rect(st->width, st->height, dev_aspect, st->fit_mode, &f->tr, &f->full);
    const uint32_t mx = f->full.width > f->full.height ? f->full.width : f->full.height;
    f->log2res = (uint32_t)ceil(log2((double)mx));
    f->res = 1u << f->log2res;
    return 0;
}

/* Film position of sample `sidx` of the pixel at (sx, sy) inside the render rect (sobolStart), and
 * its Sobol index. */
static void sample_point(const pb2_render_settings* st, const frame_ctx* f, uint32_t sx, uint32_t sy, uint32_t sidx,
                         uint64_t* index, float* px, float* py) {
    float off[2];
    or_sobol_start(f->res, f->log2res, sx, sy, sidx, index, off);
    (void)st;
    *px = off[0] + (float)(f->full.left + sx);
    *py = off[1] + (float)(f->full.top + sy);
}

/* One sample: piperMain (Tracer/Embree/Kernel.cpp:47-99) from the sample point to the path radiance. */
static spec render_sample(const or_scene* s, const pb2_render_settings* st, const frame_ctx* f, uint64_t index,
                          float px, float py, int* overflow) {
    path_ctx c;
    memset(&c, 0, sizeof(c));
    c.s = s;
    c.dim = 5;
    c.index = index;
    c.scramble = st->scramble;
    c.seed = st->scramble_seed;
    const real ndc_x = f->tr.ox + f->tr.sx * px / (real)st->width;
    const real ndc_y = f->tr.oy + f->tr.sy * py / (real)st->height;
    const real u1 = or_sobol_sample_scrambled(c.index, 3, st->scramble, st->scramble_seed);
    const real u2 = or_sobol_sample_scrambled(c.index, 4, st->scramble, st->scramble_seed);
    v3 o, d;
    camera_ray(&st->camera, ndc_x, ndc_y, u1, u2, &o, &d);
    uint32_t depth;
    const spec v = trace_path(&c, st, o, d, &depth);
    *overflow |= c.overflow;
    return v;
}

int or_render(const or_scene* s, const pb2_render_settings* st, const pb2_rect* rect, uint32_t sample_begin,
              uint32_t sample_count, float* rgbw, float* sample_out, int threads) {
    frame_ctx f;
    const int rc = frame_setup(st, &f);
    if (rc) return rc;
    const size_t nsamp = (size_t)rect->width * rect->height * sample_count;
    float* out = sample_out ? sample_out : (float*)malloc(sizeof(float) * 5 * (nsamp ? nsamp : 1));
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1) reduction(| : overflow)
    for (int64_t row = 0; row < (int64_t)rect->height; ++row) {
        for (uint32_t col = 0; col < rect->width; ++col) {
            for (uint32_t k = 0; k < sample_count; ++k) {
                const uint32_t sx = rect->left + col - f.full.left;
                const uint32_t sy = rect->top + (uint32_t)row - f.full.top;
                uint64_t index;
                float px, py;
                sample_point(st, &f, sx, sy, sample_begin + k, &index, &px, &py);
                const spec v = render_sample(s, st, &f, index, px, py, &overflow);
                float* o = out + 5 * (((size_t)row * rect->width + col) * sample_count + k);
                o[0] = px; o[1] = py; o[2] = (float)v.r; o[3] = (float)v.g; o[4] = (float)v.b;
            }
        }
    }
    if (rgbw) {
        for (size_t i = 0; i < nsamp; ++i) {
            const float* o = out + 5 * i;
            splat(st, rgbw, o[0], o[1], mksp(o[2], o[3], o[4]));
        }
    }
    if (!sample_out) free(out);
    return overflow ? -3 : 0;
}

/* Resolved film value (radiance / weight, the resolve of FixedSampler.cpp:122-131) of chosen pixels
 * over samples [sample_begin, sample_begin + sample_count), accumulated in double.  A pixel receives
 * the splats of its own samples and of the samples of its eight neighbours whose 2x2 footprint covers
 * it; each candidate sample's film position is computed first and only the samples that reach the
 * pixel are traced, about four pixels' worth per pixel.  pixels: npix (x, y) pairs in film
 * coordinates; out: npix x 4 (r, g, b, weight sum).  Pixels run in parallel. */
int or_render_pixels(const or_scene* s, const pb2_render_settings* st, const uint32_t* pixels, uint32_t npix,
                     uint32_t sample_begin, uint32_t sample_count, double* out, int threads) {
    frame_ctx f;
    const int rc = frame_setup(st, &f);
    if (rc) return rc;
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1) reduction(| : overflow)
    for (int64_t i = 0; i < (int64_t)npix; ++i) {
        const int64_t tx = pixels[2 * i], ty = pixels[2 * i + 1];
        double acc[4] = { 0.0, 0.0, 0.0, 0.0 };
        for (int64_t ny = ty - 1; ny <= ty + 1; ++ny) {
            for (int64_t nx = tx - 1; nx <= tx + 1; ++nx) {
                if (nx < (int64_t)f.full.left || ny < (int64_t)f.full.top ||
                    nx >= (int64_t)f.full.left + f.full.width || ny >= (int64_t)f.full.top + f.full.height)
                    continue;
                for (uint32_t k = 0; k < sample_count; ++k) {
                    uint64_t index;
                    float px, py;
                    sample_point(st, &f, (uint32_t)(nx - f.full.left), (uint32_t)(ny - f.full.top), sample_begin + k,
                                 &index, &px, &py);
                    const int32_t bx = (int32_t)(px - 0.5f), by = (int32_t)(py - 0.5f);
                    if (!((tx == bx || tx == bx + 1) && (ty == by || ty == by + 1))) continue;
                    const real w = filter_weight(st, px - ((float)tx + 0.5f), py - ((float)ty + 0.5f));
                    const spec v = render_sample(s, st, &f, index, px, py, &overflow);
                    acc[0] += (double)(v.r * w);
                    acc[1] += (double)(v.g * w);
                    acc[2] += (double)(v.b * w);
                    acc[3] += (double)w;
                }
            }
        }
        for (int c = 0; c < 4; ++c) out[4 * i + c] = acc[c];
    }
    return overflow ? -3 : 0;
}

/* conv (Src/Test/conv.hpp:22-37): z[idx] = sum over the kernel window inside the image of x * y, accumulated in
 * float in the reference's loop order (i over x offsets, then j over y offsets). */
void or_conv(const float* x, const float* y, float* z, uint32_t width, uint32_t height, uint32_t kernel_size) {
    const uint32_t half = kernel_size / 2;
    const uint32_t count = width * height;
    for (uint32_t idx = 0; idx < count; ++idx) {
        const uint32_t py = idx / width, px = idx % width;
        float res = 0.0f;
        for (int32_t i = 0; i < (int32_t)kernel_size; ++i) {
            const int32_t nx = (int32_t)(px + (uint32_t)i - half);
            if (nx >= 0 && nx < (int32_t)width)
                for (int32_t j = 0; j < (int32_t)kernel_size; ++j) {
                    const int32_t ny = (int32_t)(py + (uint32_t)j - half);
                    if (ny >= 0 && ny < (int32_t)height) res += x[ny * (int32_t)width + nx] * y[i * (int32_t)kernel_size + j];
                }
        }
        z[idx] = res;
    }
}
