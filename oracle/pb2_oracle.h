/*
 * pb2_oracle.h -- CPU oracle for the Piper2 render path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline call it to produce the expected results the CUDA library is compared against.  Nothing in
 * the product (piper2_b200/) links or calls it.
 *
 * It restates, in plain C, the reference's device code for the path Sobol sample -> camera ray ->
 * traversal -> BxDF / NEE + MIS -> film (each function cites the reference file:line it follows) and
 * replaces Embree's traversal with a watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013)
 * over brute force or a binned-SAH BVH.  It shares two things with the product by design: the
 * elementary-function definitions (piper2_b200/csrc/pb2_math.h) and the generated Sobol tables; both
 * are pinned separately by tests.
 */
#ifndef PB2_ORACLE_H
#define PB2_ORACLE_H
#include <stdint.h>
#include "../include/piper2_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_scene or_scene;

float or_sobol_sample(uint64_t index, uint32_t dim);
/* Dimension `dim` of a sample with optional Owen scrambling (scramble = 1, extension). */
float or_sobol_sample_scrambled(uint64_t index, uint32_t dim, uint32_t scramble, uint32_t seed);
uint64_t or_sobol_interval_to_index(uint32_t m, uint32_t sample, uint32_t px, uint32_t py);
void or_sobol_start(uint32_t resolution, uint32_t log2_resolution, uint32_t px, uint32_t py,
                    uint32_t sample, uint64_t* index, float offset[2]);
const char* or_sobol_digest(void);

float or_remap_roughness(float roughness);
/* pb2_logf and the per-point roughness remap of a textured roughness (checks of the shared math) */
float or_logf(float x);
float or_remap_roughness_point(float roughness);
/* A texture's value at (tu, tv): CheckBoard or the bilinear SampledTexture, out[0..channel). */
void or_texture_sample(const pb2_texture* t, float tu, float tv, float* out);
void or_camera_ray(const pb2_camera* cam, float ndc_x, float ndc_y, float u1, float u2, pb2_ray* ray);

/* Scene: flattens meshes (translation baked in) and builds a BVH if use_bvh != 0. */
or_scene* or_scene_create(const pb2_scene* scene, int use_bvh);
void or_scene_destroy(or_scene* s);
uint32_t or_scene_triangle_count(const or_scene* s);

/* Watertight test of one triangle; returns 1 and writes t, u, v on a hit in (tmin, tmax). */
int or_intersect_triangle(const float ray[8], const float v0[3], const float v1[3], const float v2[3],
                          float* t, float* u, float* v);

/* Batch traversal: closest hit over triangles + planes, and any hit over triangles. */
void or_trace_closest(const or_scene* s, const pb2_ray* rays, uint32_t n, pb2_hit* hits, int threads);
void or_trace_any(const or_scene* s, const pb2_ray* rays, uint32_t n, uint32_t* occluded, int threads);
/* Work counters of the BVH traversal (node visits, triangle tests) for the byte model. */
void or_trace_counters(const or_scene* s, const pb2_ray* rays, uint32_t n, int closest,
                       uint64_t* node_visits, uint64_t* tri_tests);

/* Single-ray triangle queries used by the reference harness in oracle/ref (triangles only). */
int or_closest_triangle(const or_scene* s, const pb2_ray* ray, pb2_hit* hit);
int or_any_triangle(const or_scene* s, const pb2_ray* ray);
const float* or_triangle_vertices(const or_scene* s, uint32_t prim);

/* Renders samples [sample_begin, sample_begin + sample_count) of `rect` into rgbw (W*H*4) and, if
 * sample_out != NULL, the per-sample (point.x, point.y, r, g, b) in (y, x, sample) order.
 * Returns 0, or a negative value if the settings are not supported. */
int or_render(const or_scene* s, const pb2_render_settings* settings, const pb2_rect* rect,
              uint32_t sample_begin, uint32_t sample_count, float* rgbw, float* sample_out, int threads);
/* Resolved film value of chosen pixels: for each (x, y) in `pixels` (npix pairs), the sums of
 * radiance x filter weight (r, g, b) and of the weights over every sample of samples
 * [sample_begin, sample_begin + sample_count) whose splat reaches the pixel, accumulated in double
 * (out: npix x 4).  In liboracle_fp64.so (built with -DOR_FP64) every path is computed in double:
 * the ground truth of the error measurements. */
int or_render_pixels(const or_scene* s, const pb2_render_settings* settings, const uint32_t* pixels,
                     uint32_t npix, uint32_t sample_begin, uint32_t sample_count, double* out, int threads);
void or_calc_render_rect(uint32_t width, uint32_t height, float device_aspect, uint32_t fit_mode,
                         pb2_ndc_transform* transform, pb2_rect* rect);
void or_plane_make(const float origin[3], const float u[3], const float v[3], pb2_plane* out);
/* BxDF of scene material `mat` in its shading frame (geometric normal +z): sampling and evaluation. */
void or_bsdf_sample(const or_scene* s, uint32_t mat, int front, const float wo[3], uint32_t n, const float* u,
                    float* wi, float* f, float* pdf);
void or_bsdf_eval(const or_scene* s, uint32_t mat, int front, const float wo[3], uint32_t n, const float* wi,
                  float* f, float* pdf);

/* The Accelerator test's convolution kernel (Src/Test/conv.hpp:22-37), every output of a width x height image
 * (the CPU loop of Src/Test/Accelerator-Test.cpp:79-81). */
void or_conv(const float* x, const float* y, float* z, uint32_t width, uint32_t height, uint32_t kernel_size);

#ifdef __cplusplus
}
#endif
#endif
