// render.cu -- the render pipeline: Sobol sampler, camera, wavefront path tracer, film.
//
// One launch renders `sample_count` samples of every pixel of a rectangle.  Each (pixel, sample) is a
// path with SoA state in device memory.  A bounce is a fixed sequence of kernels over index queues:
//   extend (closest hit of every active path) -> classify (emission, area-light pass-through, miss,
//   depth limit; surface hits go to one queue per material type) -> shade<material> (NEE light
//   sample + shadow ray, MIS BSDF sample + ray, continuation sample, Russian roulette) -> shadow
//   (any hit) and MIS (closest hit) traces -> finish (adds the MIS estimate, re-queues or splats).
// All per-path arithmetic is the reference's (PathTracing/Kernel.cpp:23-193) in its operation order,
// so each path's radiance equals the CPU oracle's bit for bit; only the film sums, which use
// atomics in any order (as the reference's CAS loop does), differ in rounding.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "guiding.cuh"
#include "guiding_tc.cuh"
#include "pb2_internal.h"
#include "shading.cuh"
#include "traverse.cuh"

#define PB2_SOBOL_STORAGE static __device__ const
#include "sobol_tables.h"

namespace pb2 {

__device__ __forceinline__ uint32_t sobol_bits(uint64_t index, uint32_t dim) {
    uint32_t v = 0;
    for (uint32_t i = dim * PB2_SOBOL_MATRIX_SIZE; index; index >>= 1, i++)
        if (index & 1) v ^= __ldg(&pb2_sobol_matrices32[i]);
    return v;
}
__device__ __forceinline__ float sobol_sample(uint64_t index, uint32_t dim) {
    return (float)sobol_bits(index, dim) * 0x1p-32f;
}

// Byte tables of the generator matrices for the render kernels: entry [d][k][b] is the XOR of the columns
// 8k + j of dimension d over the set bits j of b (the same column index d * 52 + 8k + j that the bitwise
// loop above reads), so a sample is the XOR of one entry per byte of its index instead of one column per
// set bit.  XOR is associative, so the value is the same bit for bit.  Filled by k_sobol_byte_tables when
// a pipeline is created (every GPU that loads the library holds the 7 MiB until exit).
constexpr uint32_t kSobolIndexBytes = 7;  // indices below 2^56 (a render's indices stay below 2^53)
static __device__ uint32_t g_sobol_bytes[PB2_SOBOL_DIMS * kSobolIndexBytes * 256];

__global__ void k_sobol_byte_tables() {
    constexpr uint32_t kColumns = PB2_SOBOL_DIMS * PB2_SOBOL_MATRIX_SIZE;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < PB2_SOBOL_DIMS * kSobolIndexBytes * 256;
         e += gridDim.x * blockDim.x) {
        const uint32_t b = e & 255u, k = (e >> 8) % kSobolIndexBytes, d = (e >> 8) / kSobolIndexBytes;
        uint32_t v = 0;
        for (uint32_t j = 0; j < 8; ++j) {
            const uint32_t col = d * PB2_SOBOL_MATRIX_SIZE + 8 * k + j;
            if (((b >> j) & 1u) && col < kColumns) v ^= pb2_sobol_matrices32[col];
        }
        g_sobol_bytes[e] = v;
    }
}

__device__ __forceinline__ uint32_t sobol_bits_bytes(uint64_t index, uint32_t dim) {
    const uint32_t* t = g_sobol_bytes + (size_t)dim * (kSobolIndexBytes * 256);
    uint32_t v = 0;
    for (uint32_t k = 0; index && k < kSobolIndexBytes; ++k, index >>= 8, t += 256) v ^= __ldg(t + (index & 0xFFu));
    return v;
}
__device__ __forceinline__ float sobol_sample_fast(uint64_t index, uint32_t dim) {
    return (float)sobol_bits_bytes(index, dim) * 0x1p-32f;
}
// A dimension >= 2 of a launch, Owen-scrambled when the settings ask for it (extension; see pb2_math.h).
__device__ __forceinline__ float sobol_sample_s(uint64_t index, uint32_t dim, uint32_t scramble, uint32_t seed) {
    uint32_t v = sobol_bits_bytes(index, dim);
    if (scramble) v = pb2_owen_scramble(v, pb2_owen_dim_seed(seed, dim));
    return (float)v * 0x1p-32f;
}

__device__ __forceinline__ uint64_t sobol_interval_to_index(uint32_t m, uint32_t sample, uint32_t px, uint32_t py) {
    if (m == 0) return 0;
    const uint32_t m2 = m << 1;
    uint64_t index = (uint64_t)sample << m2;
    uint64_t delta = 0;
    for (int c = 0; sample; sample >>= 1, ++c)
        if (sample & 1) delta ^= __ldg(&pb2_vdc_sobol_matrices[m - 1][c]);
    uint64_t b = (((uint64_t)px << m) | py) ^ delta;
    for (int c = 0; b; b >>= 1, ++c)
        if (b & 1) index ^= __ldg(&pb2_vdc_sobol_matrices_inv[m - 1][c]);
    return index;
}

__global__ void k_sobol_generate(const uint64_t* __restrict__ idx, const uint32_t* __restrict__ dim, uint32_t n,
                                 float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = dim[i] < PB2_SOBOL_DIMS ? sobol_sample(idx[i], dim[i]) : 0.0f;
}

__global__ void k_sobol_start(uint32_t log2res, const uint32_t* __restrict__ pxs, uint32_t n, uint64_t* __restrict__ idx,
                              float* __restrict__ off) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t px = pxs[3 * i], py = pxs[3 * i + 1], s = pxs[3 * i + 2];
    const uint64_t id = sobol_interval_to_index(log2res, s, px, py);
    const float res = (float)(1u << log2res);
    idx[i] = id;
    off[2 * i] = fminf(fmaxf(sobol_sample(id, 0) * res - (float)px, 0.0f), 1.0f);
    off[2 * i + 1] = fminf(fmaxf(sobol_sample(id, 1) * res - (float)py, 0.0f), 1.0f);
}

// ---- pipeline state ------------------------------------------------------------------------------

struct DevLight {
    float radiance[3];
    uint32_t first_plane, plane_count;
    float area, inverse_area;
    float translation[3];
};

constexpr int kNumSurfaceTypes = 7;

// Counter slots in Paths::counts
enum : int {
    C_EXT_CUR = 0, C_EXT_NEXT = 1, C_SHADOW = 2, C_MIS = 3, C_SHADED = 4, C_SURF0 = 5,  // 5..11 per type
    C_GUIDE = 12,  // vertices whose continuation samples the guide (guided launches)
    C_STAT_CLOSEST = 16, C_STAT_SHADOW = 18, C_STAT_VERTICES = 20, C_ERROR = 24,
    C_CHECK = 25,  // 25..28: first failed index check (code, kernel, slot, value)
    C_FREE = 29,   // refilled and batched launches: free slots (their bits are set in the free bitmap)
    C_TC_ERROR = 31,  // a tensor-core wait of the guide inference timed out
    C_COUNT = 32
};

struct Paths {
    float4* o;       // ray origin
    float4* d;       // ray direction
    float4* pf;      // throughput rgb, w = specular flag (0/1)
    float4* rad;     // radiance rgb
    unsigned long long* sidx;
    uint32_t* dim;
    uint32_t* depth;
    float2* point;
    float4* hit;     // t, prim, u, v (prim = PB2_INVALID_PRIM on a miss)
    uint32_t* hit_slot;
    // pending next-event estimation and MIS-BSDF sample of the current vertex
    float4* mis_pf;    // pf at the vertex, w = 1 / select pdf... stored as the pdf itself
    float4* nee;       // candidate light contribution (f * rad * w), w = 1 if a shadow ray was queued
    float4* sh_o;      // shadow ray origin, w = tmin
    float4* sh_d;      // shadow ray direction, w = tmax
    float4* mr_o;      // MIS ray origin
    float4* mr_d;      // MIS ray direction
    float4* mr_f;      // sampled f, w = |wi.z| / pdf
    float2* mr_pdf;    // x = bsdf pdf, y = selected light (as uint bits; 0 = environment)
    uint32_t* flags;   // bit0 = has MIS, bit1 = continue, bit2 = MIS ray queued
    uint32_t* occ;
    float4* mhit;
    // queues
    uint32_t* ext[2];
    uint32_t* surf[kNumSurfaceTypes];
    uint32_t* shadow_q;
    uint32_t* mis_q;
    uint32_t* shaded_q;
    uint32_t* guide_q;  // slots of the vertices the guide is evaluated for (guided launches)
    uint32_t* counts;  // C_COUNT entries
    // refilled and batched launches: the path index or scene of each slot; the free slots as a bitmap (one bit per
    // slot), with the per-word exclusive prefix of the free bits within 1024-word blocks and the blocks' prefix, so
    // that a claim takes the lowest free slots in slot order
    uint32_t* scene;
    uint32_t* free_bits;
    uint32_t* free_scan;
    uint32_t* free_block;
};

struct LaunchParams {
    pb2_rect rect;        // launch rectangle
    pb2_rect full;        // full render rectangle
    pb2_ndc_transform ndc;
    uint32_t width, height;
    uint32_t log2res;
    uint32_t sample_begin, sample_count;
    uint32_t max_depth, min_rr_depth;
    uint32_t filter;
    float gauss_neg_alpha, gauss_sub;
    pb2_camera cam;
    uint32_t num_lights;  // area lights
    float env[3];
    uint32_t path_count;  // path slots of a single-scene launch (its capacity)
    uint32_t refill;      // 1: the launch has more paths than slots, finished paths free their slots
    uint32_t checks;      // PB2_DEBUG_CHECKS: verify indices, record the first violation, skip the path
    uint32_t scramble, scramble_seed;  // Owen scrambling of dimensions >= 2 (extension)
};

struct SceneView {
    const DevMaterial* materials;
    const DevTexture* textures;
    const float2* tri_uv;  // texture coordinates of each primitive's three vertices (index order), if textured
    const uint32_t* prim_material;
    const DevLight* lights;
    const float* plane_cdf;
    const float* plane_pdf;
    BvhView bvh;
    uint32_t material_count;
};

// Guided sampling state of a launch (all pointers device memory, indexed by path slot unless noted).
constexpr int kMaxRecords = 3;  // pending training records per path (its first guided vertices)
constexpr uint32_t kMaxCells = 16 * 16 * 16;  // spatial cells of the training-weight normalisation
struct GuideState {
    uint32_t enabled;
    float sel_prob;
    GuideView net;
    float* mix;             // 40 floats per slot: lobe weights [8], means [8][3], concentrations [8]
    float4* rec;            // record r of slot s, word k: rec[(r * 5 + k) * cap + s]
    uint32_t* nrec;
    uint32_t cap;
    float* train;           // training records, 16 floats each
    uint32_t* train_count;  // [0] written, [1] offered
    uint32_t train_capacity;
    float accept_prob;
    uint32_t salt;
    float bmin[3], binv[3];
    uint32_t types;         // bit t set: vertices of surface type t sample the guide
    uint32_t max_depth;     // only vertices at path depth < max_depth sample the guide
    float* dump;            // optional (pb2_pipeline_set_guide_dump): kGuideDumpFloats per inferred vertex
    uint32_t* dump_count;
    uint32_t dump_cap;
};
// A dumped row: the vertex's 9 input features (position in the unit box, normal, outgoing direction), then
// its 40 mixture parameters in the layout of GuideState::mix, 3 floats of padding.
constexpr uint32_t kGuideDumpFloats = 52;

// Whether a surface vertex of type `type` at path depth `depth` samples the guide (classification and
// shading must agree: the guide is evaluated exactly for these vertices).
__device__ __forceinline__ bool guide_vertex(const GuideState& gs, uint32_t type, uint32_t depth) {
    return gs.enabled && ((gs.types >> type) & 1u) && depth < gs.max_depth;
}

// Where a kernel finds the launch parameters, scene and film of a path slot.
// One scene per launch: everything is a kernel parameter.
struct SingleCtx {
    static constexpr bool kBatch = false;
    LaunchParams lp;
    SceneView sv;
    float4* film;
    float* sample_out;
    __device__ __forceinline__ const LaunchParams& P(uint32_t) const { return lp; }
    __device__ __forceinline__ const SceneView& S(uint32_t) const { return sv; }
    __device__ __forceinline__ const BvhView& bvh(uint32_t) const { return sv.bvh; }
    __device__ __forceinline__ float4* film_of(uint32_t) const { return film; }
    __device__ __forceinline__ uint32_t capacity() const { return lp.path_count; }
    __device__ __forceinline__ bool checks() const { return lp.checks != 0u; }
};

// Many scenes per launch: each slot carries its scene; the scene table is in device memory.
struct BatchScene {
    LaunchParams lp;      // rect = full frame, sample_begin 0, sample_count = the scene's spp
    SceneView sv;
    float4* film;
    uint64_t path_begin;  // first global path index of the scene
    uint64_t path_count;  // width x height x spp
};
struct BatchState {
    unsigned long long next;   // next global path index to generate
    unsigned long long total;  // sum of the scenes' path counts
    unsigned long long claim_begin;
    uint32_t claim_count;
    uint32_t claim_base;       // extend-queue position of the first regenerated path
    unsigned long long t_start;
};
struct BatchCtx {
    static constexpr bool kBatch = true;
    const BatchScene* scenes;
    uint32_t scene_count;
    uint32_t cap;
    uint32_t check;
    uint32_t* remaining;          // per scene: paths not yet splatted
    unsigned long long* done_ns;  // per scene: %globaltimer when its last path was splatted
    BatchState* state;
    const uint32_t* scene_of;     // = Paths::scene
    __device__ __forceinline__ const BatchScene& B(uint32_t slot) const { return scenes[scene_of[slot]]; }
    __device__ __forceinline__ const LaunchParams& P(uint32_t slot) const { return B(slot).lp; }
    __device__ __forceinline__ const SceneView& S(uint32_t slot) const { return B(slot).sv; }
    __device__ __forceinline__ const BvhView& bvh(uint32_t slot) const { return B(slot).sv.bvh; }
    __device__ __forceinline__ float4* film_of(uint32_t slot) const { return B(slot).film; }
    __device__ __forceinline__ uint32_t capacity() const { return cap; }
    __device__ __forceinline__ bool checks() const { return check != 0u; }
};

// ---- helpers ----------------------------------------------------------------------------------------

// Warp-aggregated queue append: the active lanes that push to the same counter (lanes may push to
// different queues, e.g. one per material type) share one atomic.
__device__ __forceinline__ uint32_t warp_push(uint32_t* counter) {
    const unsigned mask = __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(counter));
    const int leader = __ffs(mask) - 1;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Adds the active lanes' v to a 64-bit counter with one atomic per warp (any subset of lanes may call it).
__device__ __forceinline__ void warp_count(unsigned long long* counter, uint32_t v) {
    const unsigned mask = __activemask();
    const uint32_t sum = __reduce_add_sync(mask, v);
    if ((int)(threadIdx.x & 31u) == __ffs(mask) - 1) atomicAdd(counter, (unsigned long long)sum);
}

// Debug index checks (LaunchParams::checks): the first failure is recorded and the access skipped.
enum CheckKernel : uint32_t { K_CLASSIFY = 1, K_SHADE = 2, K_FINISH = 3 };
__device__ __noinline__ void check_failed(uint32_t* counts, uint32_t code, uint32_t kernel, uint32_t slot, uint32_t v) {
    if (atomicCAS(&counts[C_CHECK], 0u, code) == 0u) {
        counts[C_CHECK + 1] = kernel;
        counts[C_CHECK + 2] = slot;
        counts[C_CHECK + 3] = v;
    }
}
#define PB2_CHECK(cond, code, kernel, slot, v)                              \
    if (ctx.checks() && !(cond)) {                                          \
        check_failed(ps.counts, (code), (kernel), (uint32_t)(slot), (uint32_t)(v)); \
        continue;                                                           \
    }

// The pixel/sample of path p: p = ((row * rect.width) + col) * sample_count + k
__device__ __forceinline__ void path_coords(const LaunchParams& lp, uint32_t p, uint32_t& sx, uint32_t& sy,
                                            uint32_t& s) {
    const uint32_t k = p % lp.sample_count;
    const uint32_t pix = p / lp.sample_count;
    const uint32_t col = pix % lp.rect.width, row = pix / lp.rect.width;
    sx = lp.rect.left + col - lp.full.left;
    sy = lp.rect.top + row - lp.full.top;
    s = lp.sample_begin + k;
}

// PerspectiveCamera rayGen (Src/BuiltinComponent/Sensor/PerspectiveCamera/Kernel.cpp:22-48)
__device__ __forceinline__ void camera_ray(const pb2_camera& cam, float ndc_x, float ndc_y, float u1, float u2, v3& org,
                                           v3& dir) {
    const v3 base = mk3(cam.position[0], cam.position[1], cam.position[2]);
    const v3 look = mk3(cam.look_at[0], cam.look_at[1], cam.look_at[2]);
    const v3 forward = normalize3(sub3(look, base));
    const v3 right = cross3(forward, mk3(cam.up[0], cam.up[1], cam.up[2]));
    const v3 up = cross3(right, forward);
    const v3 film_hit = add3(add3(base, mul3s(right, cam.sensor_size[0] * (0.5f - ndc_x))),
                             mul3s(up, cam.sensor_size[1] * (ndc_y - 0.5f)));
    const float focal_distance = dot3(sub3(look, base), forward);
    const float film_distance = 1.0f / (1.0f / cam.focal_length - 1.0f / focal_distance);
    const v3 lens_center = add3(base, mul3s(forward, film_distance));
    const float ang = u1 * kTwoPi;
    const float rad = sqrt_safe(u2);
    float s, c;
    pb2_sincosf(ang, &s, &c);
    const float lx = rad * c, ly = rad * s;
    const v3 lens_hit = add3(add3(lens_center, mul3s(right, cam.aperture_radius * lx)), mul3s(up, cam.aperture_radius * ly));
    const v3 d = sub3(lens_center, film_hit);
    const v3 focus_hit = add3(lens_center, mul3s(d, focal_distance / dot3(d, forward)));
    org = lens_hit;
    dir = normalize3(sub3(focus_hit, lens_hit));
}

// piperMain's sample set-up (Src/BuiltinComponent/Tracer/Embree/Kernel.cpp:47-90)
__device__ __forceinline__ void primary_ray(const LaunchParams& lp, uint32_t sx, uint32_t sy, uint32_t s,
                                            uint64_t& index, float& px, float& py, v3& org, v3& dir) {
    const float res = (float)(1u << lp.log2res);
    index = sobol_interval_to_index(lp.log2res, s, sx, sy);
    const float offx = fminf(fmaxf(sobol_sample_fast(index, 0) * res - (float)sx, 0.0f), 1.0f);
    const float offy = fminf(fmaxf(sobol_sample_fast(index, 1) * res - (float)sy, 0.0f), 1.0f);
    px = offx + (float)(lp.full.left + sx);
    py = offy + (float)(lp.full.top + sy);
    const float ndc_x = lp.ndc.ox + lp.ndc.sx * px / (float)lp.width;
    const float ndc_y = lp.ndc.oy + lp.ndc.sy * py / (float)lp.height;
    const float u1 = sobol_sample_s(index, 3, lp.scramble, lp.scramble_seed);
    const float u2 = sobol_sample_s(index, 4, lp.scramble, lp.scramble_seed);
    camera_ray(lp.cam, ndc_x, ndc_y, u1, u2, org, dir);
}

__global__ void k_camera_rays(LaunchParams lp, uint32_t sample, float4* __restrict__ rays, float2* __restrict__ points) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lp.rect.width * lp.rect.height) return;
    const uint32_t col = i % lp.rect.width, row = i / lp.rect.width;
    const uint32_t sx = lp.rect.left + col - lp.full.left, sy = lp.rect.top + row - lp.full.top;
    uint64_t index;
    float px, py;
    v3 o, d;
    primary_ray(lp, sx, sy, sample, index, px, py, o, d);
    rays[2 * i] = make_float4(o.x, o.y, o.z, 1e-3f);
    rays[2 * i + 1] = make_float4(d.x, d.y, d.z, 1e5f);
    points[i] = make_float2(px, py);
}

// ---- traversal over queues -----------------------------------------------------------------------

constexpr int kQThreads = 128;
constexpr int kQRefill = 4;
constexpr int kQSteps = 4;

enum QueueTraceKind : int { Q_EXTEND, Q_MIS, Q_SHADOW };

// The MIS ray of a vertex only matters if its closest hit is a plane of the selected light, or nothing
// (the environment).  So it is answered with the planes first (all lights' parallelograms, tested in
// order, as the closest-hit query's plane pass does) and an occlusion query over the triangles:
//   nearest plane belongs to the selected light at t_L -> any hit on (tmin, next float after t_L): a
//     triangle at t <= t_L wins the closest-hit query (planes lose ties), otherwise the plane is the hit;
//   nearest plane belongs to another light -> that plane or a triangle is hit: neither counts, no query;
//   no plane -> any hit on (tmin, tmax): occluded means a triangle is hit, free means a miss.
// The record (t, prim) written is what k_finish needs: the plane and its t, PB2_INVALID_PRIM for a miss,
// or the occluding triangle.  k_finish's result is that of the closest-hit query.
// Resident blocks per SM the register budget is sized for: 10 for closest hit, 9 for the any-hit queries
// (as the API kernels; at 10 the any-hit queries spilled about 90 bytes).
// kCount: the counting build (pipelines with counting on): adds the rays, node visits and triangle tests of
// the queue to trace_counters[3 kKind .. 3 kKind + 2] for the byte model of the render roofline.
template <int kKind, class Ctx, bool kCount = false>
__global__ void __launch_bounds__(kQThreads, kKind == Q_EXTEND ? 10 : 9) k_trace_queue(const __grid_constant__ Ctx ctx, Paths ps,
                                                           const uint32_t* __restrict__ queue,
                                                           const uint32_t* __restrict__ count_ptr, uint32_t* work,
                                                           unsigned long long* stat,
                                                           unsigned long long* trace_counters = nullptr) {
    constexpr bool kClosest = kKind == Q_EXTEND;
    const uint32_t n = *count_ptr;
    __shared__ uint2 stack_smem[kSharedStack * kQThreads];
    Traverser<kClosest, kCount, kQThreads> tr;
    uint32_t nv = 0, nt = 0;
    tr.bind_stack(stack_smem);
    bool active = false;
    uint32_t slot = 0;
    float mis_t = 0.0f;      // Q_MIS: nearest plane's t and index (kInvalidPrim: none)
    uint32_t mis_plane = 0;
    BvhView bvh{};
    if constexpr (!Ctx::kBatch) bvh = ctx.bvh(0);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t rays = 0;
    for (;;) {
        const unsigned inactive = __ballot_sync(0xFFFFFFFFu, !active);
        if (__popc(inactive) >= kQRefill) {
            const int leader = __ffs(inactive) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(work, (uint32_t)__popc(inactive));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (!active) {
                const uint32_t idx = base + __popc(inactive & lt_mask);
                if (idx < n) {
                    slot = queue[idx];
                    if constexpr (Ctx::kBatch) bvh = ctx.bvh(slot);
                    float4 a, b;
                    if (kKind == Q_EXTEND) {
                        a = ps.o[slot]; b = ps.d[slot];
                        a.w = 1e-3f; b.w = 1e5f;
                    } else if (kKind == Q_MIS) {
                        a = ps.mr_o[slot]; b = ps.mr_d[slot];
                        a.w = 1e-3f; b.w = 1e5f;
                    } else {
                        a = ps.sh_o[slot]; b = ps.sh_d[slot];
                    }
                    tr.init(bvh, a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w);
                    active = true;
                    ++rays;
                    if (kKind == Q_MIS) {
                        mis_t = tr.p.tmax;
                        mis_plane = kInvalidPrim;
                        for (uint32_t i = 0; i < bvh.plane_count; ++i) {
                            float t, u, v;
                            bool front;
                            if (plane_test(bvh.planes[i], tr.p, tr.p.tmin, mis_t, t, u, v, front)) {
                                mis_t = t;
                                mis_plane = i;
                            }
                        }
                        const uint32_t sel = __float_as_uint(ps.mr_pdf[slot].y);
                        if (mis_plane != kInvalidPrim && !(sel != 0u && bvh.planes[mis_plane].light == sel - 1u)) {
                            tr.done = true;  // another light's plane: the ray completes at once with that plane
                        } else if (mis_plane != kInvalidPrim) {
                            tr.p.tmax = __uint_as_float(__float_as_uint(mis_t) + 1u);  // the next float after t_L
                            tr.tbest = tr.p.tmax;
                        }
                    }
                }
            }
            if (__ballot_sync(0xFFFFFFFFu, active) == 0u) break;
        }
        if (active) {
#pragma unroll 1
            for (int it = 0; it < kQSteps && !tr.done; ++it) tr.iteration(bvh);
            if (tr.done) {
                if (kClosest) {
                    bool front;
                    tr.finish_planes(bvh, front);
                    ps.hit[slot] = make_float4(tr.tbest, __uint_as_float(tr.best_prim), tr.bu, tr.bv);
                    ps.hit_slot[slot] = tr.best_slot;
                } else if (kKind == Q_MIS) {
                    // the occluding triangle's id, or the nearest plane (kInvalidPrim: none); no marker
                    // values: every prim written is a real triangle, a plane, or PB2_INVALID_PRIM
                    const uint32_t prim = tr.best_prim != kInvalidPrim ? tr.best_prim
                                          : (mis_plane == kInvalidPrim ? kInvalidPrim : (kPlaneFlag | mis_plane));
                    ps.mhit[slot] = make_float4(tr.best_prim != kInvalidPrim ? tr.tbest : mis_t, __uint_as_float(prim),
                                                0.0f, 0.0f);
                } else {
                    ps.occ[slot] = tr.best_prim != kInvalidPrim ? 1u : 0u;
                }
                if (tr.overflow) atomicOr(&ps.counts[C_ERROR], 1u);
                if constexpr (kCount) {
                    nv += tr.node_visits;
                    nt += tr.tri_tests;
                }
                active = false;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) rays += __shfl_xor_sync(0xFFFFFFFFu, rays, o);
    if (lane == 0 && rays) atomicAdd(stat, (unsigned long long)rays);
    if constexpr (kCount) {
        for (int o = 16; o > 0; o >>= 1) {
            nv += __shfl_xor_sync(0xFFFFFFFFu, nv, o);
            nt += __shfl_xor_sync(0xFFFFFFFFu, nt, o);
        }
        if (lane == 0) {
            atomicAdd(trace_counters + 3 * kKind + 0, (unsigned long long)rays);
            atomicAdd(trace_counters + 3 * kKind + 1, (unsigned long long)nv);
            atomicAdd(trace_counters + 3 * kKind + 2, (unsigned long long)nt);
        }
    }
}

// ---- film -------------------------------------------------------------------------------------------

__device__ __forceinline__ float filter_weight(const LaunchParams& lp, float dx, float dy) {
    if (lp.filter == PB2_FILTER_TRIANGLE) return fmaxf(0.0f, 1.0f - fabsf(dx)) * fmaxf(0.0f, 1.0f - fabsf(dy));
    if (lp.filter == PB2_FILTER_GAUSSIAN) {
        const float wx = fmaxf(pb2_expf(lp.gauss_neg_alpha * dx * dx) - lp.gauss_sub, 0.0f);
        const float wy = fmaxf(pb2_expf(lp.gauss_neg_alpha * dy * dy) - lp.gauss_sub, 0.0f);
        return wx * wy;
    }
    return 1.0f;
}

// accumulate (Src/BuiltinComponent/RenderDriver/FixedSampler/Kernel.cpp:30-52)
__device__ __forceinline__ void splat(const LaunchParams& lp, float4* film, float px, float py, spec v) {
    const int32_t bx = (int32_t)(px - 0.5f), by = (int32_t)(py - 0.5f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t x = (uint32_t)(bx + (k & 1)), y = (uint32_t)(by + (k >> 1));
        if (!(x < lp.width && y < lp.height)) continue;
        const float w = filter_weight(lp, px - ((float)x + 0.5f), py - ((float)y + 0.5f));
        atomicAdd(&film[(size_t)x + (size_t)y * lp.width], make_float4(v.r * w, v.g * w, v.b * w, w));
    }
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// A finished path's slot becomes free for a later iteration's claim: its bit of the free bitmap is set (lanes freeing
// slots of one 32-slot word set their bits with one atomic) and the free count grows by one.
__device__ __forceinline__ void free_slot(const Paths& ps, uint32_t slot) {
    const uint32_t w = slot >> 5;
    const unsigned grp = __match_any_sync(__activemask(), w);
    const uint32_t bits = __reduce_or_sync(grp, 1u << (slot & 31u));
    if ((int)(threadIdx.x & 31u) == __ffs(grp) - 1) atomicOr(&ps.free_bits[w], bits);
    warp_push(&ps.counts[C_FREE]);
}

// A finished path: splat its radiance; in a batched launch also free its slot and count the scene down.
template <class Ctx>
__device__ __forceinline__ void terminate_path(const Ctx& ctx, const Paths& ps, uint32_t slot, uint32_t cur) {
    const float4 r = ps.rad[slot];
    const float2 pt = ps.point[slot];
    float4* film = ctx.film_of(slot);
    if (film) splat(ctx.P(slot), film, pt.x, pt.y, mksp(r.x, r.y, r.z));
    if constexpr (Ctx::kBatch) {
        const uint32_t scene = ps.scene[slot];
        free_slot(ps, slot);
        // one atomic per scene among the lanes finishing together (every finished path of a scene counts the
        // same word down, so a per-path atomic serialises at that word's L2 slice)
        const unsigned grp = __match_any_sync(__activemask(), scene);
        if ((int)(threadIdx.x & 31u) == __ffs(grp) - 1) {
            const uint32_t cnt = (uint32_t)__popc(grp);
            if (atomicSub(&ctx.remaining[scene], cnt) == cnt) ctx.done_ns[scene] = globaltimer();
        }
    } else {
        if (ctx.sample_out) {  // at the path's launch-relative index (a slot serves many paths)
            float* o = ctx.sample_out + 5 * (size_t)ps.scene[slot];
            o[0] = pt.x; o[1] = pt.y; o[2] = r.x; o[3] = r.y; o[4] = r.z;
        }
        if (ctx.lp.refill) free_slot(ps, slot);
    }
}

__device__ __forceinline__ float luminance(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Turns the path's pending guided vertices into training records: the incident radiance estimate along
// the sampled direction is (radiance gathered after the vertex) / (throughput before the vertex's
// sampling) x pdf / (f cos), so target / pdf = lum(S_end - S_v) / lum(pf_v).
// The two record counters are shared by every path of the launch, so both are added to once per warp, not once per
// record.
__device__ __forceinline__ void flush_records(const GuideState& gs, uint32_t slot, float4 s_end) {
    const uint32_t n = gs.nrec[slot];
    uint32_t seen = 0;
    for (uint32_t r = 0; r < n; ++r) {
        const float4 a = gs.rec[(r * 5 + 0) * gs.cap + slot];
        const float4 b = gs.rec[(r * 5 + 1) * gs.cap + slot];
        const float4 c = gs.rec[(r * 5 + 2) * gs.cap + slot];
        const float4 pf = gs.rec[(r * 5 + 3) * gs.cap + slot];
        const float4 sv = gs.rec[(r * 5 + 4) * gs.cap + slot];
        const float lpf = luminance(pf.x, pf.y, pf.z);
        const float dl = luminance(s_end.x - sv.x, s_end.y - sv.y, s_end.z - sv.z);
        if (!(dl > 0.f && lpf > 0.f)) continue;
        const float w = dl / lpf;
        if (!(w < 3.0e38f)) continue;
        ++seen;
        const float u = (float)(hash32(slot * 3u + r + gs.salt * 0x9E3779B9u) >> 8) * (1.0f / 16777216.0f);
        if (u >= gs.accept_prob) continue;
        const uint32_t idx = warp_push(&gs.train_count[0]);
        if (idx >= gs.train_capacity) continue;
        float4* o = reinterpret_cast<float4*>(gs.train + 16 * (size_t)idx);
        o[0] = make_float4(a.x, a.y, a.z, a.w);
        o[1] = make_float4(b.x, b.y, b.z, b.w);
        o[2] = make_float4(c.x, c.y, c.z, c.w);
        o[3] = make_float4(w, 0.f, 0.f, 0.f);
    }
    const unsigned mask = __activemask();
    const uint32_t seen_warp = __reduce_add_sync(mask, seen);
    if ((int)(threadIdx.x & 31u) == __ffs(mask) - 1 && seen_warp) atomicAdd(&gs.train_count[1], seen_warp);
    gs.nrec[slot] = 0;
}

// ---- classify extend results (PathTracing/Kernel.cpp:116-149) ------------------------------------

template <class Ctx>
__global__ void k_classify(const __grid_constant__ Ctx ctx, Paths ps, GuideState gs, uint32_t cur) {
    const uint32_t n = ps.counts[C_EXT_CUR];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        PB2_CHECK(n <= ctx.capacity(), 1, K_CLASSIFY, 0, n);
        const uint32_t slot = ps.ext[cur][i];
        PB2_CHECK(slot < ctx.capacity(), 2, K_CLASSIFY, slot, i);
        const LaunchParams& lp = ctx.P(slot);
        const SceneView& sv = ctx.S(slot);
        const float4 h = ps.hit[slot];
        const uint32_t prim = __float_as_uint(h.y);
        PB2_CHECK(prim == kInvalidPrim || ((prim & kPlaneFlag) ? (prim & ~kPlaneFlag) < sv.bvh.plane_count
                                                                : prim < sv.bvh.tri_count),
                  3, K_CLASSIFY, slot, prim);
        const bool missing = prim == kInvalidPrim;
        const bool area = !missing && (prim & kPlaneFlag);
        if (!missing && !area) {
            // a surface hit (most paths): only its material and the path depth are read here
            if (ps.depth[slot] >= lp.max_depth) {
                if (gs.enabled) flush_records(gs, slot, ps.rad[slot]);
                terminate_path(ctx, ps, slot, cur);
                continue;
            }
            PB2_CHECK(sv.prim_material[prim] < sv.material_count, 4, K_CLASSIFY, slot, sv.prim_material[prim]);
            const uint32_t type = sv.materials[sv.prim_material[prim]].type;
            PB2_CHECK(type < (uint32_t)kNumSurfaceTypes, 5, K_CLASSIFY, slot, type);
            // a vertex that samples the guide is shaded by its type's guided kernel over the guide queue, every
            // other one by the plain kernel over its type's queue
            if (guide_vertex(gs, type, ps.depth[slot])) ps.guide_q[warp_push(&ps.counts[C_GUIDE])] = slot;
            else ps.surf[type][warp_push(&ps.counts[C_SURF0 + type])] = slot;
            continue;
        }
        // a miss or an area light: emission on specular paths, pass-through, termination
        const float4 o4 = ps.o[slot], d4 = ps.d[slot];
        const float4 pf4 = ps.pf[slot];
        const bool specular = pf4.w != 0.0f;
        spec sample = mksp(ps.rad[slot].x, ps.rad[slot].y, ps.rad[slot].z);
        const spec pf = mksp(pf4.x, pf4.y, pf4.z);
        const v3 d = mk3(d4.x, d4.y, d4.z);
        if (specular && (area || missing)) {
            spec rad;
            if (area) {
                const DevPlane& pl = sv.bvh.planes[prim & ~kPlaneFlag];
                // planeSurface: N faces the ray (face from the renormalised direction, Embree.cpp:573-577)
                const v3 dn = normalize3(d);
                const v3 nrm = mk3(pl.normal[0], pl.normal[1], pl.normal[2]);
                const bool front = dot3(dn, nrm) > 0.0f;
                const v3 N = front ? neg3(nrm) : nrm;
                const v3 wi = normalize3(mul3s(d, h.x));
                const DevLight& L = sv.lights[pl.light];
                rad = dot3(N, wi) < 0.0f ? mksp(L.radiance[0], L.radiance[1], L.radiance[2]) : sp_zero();
            } else {
                rad = mksp(lp.env[0], lp.env[1], lp.env[2]);
            }
            sample = sp_add(sample, sp_mul(pf, rad));
            ps.rad[slot] = make_float4(sample.r, sample.g, sample.b, 0.0f);
        }
        if (area) {
            // pass through the light, one bounce credited back (the uint32 depth may wrap)
            ps.depth[slot] = ps.depth[slot] - 1u;
            const v3 o = add3(mk3(o4.x, o4.y, o4.z), mul3s(d, h.x + 0.001f));
            ps.o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
            ps.ext[cur ^ 1][warp_push(&ps.counts[C_EXT_NEXT])] = slot;
            continue;
        }
        if (gs.enabled) flush_records(gs, slot, ps.rad[slot]);  // a miss ends the path
        terminate_path(ctx, ps, slot, cur);
    }
}

// ---- shading (PathTracing/Kernel.cpp:23-107, 150-190) ---------------------------------------------

struct SampleCursor {
    uint64_t index;
    uint32_t dim;
    uint32_t scramble, seed;
    __device__ __forceinline__ float next() {
        if (dim >= PB2_SOBOL_DIMS) return 0.5f;  // unreachable: the pipeline rejects depths that could get here
        return sobol_sample_s(index, dim++, scramble, seed);
    }
    // the two piperSample() arguments of one call are evaluated right to left (u2 first)
    __device__ __forceinline__ void pair(float& u1, float& u2) {
        u2 = next();
        u1 = next();
    }
};

// select() of Src/Kernel/Sampling.hpp:52-63 (u remapped with cdf[r] itself)
__device__ __forceinline__ uint32_t cdf_select(const float* cdf, const float* pdf, uint32_t size, float& u) {
    uint32_t l = 0, r = size;
    while (l < r) {
        const uint32_t mid = (l + r) >> 1;
        if (u >= cdf[mid]) l = mid + 1;
        else r = mid;
    }
    // u rounds to 1.0f when the Sobol value is within 2^-25 of 1 (its float conversion rounds up); the
    // reference then reads one past the end, here the last entry is used
    if (r >= size) r = size - 1;
    u = (u - cdf[r]) / pdf[r];
    return r;
}

struct LightSample {
    v3 dir;
    spec rad;
    float pdf, distance;
};

// diffuseSample over planeSample (AreaLight/Kernel.cpp:24-41, BasicShapes/Kernel.cpp:113-134)
__device__ __forceinline__ void area_sample(const SceneView& sv, uint32_t li, v3 hit, float u1, float u2, LightSample& ls) {
    const DevLight& L = sv.lights[li];
    const uint32_t idx = cdf_select(sv.plane_cdf + L.first_plane, sv.plane_pdf + L.first_plane, L.plane_count, u1);
    const DevPlane& pl = sv.bvh.planes[L.first_plane + idx];
    const v3 lp = add3(add3(mk3(pl.origin[0], pl.origin[1], pl.origin[2]), mul3s(mk3(pl.u[0], pl.u[1], pl.u[2]), u1)),
                       mul3s(mk3(pl.v[0], pl.v[1], pl.v[2]), u2));
    const v3 src = add3(lp, mk3(L.translation[0], L.translation[1], L.translation[2]));
    v3 n = mk3(pl.normal[0], pl.normal[1], pl.normal[2]);
    if (dot3(sub3(hit, src), n) <= 0.0f) n = neg3(n);
    const float pdf = L.inverse_area;
    const v3 delta = sub3(src, hit);
    if (pdf == 0.0f || dot3(delta, n) >= 0.0f) {
        ls.pdf = 0.0f;
        return;
    }
    ls.rad = mksp(L.radiance[0], L.radiance[1], L.radiance[2]);
    const float dis2 = len2_3(delta);
    ls.distance = sqrtf(dis2);
    ls.dir = div3s(delta, ls.distance);
    ls.pdf = pdf * dis2 / fabsf(dot3(n, ls.dir));
}

// SESample (BasicLight/Kernel.cpp:61-73)
__device__ __forceinline__ void env_sample(const LaunchParams& lp, float u1, float u2, LightSample& ls) {
    ls.rad = mksp(lp.env[0], lp.env[1], lp.env[2]);
    const float theta = u1 * kPi, phi = u2 * kPi;
    float st, ct, sp, cp;
    pb2_sincosf(theta, &st, &ct);
    pb2_sincosf(phi, &sp, &cp);
    ls.dir = mk3(st * cp, st * sp, ct);
    ls.pdf = st == 0.0f ? 0.0f : 1.0f / ((2.0f * kSqrPi) * st);
    ls.distance = 1e5f;
}

// SEPdf (BasicLight/Kernel.cpp:80-89)
__device__ __forceinline__ float env_pdf(v3 dir) {
    const float theta = pb2_acosf(fmaxf(-1.0f, fminf(1.0f, dir.z)));
    const float st = pb2_sinf(theta);
    return st == 0.0f ? 0.0f : 1.0f / ((2.0f * kSqrPi) * st);
}

struct Frame {
    v3 T, B, N, Ng;
};
__device__ __forceinline__ v3 to_shading(const Frame& f, v3 v) { return mk3(dot3(f.T, v), dot3(f.B, v), dot3(f.N, v)); }
__device__ __forceinline__ v3 to_local(const Frame& f, v3 v) {
    return mk3(f.T.x * v.x + f.B.x * v.y + f.N.x * v.z, f.T.y * v.x + f.B.y * v.y + f.N.y * v.z,
               f.T.z * v.x + f.B.z * v.y + f.N.z * v.z);
}

// Material types whose continuation is guided: those whose BxDF sampler draws exactly the density its pdf
// reports (Lambert and Oren-Nayar cosine sampling, the conductor's visible-normal sampling).  One-sample MIS
// with the guide needs that density; the reference's microfacet lobes (Plastic, rough Glass, Substrate) report
// a pdf that is not their sampler's density (Classic/Kernel.cpp:405-412), so they keep plain BxDF sampling.
__host__ __device__ constexpr bool guided_type(int t) { return t == PB2_SURFACE_MATTE || t == PB2_SURFACE_CONDUCTOR; }

// (No launch bounds: batched renders launch it with the autotuned block size, up to 512 threads.  A
// sweep of register budgets for 4-8 resident 128-thread blocks changed render times by under 2 %.)
// kGuided: the variant launched while a guide is attached (guided sampling and training records compiled in);
// plain launches use the variant without them, which needs fewer registers.
// The plain variants are held to 64 registers (__launch_bounds__(512, 2): two 512-thread blocks, or eight of 128,
// per SM): the kernel is latency-bound, and the texture lookups had taken the Matte variant to 72 registers and
// 28 resident warps.
template <int kType, class Ctx, bool kGuided = false>
__global__ void __launch_bounds__(512, kGuided ? 1 : 2) k_shade(const __grid_constant__ Ctx ctx, Paths ps, GuideState gs,
                                                                 uint32_t cur) {
    // the guided variant shades the guide queue (the vertices of the guided types that sample the guide), taking
    // the vertices of its own type; the plain variant shades its type's queue
    const uint32_t* queue = kGuided ? ps.guide_q : ps.surf[kType];
    const uint32_t n = kGuided ? ps.counts[C_GUIDE] : ps.counts[C_SURF0 + kType];
    uint32_t vertices = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        PB2_CHECK(n <= ctx.capacity(), 10, K_SHADE, 0, n);
        const uint32_t slot = queue[i];
        PB2_CHECK(slot < ctx.capacity(), 11, K_SHADE, slot, i);
        const LaunchParams& lp = ctx.P(slot);
        const SceneView& sv = ctx.S(slot);
        const float4 h = ps.hit[slot];
        const uint32_t prim = __float_as_uint(h.y);
        PB2_CHECK(prim < sv.bvh.tri_count, 12, K_SHADE, slot, prim);
        if constexpr (kGuided)
            if (sv.materials[sv.prim_material[prim]].type != (uint32_t)kType) continue;  // another guided type's vertex
        ++vertices;
        PB2_CHECK(ps.hit_slot[slot] < sv.bvh.tri_count, 13, K_SHADE, slot, ps.hit_slot[slot]);
        PB2_CHECK(ps.dim[slot] <= PB2_SOBOL_DIMS, 14, K_SHADE, slot, ps.dim[slot]);
        const float4 o4 = ps.o[slot], d4 = ps.d[slot], pf4 = ps.pf[slot];
        const v3 o = mk3(o4.x, o4.y, o4.z), d = mk3(d4.x, d4.y, d4.z);
        spec pf = mksp(pf4.x, pf4.y, pf4.z);
        uint32_t depth = ps.depth[slot];
        SampleCursor sc{ ps.sidx[slot], ps.dim[slot], lp.scramble, lp.scramble_seed };
        // calcTriangleMeshSurface (Tracer/Embree/Kernel.cpp:170-192) with face from Embree.cpp:336
        const uint32_t hs = ps.hit_slot[slot];
        const float4* t4 = reinterpret_cast<const float4*>(sv.bvh.tris + hs);
        const float4 a = t4[0], b = t4[1], c = t4[2];
        const v3 p0 = mk3(a.x, a.y, a.z), p1 = mk3(b.x, b.y, b.z), p2 = mk3(c.x, c.y, c.z);
        const v3 ng = normalize3(cross3(sub3(p1, p0), sub3(p2, p0)));
        const bool front = dot3(d, ng) < 0.0f;
        Frame fr;
        fr.N = fr.Ng = front ? ng : neg3(ng);
        if (fabsf(dot3(fr.N, mk3(1.0f, 0.0f, 0.0f))) < fabsf(dot3(fr.N, mk3(0.0f, 1.0f, 0.0f))))
            fr.T = cross3(fr.N, mk3(1.0f, 0.0f, 0.0f));
        else
            fr.T = cross3(fr.N, mk3(0.0f, 1.0f, 0.0f));
        fr.B = cross3(fr.N, fr.T);
        const v3 wo = to_shading(fr, neg3(d));
        const v3 ng_sh = to_shading(fr, fr.Ng);
        Bsdf bsdf;
        DevMaterial mat = sv.materials[sv.prim_material[prim]];
        if (mat.tex[0] | mat.tex[1] | mat.tex[2] | mat.tex[3]) {
            // calcTriangleMeshSurface's texCoord (Tracer/Embree/Kernel.cpp:181-190): tc[i1] u + tc[i2] v + tc[i0] w
            float tu = 0.0f, tv = 0.0f;
            if (sv.tri_uv) {
                const float2* q = sv.tri_uv + 3 * (size_t)prim;
                const float bw = (1.0f - h.z) - h.w;
                tu = (q[1].x * h.z + q[2].x * h.w) + q[0].x * bw;
                tv = (q[1].y * h.z + q[2].y * h.w) + q[0].y * bw;
            }
            apply_textures(mat, sv.textures, tu, tv);
        }
        bsdf_init<kType>(mat, front, bsdf);
        const v3 hit = add3(o, mul3s(d, h.x));
        uint32_t flags = 0;
        if (bsdf.no_specular) {
            // multipleImportanceSampling (PathTracing/Kernel.cpp:23-107)
            flags |= 1u;
            const uint32_t count = 1u + lp.num_lights;
            const float u = sc.next();
            uint32_t sel = (uint32_t)floorf(u * (float)count);
            if (sel > count - 1) sel = count - 1;
            PB2_CHECK(sel == 0 || sv.lights[sel - 1].first_plane + sv.lights[sel - 1].plane_count <= sv.bvh.plane_count,
                      15, K_SHADE, slot, sel);
            const float sel_pdf = 1.0f / (float)count;
            ps.mis_pf[slot] = make_float4(pf.r, pf.g, pf.b, sel_pdf);
            float4 nee = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            {
                LightSample ls;
                float u1, u2;
                sc.pair(u1, u2);
                if (sel == 0) env_sample(lp, u1, u2, ls);
                else area_sample(sv, sel - 1, hit, u1, u2, ls);
                if (ls.pdf > 0.0f && sp_valid(ls.rad)) {
                    const v3 wi = to_shading(fr, ls.dir);
                    const spec f = bsdf_eval(bsdf, wo, wi, ng_sh, kPartNoSpecular);
                    if (sp_valid(f)) {
                        float w = fabsf(wi.z) / ls.pdf;
                        const float bp = bsdf_pdf(bsdf, wo, wi, kPartNoSpecular);
                        w = w * power_heuristic(ls.pdf, bp);
                        const spec cand = sp_muls(sp_mul(f, ls.rad), w);
                        nee = make_float4(cand.r, cand.g, cand.b, 1.0f);
                        ps.sh_o[slot] = make_float4(hit.x, hit.y, hit.z, fminf(1e-3f, ls.distance));
                        ps.sh_d[slot] = make_float4(ls.dir.x, ls.dir.y, ls.dir.z, ls.distance);
                        ps.shadow_q[warp_push(&ps.counts[C_SHADOW])] = slot;
                    }
                }
            }
            ps.nee[slot] = nee;
            {
                BsdfSample bs;
                float u1, u2;
                sc.pair(u1, u2);
                bsdf_sample(bsdf, u1, u2, wo, ng_sh, kPartNoSpecular, bs);
                if (bs.pdf > 0.0f && sp_valid(bs.f)) {
                    const float weight = fabsf(bs.wi.z) / bs.pdf;
                    const v3 dir = to_local(fr, bs.wi);
                    ps.mr_o[slot] = make_float4(hit.x, hit.y, hit.z, 0.0f);
                    ps.mr_d[slot] = make_float4(dir.x, dir.y, dir.z, 0.0f);
                    ps.mr_f[slot] = make_float4(bs.f.r, bs.f.g, bs.f.b, weight);
                    ps.mr_pdf[slot] = make_float2(bs.pdf, __uint_as_float(sel));
                    ps.mis_q[warp_push(&ps.counts[C_MIS])] = slot;
                    flags |= 4u;
                }
            }
        }
        // continuation (PathTracing/Kernel.cpp:164-190); guided vertices sample 0.5 BxDF + 0.5 mixture
        const bool guided = kGuided && guided_type(kType) && guide_vertex(gs, kType, depth) && bsdf.no_specular;
        v3 wi_sh;
        spec fval;
        float pdf;
        int part;
        bool cont;
        if (!guided) {
            BsdfSample ss;
            float u1, u2;
            sc.pair(u1, u2);
            bsdf_sample(bsdf, u1, u2, wo, ng_sh, kPartAll, ss);
            cont = ss.pdf > 0.0f && sp_valid(ss.f);
            wi_sh = ss.wi;
            fval = ss.f;
            pdf = ss.pdf;
            part = ss.part;
        } else {
            const float uc = sc.next();
            float u1, u2;
            sc.pair(u1, u2);
            guide::Mixture mx;
            const float* mp = gs.mix + 40 * (size_t)slot;
#pragma unroll
            for (int k = 0; k < guide::kLobes; ++k) {
                mx.w[k] = mp[k];
                mx.mu[k][0] = mp[8 + 3 * k];
                mx.mu[k][1] = mp[9 + 3 * k];
                mx.mu[k][2] = mp[10 + 3 * k];
                mx.kappa[k] = mp[32 + k];
            }
            float pb, pg;
            cont = true;
            if (uc < gs.sel_prob) {
                float x, y, z;
                guide::mixture_sample(mx, uc / gs.sel_prob, u1, u2, x, y, z);
                wi_sh = to_shading(fr, mk3(x, y, z));
                fval = bsdf_eval(bsdf, wo, wi_sh, ng_sh, kPartAll);
                pb = bsdf_pdf(bsdf, wo, wi_sh, kPartAll);
                pg = guide::mixture_pdf(mx, x, y, z);
            } else {
                BsdfSample ss;
                bsdf_sample(bsdf, u1, u2, wo, ng_sh, kPartAll, ss);
                cont = ss.pdf > 0.0f && sp_valid(ss.f);
                wi_sh = ss.wi;
                fval = ss.f;
                pb = ss.pdf;
                const v3 wl = to_local(fr, ss.wi);
                pg = cont ? guide::mixture_pdf(mx, wl.x, wl.y, wl.z) : 0.0f;
            }
            pdf = gs.sel_prob * pg + (1.0f - gs.sel_prob) * pb;
            cont = cont && pdf > 0.0f && sp_valid(fval);
            part = (dot3(wo, ng_sh) * dot3(wi_sh, ng_sh)) > 0.0f ? kPartR : kPartT;
        }
        const spec pf_in = pf;
        if (cont) {
            pf = sp_muls(sp_mul(pf, fval), fabsf(wi_sh.z) / pdf);
            if (depth > lp.min_rr_depth) {
                const float p = fmaxf(0.05f, 1.0f - fmaxf(pf.r, fmaxf(pf.g, pf.b)));
                if (sc.next() < p) cont = false;
                else pf = sp_divs(pf, 1.0f - p);
            }
        }
        if (cont) {
            const v3 nd = to_local(fr, wi_sh);
            const v3 no = add3(hit, mul3s(fr.Ng, (part & kPartR) ? 0.001f : -0.001f));
            ps.o[slot] = make_float4(no.x, no.y, no.z, 0.0f);
            ps.d[slot] = make_float4(nd.x, nd.y, nd.z, 0.0f);
            ps.pf[slot] = make_float4(pf.r, pf.g, pf.b, (part & kPartSpecular) ? 1.0f : 0.0f);
            ps.depth[slot] = depth + 1u;
            flags |= 2u;
            if (guided) {
                const uint32_t r = gs.nrec[slot];
                if (r < (uint32_t)kMaxRecords) {
                    const v3 wl = to_local(fr, wo);
                    const float px = (hit.x - gs.bmin[0]) * gs.binv[0], py = (hit.y - gs.bmin[1]) * gs.binv[1],
                                pz = (hit.z - gs.bmin[2]) * gs.binv[2];
                    gs.rec[(r * 5 + 0) * gs.cap + slot] = make_float4(px, py, pz, fr.N.x);
                    gs.rec[(r * 5 + 1) * gs.cap + slot] = make_float4(fr.N.y, fr.N.z, wl.x, wl.y);
                    gs.rec[(r * 5 + 2) * gs.cap + slot] = make_float4(wl.z, nd.x, nd.y, nd.z);
                    gs.rec[(r * 5 + 3) * gs.cap + slot] = make_float4(pf_in.r, pf_in.g, pf_in.b, 0.0f);
                    gs.nrec[slot] = r + 1;
                    flags |= 8u;
                }
            }
        }
        ps.dim[slot] = sc.dim;
        ps.flags[slot] = flags;
        ps.shaded_q[warp_push(&ps.counts[C_SHADED])] = slot;
    }
    if (vertices) warp_count(reinterpret_cast<unsigned long long*>(ps.counts + C_STAT_VERTICES), vertices);
}

// ---- guide inference for the surface queues of the guided material types ------------------------------

// Rows of the guide's forward pass: the vertices in the guided material types' surface queues, in queue
// order; a row's key is its path slot, whose mixture parameters the output writes.
struct GuideRows {
    static constexpr bool kStaged = false;  // outputs go to each vertex's path slot
    SceneView sv;
    Paths ps;
    GuideState gs;
    __device__ __forceinline__ void features(uint32_t row, float (&f)[9], uint32_t& slot) const {
        slot = ps.guide_q[row];
        slot_features(slot, f);
    }
    __device__ __forceinline__ void slot_features(uint32_t slot, float (&f)[9]) const {
        const float4 h = ps.hit[slot];
        const float4 o4 = ps.o[slot], d4 = ps.d[slot];
        const v3 d = mk3(d4.x, d4.y, d4.z);
        const v3 hit = add3(mk3(o4.x, o4.y, o4.z), mul3s(d, h.x));
        const float4* t4 = reinterpret_cast<const float4*>(sv.bvh.tris + ps.hit_slot[slot]);
        const float4 a = t4[0], b = t4[1], c = t4[2];
        const v3 ng = normalize3(cross3(sub3(mk3(b.x, b.y, b.z), mk3(a.x, a.y, a.z)),
                                        sub3(mk3(c.x, c.y, c.z), mk3(a.x, a.y, a.z))));
        const v3 N = dot3(d, ng) < 0.0f ? ng : neg3(ng);
        f[0] = (hit.x - gs.bmin[0]) * gs.binv[0];
        f[1] = (hit.y - gs.bmin[1]) * gs.binv[1];
        f[2] = (hit.z - gs.bmin[2]) * gs.binv[2];
        f[3] = N.x; f[4] = N.y; f[5] = N.z;
        f[6] = -d.x; f[7] = -d.y; f[8] = -d.z;
    }
    __device__ __forceinline__ void output(uint32_t slot, const float (&y)[guide::kOut]) const {
        guide::Mixture m;
        guide::mixture_from_raw(y, m);
        float* mp = gs.mix + 40 * (size_t)slot;
        for (int k = 0; k < guide::kLobes; ++k) {
            mp[k] = m.w[k];
            mp[8 + 3 * k] = m.mu[k][0];
            mp[9 + 3 * k] = m.mu[k][1];
            mp[10 + 3 * k] = m.mu[k][2];
            mp[32 + k] = m.kappa[k];
        }
        if (gs.dump) {  // verification copy of the vertex's inputs and mixture
            const uint32_t i = atomicAdd(gs.dump_count, 1u);
            if (i < gs.dump_cap) {
                float f[9];
                slot_features(slot, f);
                float* o = gs.dump + (size_t)kGuideDumpFloats * i;
                for (int k = 0; k < 9; ++k) o[k] = f[k];
                for (int k = 0; k < 40; ++k) o[9 + k] = mp[k];
            }
        }
    }
};

// The guide's mixture for every vertex of the guided material types, on the tcgen05 tensor cores.
__global__ void __launch_bounds__(guide::TcLayout<guide::kTcGroupsInfer>::kThreads, 1) k_guide_infer(SceneView sv, Paths ps,
                                                                                               GuideState gs) {
    extern __shared__ __align__(1024) unsigned char smem[];
    GuideRows rows{ sv, ps, gs };
    guide::forward_tc_tiles<guide::kTcGroupsInfer>(gs.net, ps.counts[C_GUIDE], rows, ps.counts + C_TC_ERROR, smem);
}

// Per spatial cell (res^3 cells over the scene box) sum and count of the records' weights.
__global__ void k_cell_sums(const float* __restrict__ rec, uint32_t count, uint32_t res, float* __restrict__ sum,
                            uint32_t* __restrict__ cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float* r = rec + 16 * (size_t)i;
        uint32_t c[3];
        for (int k = 0; k < 3; ++k) c[k] = min((uint32_t)fmaxf(r[k] * (float)res, 0.0f), res - 1u);
        const uint32_t cell = (c[2] * res + c[1]) * res + c[0];
        atomicAdd(&sum[cell], r[12]);
        atomicAdd(&cnt[cell], 1u);
    }
}

// Divides each record's weight by its cell's mean weight, so every region of the scene has a comparable
// share of the loss however bright it is.
__global__ void k_cell_normalize(float* __restrict__ rec, uint32_t count, uint32_t res, const float* __restrict__ sum,
                                 const uint32_t* __restrict__ cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        float* r = rec + 16 * (size_t)i;
        uint32_t c[3];
        for (int k = 0; k < 3; ++k) c[k] = min((uint32_t)fmaxf(r[k] * (float)res, 0.0f), res - 1u);
        const uint32_t cell = (c[2] * res + c[1]) * res + c[0];
        const float mean = sum[cell] / (float)cnt[cell];
        if (mean > 0.0f) r[12] = r[12] / mean;
    }
}

// log2 histogram of the training records' weights (64 bins, exponent -32 .. 31)
__global__ void k_weight_hist(const float* __restrict__ rec, uint32_t count, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[64];
    if (threadIdx.x < 64) h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int e = (int)((__float_as_uint(rec[16 * (size_t)i + 12]) >> 23) & 0xFFu) - 127;
        atomicAdd(&h[min(max(e + 32, 0), 63)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 64 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// a training batch drawn uniformly from the records, weights clamped at `clamp`
__global__ void k_gather_batch(const float* __restrict__ src, uint32_t count, float* __restrict__ dst, uint32_t batch,
                               uint32_t salt, float clamp) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const uint32_t j = hash32(i * 0x27d4eb2du + salt) % count;
    const float4* s4 = reinterpret_cast<const float4*>(src + 16 * (size_t)j);
    float4* d4 = reinterpret_cast<float4*>(dst + 16 * (size_t)i);
    d4[0] = s4[0];
    d4[1] = s4[1];
    d4[2] = s4[2];
    float4 w = s4[3];
    w.x = fminf(w.x, clamp);
    d4[3] = w;
}

// ---- finish: add the vertex's MIS estimate, then re-queue or splat --------------------------------

template <class Ctx>
__global__ void k_finish(const __grid_constant__ Ctx ctx, Paths ps, GuideState gs, uint32_t cur) {
    const uint32_t n = ps.counts[C_SHADED];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        PB2_CHECK(n <= ctx.capacity(), 20, K_FINISH, 0, n);
        const uint32_t slot = ps.shaded_q[i];
        PB2_CHECK(slot < ctx.capacity(), 21, K_FINISH, slot, i);
        const LaunchParams& lp = ctx.P(slot);
        const SceneView& sv = ctx.S(slot);
        const uint32_t flags = ps.flags[slot];
        PB2_CHECK(!(flags & 4u) || __float_as_uint(ps.mhit[slot].y) == kInvalidPrim ||
                      ((__float_as_uint(ps.mhit[slot].y) & kPlaneFlag)
                           ? (__float_as_uint(ps.mhit[slot].y) & ~kPlaneFlag) < sv.bvh.plane_count
                           : __float_as_uint(ps.mhit[slot].y) < sv.bvh.tri_count),
                  22, K_FINISH, slot, __float_as_uint(ps.mhit[slot].y));
        if (flags & 1u) {
            const float4 nee = ps.nee[slot];
            spec part_a = sp_zero();
            if (nee.w != 0.0f && ps.occ[slot] == 0u) part_a = mksp(nee.x, nee.y, nee.z);
            spec part_b = sp_zero();
            if (flags & 4u) {
                const float4 mh = ps.mhit[slot];
                const uint32_t prim = __float_as_uint(mh.y);
                const float2 mp = ps.mr_pdf[slot];
                const uint32_t sel = __float_as_uint(mp.y);
                const float4 md = ps.mr_d[slot];
                const v3 dir = mk3(md.x, md.y, md.z);
                const bool missing = prim == kInvalidPrim;
                bool is_sel_light = false;
                uint32_t light = 0;
                if (!missing && (prim & kPlaneFlag)) {
                    light = sv.bvh.planes[prim & ~kPlaneFlag].light;
                    is_sel_light = sel != 0 && light == sel - 1;
                }
                if (is_sel_light || missing) {
                    spec rad;
                    float pdf;
                    if (missing) {
                        rad = mksp(lp.env[0], lp.env[1], lp.env[2]);
                        pdf = sp_valid(rad) ? env_pdf(dir) : 0.0f;
                    } else {
                        const DevPlane& pl = sv.bvh.planes[prim & ~kPlaneFlag];
                        const v3 dn = normalize3(dir);
                        const v3 nrm = mk3(pl.normal[0], pl.normal[1], pl.normal[2]);
                        const v3 N = dot3(dn, nrm) > 0.0f ? neg3(nrm) : nrm;
                        const DevLight& L = sv.lights[light];
                        rad = dot3(N, dir) < 0.0f ? mksp(L.radiance[0], L.radiance[1], L.radiance[2]) : sp_zero();
                        pdf = mh.x * mh.x / (fabsf(dot3(N, dir)) * L.area);
                    }
                    if (sp_valid(rad) && pdf > 0.0f) {
                        const float4 mf = ps.mr_f[slot];
                        const float weight = mf.w * power_heuristic(mp.x, pdf);
                        part_b = sp_muls(sp_mul(rad, mksp(mf.x, mf.y, mf.z)), weight);
                    }
                }
            }
            const float4 mpf = ps.mis_pf[slot];
            const spec mis = sp_divs(sp_add(part_a, part_b), mpf.w);
            const float4 r = ps.rad[slot];
            const spec sample = sp_add(mksp(r.x, r.y, r.z), sp_mul(mksp(mpf.x, mpf.y, mpf.z), mis));
            ps.rad[slot] = make_float4(sample.r, sample.g, sample.b, 0.0f);
        }
        if (flags & 8u) gs.rec[((gs.nrec[slot] - 1u) * 5 + 4) * gs.cap + slot] = ps.rad[slot];
        if (flags & 2u) {
            ps.ext[cur ^ 1][warp_push(&ps.counts[C_EXT_NEXT])] = slot;
        } else {
            if (gs.enabled) flush_records(gs, slot, ps.rad[slot]);
            terminate_path(ctx, ps, slot, cur);
        }
    }
}

// ---- batched launches: slot regeneration from one global path index space ------------------------

__global__ void k_batch_init(Paths ps, uint32_t cap, BatchState* st, unsigned long long total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cap) {
        ps.scene[i] = 0;
    }
    if (i < (cap + 31) / 32) ps.free_bits[i] = cap - 32 * i >= 32 ? 0xFFFFFFFFu : (1u << (cap - 32 * i)) - 1u;
    if (i == 0) {
        ps.counts[C_FREE] = cap;
        st->next = 0;
        st->total = total;
        st->claim_count = 0;
    }
}

// Start of the timed region of a batched render (the per-scene completion times are relative to it).
__global__ void k_batch_clock(BatchState* st) { st->t_start = globaltimer(); }

// Claims min(free slots, paths left) new paths for the iteration and reserves their extend-queue places;
// clears the traversal work counters of the iteration.
__global__ void k_batch_claim(Paths ps, BatchState* st, uint32_t* work) {
    const uint32_t f = ps.counts[C_FREE];  // free slots; those not claimed now stay free
    const unsigned long long left = st->total - st->next;
    const uint32_t m = left < (unsigned long long)f ? (uint32_t)left : f;
    ps.counts[C_FREE] = f - m;
    st->claim_begin = st->next;
    st->claim_count = m;
    st->next += m;
    st->claim_base = ps.counts[C_EXT_CUR];
    ps.counts[C_EXT_CUR] += m;
    work[0] = work[1] = work[2] = 0;
}

// The claimed paths' slots: claim i (of m) goes to the free slot of rank i in slot order, so that consecutive claims
// take ascending slots and a warp's new paths share cache lines of the path state (slots freed one by one scatter over
// the slot range; handing them out in the order they were freed made every state access of a refilled path a separate
// line: the path-state kernels of a refilled launch took 1.25-1.54x as long); start(i, slot) starts the path.  A warp
// owns one 32-slot word of the bitmap at a time and clears the bits it claims.
template <class Start>
__device__ __forceinline__ void for_claimed_slots(const Paths& ps, uint32_t cur, uint32_t m, uint32_t capacity,
                                                  const Start& start) {
    if (m == 0u) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t words = (capacity + 31u) / 32u;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < words; w += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t word = ps.free_bits[w];
        const uint32_t base = ps.free_block[w >> 10] + ps.free_scan[w];
        if (word == 0u || base >= m) continue;  // the same for the whole warp
        const uint32_t rank = base + __popc(word & ((1u << lane) - 1u));
        const bool claimed = ((word >> lane) & 1u) && rank < m;
        const uint32_t taken = __ballot_sync(0xFFFFFFFFu, claimed);
        if (lane == 0u) ps.free_bits[w] = word & ~taken;
        if (claimed) start(rank, 32u * w + lane);
    }
}

// Exclusive prefix of the free bits of each word within its block of 1024 words, and each block's total.
__global__ void __launch_bounds__(1024) k_free_scan(Paths ps, uint32_t words, const BatchState* st) {
    if (st->claim_count == 0u) return;
    __shared__ uint32_t part[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t w = blockIdx.x * 1024u + threadIdx.x;
    const uint32_t v = w < words ? (uint32_t)__popc(ps.free_bits[w]) : 0u;
    uint32_t x = v;
    for (uint32_t o = 1; o < 32u; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31u) part[warp] = x;
    __syncthreads();
    if (warp == 0u) {
        const uint32_t t = part[lane];
        uint32_t z = t;
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, z, o);
            if (lane >= o) z += y;
        }
        part[lane] = z - t;
        if (lane == 31u) ps.free_block[blockIdx.x] = z;
    }
    __syncthreads();
    if (w < words) ps.free_scan[w] = part[warp] + x - v;
}

// Exclusive prefix of the blocks' totals, in place (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) k_free_scan_blocks(Paths ps, uint32_t blocks, const BatchState* st) {
    if (st->claim_count == 0u) return;
    __shared__ uint32_t part[32];
    __shared__ uint32_t carry;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0u;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < blocks; c0 += 1024u) {
        const uint32_t i = c0 + threadIdx.x;
        const uint32_t v = i < blocks ? ps.free_block[i] : 0u;
        uint32_t x = v;
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31u) part[warp] = x;
        __syncthreads();
        if (warp == 0u) {
            const uint32_t t = part[lane];
            uint32_t z = t;
            for (uint32_t o = 1; o < 32u; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, z, o);
                if (lane >= o) z += y;
            }
            part[lane] = z - t;
        }
        __syncthreads();
        const uint32_t e = carry + part[warp] + x - v;
        if (i < blocks) ps.free_block[i] = e;
        __syncthreads();
        if (threadIdx.x == 1023u) carry = e + v;
        __syncthreads();
    }
}

// Starts the claimed paths of a batched iteration (see for_claimed_slots): the same camera path a single-scene
// launch of the full frame starts for that (pixel, sample).
__global__ void k_batch_regen(const __grid_constant__ BatchCtx ctx, Paths ps, uint32_t cur) {
    const BatchState& st = *ctx.state;
    for_claimed_slots(ps, cur, st.claim_count, ctx.capacity(), [&](uint32_t i, uint32_t slot) {
        const unsigned long long g = st.claim_begin + i;
        uint32_t lo = 0, hi = ctx.scene_count;  // last scene with path_begin <= g
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (ctx.scenes[mid].path_begin <= g) lo = mid;
            else hi = mid;
        }
        const BatchScene& sc = ctx.scenes[lo];
        const LaunchParams& lp = sc.lp;
        uint32_t sx, sy, smp;
        path_coords(lp, (uint32_t)(g - sc.path_begin), sx, sy, smp);
        uint64_t index;
        float px, py;
        v3 o, d;
        primary_ray(lp, sx, sy, smp, index, px, py, o, d);
        ps.o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
        ps.d[slot] = make_float4(d.x, d.y, d.z, 0.0f);
        ps.pf[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        ps.rad[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.sidx[slot] = index;
        ps.dim[slot] = 5;
        ps.depth[slot] = 0;
        ps.point[slot] = make_float2(px, py);
        ps.scene[slot] = lo;
        ps.ext[cur][st.claim_base + i] = slot;
    });
}

// Starts the paths claimed for iteration `cur` of a single-scene launch in the slots freed by the previous
// iterations (see for_claimed_slots): path g of the launch (p = ((row * rect.width) + col) * sample_count + k),
// appended to the current extend queue.  ps.scene[slot] keeps the path's index for its per-sample output.
__global__ void k_single_regen(LaunchParams lp, Paths ps, GuideState gs, const BatchState* st, uint32_t cur) {
    for_claimed_slots(ps, cur, st->claim_count, lp.path_count, [&](uint32_t i, uint32_t slot) {
        const uint32_t g = (uint32_t)(st->claim_begin + i);
        uint32_t sx, sy, smp;
        path_coords(lp, g, sx, sy, smp);
        uint64_t index;
        float px, py;
        v3 o, d;
        primary_ray(lp, sx, sy, smp, index, px, py, o, d);
        ps.o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
        ps.d[slot] = make_float4(d.x, d.y, d.z, 0.0f);
        ps.pf[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        ps.rad[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.sidx[slot] = index;
        ps.dim[slot] = 5;
        ps.depth[slot] = 0;
        ps.point[slot] = make_float2(px, py);
        ps.scene[slot] = g;
        if (gs.enabled) gs.nrec[slot] = 0;
        ps.ext[cur][st->claim_base + i] = slot;
    });
}

// Per-bounce bookkeeping: next extend queue becomes current; clear per-bounce counters.
__global__ void k_advance(uint32_t* counts) {
    counts[C_EXT_CUR] = counts[C_EXT_NEXT];
    counts[C_EXT_NEXT] = 0;
    counts[C_SHADOW] = 0;
    counts[C_MIS] = 0;
    counts[C_SHADED] = 0;
    counts[C_GUIDE] = 0;
    for (int t = 0; t < kNumSurfaceTypes; ++t) counts[C_SURF0 + t] = 0;
}

__global__ void k_resolve(const float4* __restrict__ rgbw, uint32_t n, float* __restrict__ rgb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = rgbw[i];
    if (v.w != 0.0f) {
        rgb[3 * i] = v.x / v.w;
        rgb[3 * i + 1] = v.y / v.w;
        rgb[3 * i + 2] = v.z / v.w;
    } else {
        rgb[3 * i] = rgb[3 * i + 1] = rgb[3 * i + 2] = 0.0f;
    }
}

}  // namespace pb2

// ====================================================================================================
// host side
// ====================================================================================================
using namespace pb2;

const char* pb2_sobol_table_sha256() { return PB2_SOBOL_TABLE_SHA256; }

// Path slots of a single-scene wavefront unless set otherwise (pb2_pipeline_set_path_slots): 16M slots hold
// about 4.4 GB of path state (and 6.7 GB more when a guide is attached).  Refilled slots serve paths in no
// particular order, which scatters the path state a warp touches, so the bound is set high enough that
// common launches (a 1920 x 1080 frame at 8 spp is 16.6M paths) start all or nearly all paths at once.
constexpr uint32_t kDefaultPathSlots = 1u << 24;

struct pb2_pipeline {
    pb2_accel* accel = nullptr;
    pb2_render_settings settings{};
    pb2_rect full{};
    pb2_ndc_transform ndc{};
    uint32_t log2res = 0;
    DevMaterial* materials = nullptr;
    DevTexture* textures = nullptr;
    uint8_t* texels = nullptr;
    float2* tri_uv = nullptr;
    DevLight* lights = nullptr;
    float* plane_cdf = nullptr;
    float* plane_pdf = nullptr;
    uint32_t num_lights = 0;
    uint32_t material_count = 0;
    uint32_t type_mask = 0;  // surface types of the scene's materials: the shading kernels launched per bounce
    float env[3] = { 0, 0, 0 };
    float gauss_sub = 0.0f;
    // path state: at most `path_slots` paths are in flight; a launch with more refills freed slots
    uint32_t path_slots = kDefaultPathSlots;
    BatchState* refill = nullptr;  // claim state of the slot refill (device memory)
    unsigned long long* trace_counters = nullptr;  // counting on (pb2_pipeline_set_counting): 9 counters
    uint32_t capacity = 0;
    void* state = nullptr;
    Paths ps{};
    pb2_launch_stats stats{};
    int sms = 0;
    // scene box (guide input normalisation)
    float bmin[3] = { 0, 0, 0 }, binv[3] = { 1, 1, 1 };
    // attached guide and its per-slot / training buffers
    pb2_guide* guide = nullptr;
    pb2_guide_settings guide_settings{};
    uint32_t guide_cap = 0;
    void* guide_state = nullptr;
    float* g_dump = nullptr;  // optional verification rows (pb2_pipeline_set_guide_dump), caller's memory
    uint32_t* g_dump_count = nullptr;
    uint32_t g_dump_cap = 0;
    float* g_mix = nullptr;
    float4* g_rec = nullptr;
    uint32_t* g_nrec = nullptr;
    float* g_train = nullptr;
    float* g_batch = nullptr;
    uint32_t* g_count = nullptr;
    uint32_t g_train_capacity = 0, g_batch_capacity = 0;
    uint32_t g_offered = 0;  // records offered by the launches since the last training call (host estimate)
    uint32_t g_salt = 0;
    // CUDA graphs of the bounce loop (pb2_pipeline_set_graphs): 0 refills freed slots, 1 drains; the stream
    // they are captured on
    bool use_graphs = true;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t gexec[2] = { nullptr, nullptr };
};

static int alloc_guide_slots(pb2_pipeline* pl, uint32_t cap) {
    if (pl->guide_cap >= cap) return PB2_OK;
    cudaFree(pl->guide_state);
    pl->guide_state = nullptr;
    pl->guide_cap = 0;
    const size_t c = cap;
    const size_t mix = ((c * 40 * 4 + 255) / 256) * 256, rec = ((c * kMaxRecords * 5 * 16 + 255) / 256) * 256;
    cudaError_t e = cudaMalloc(&pl->guide_state, mix + rec + c * 4);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc guide path state");
    char* p = static_cast<char*>(pl->guide_state);
    pl->g_mix = reinterpret_cast<float*>(p);
    pl->g_rec = reinterpret_cast<float4*>(p + mix);
    pl->g_nrec = reinterpret_cast<uint32_t*>(p + mix + rec);
    pl->guide_cap = cap;
    return PB2_OK;
}

static size_t infer_smem() { return guide::forward_tc_smem<guide::kTcGroupsInfer>(); }

// Carves the SoA path state of `c` slots out of `base` (or only measures it when base is null); returns the
// bytes used.  `batch` adds the per-slot scene ids (or path indices) and the free-slot bitmap with its prefix sums.
static size_t carve_paths(char* base, size_t c, bool batch, Paths& s) {
    char* p = base;
    auto carve = [&](size_t b) {
        void* r = p;
        p += ((b + 255) / 256) * 256;
        return r;
    };
    s.o = (float4*)carve(c * 16); s.d = (float4*)carve(c * 16); s.pf = (float4*)carve(c * 16);
    s.rad = (float4*)carve(c * 16); s.hit = (float4*)carve(c * 16); s.mis_pf = (float4*)carve(c * 16);
    s.nee = (float4*)carve(c * 16); s.sh_o = (float4*)carve(c * 16); s.sh_d = (float4*)carve(c * 16);
    s.mr_o = (float4*)carve(c * 16); s.mr_d = (float4*)carve(c * 16); s.mr_f = (float4*)carve(c * 16);
    s.mhit = (float4*)carve(c * 16);
    s.sidx = (unsigned long long*)carve(c * 8);
    s.dim = (uint32_t*)carve(c * 4);
    s.depth = (uint32_t*)carve(c * 4);
    s.point = (float2*)carve(c * 8);
    s.hit_slot = (uint32_t*)carve(c * 4);
    s.mr_pdf = (float2*)carve(c * 8);
    s.flags = (uint32_t*)carve(c * 4);
    s.occ = (uint32_t*)carve(c * 4);
    s.ext[0] = (uint32_t*)carve(c * 4);
    s.ext[1] = (uint32_t*)carve(c * 4);
    for (int t = 0; t < kNumSurfaceTypes; ++t) s.surf[t] = (uint32_t*)carve(c * 4);
    s.shadow_q = (uint32_t*)carve(c * 4);
    s.mis_q = (uint32_t*)carve(c * 4);
    s.shaded_q = (uint32_t*)carve(c * 4);
    s.guide_q = (uint32_t*)carve(c * 4);
    s.counts = (uint32_t*)carve(sizeof(uint32_t) * C_COUNT);
    if (batch) {
        s.scene = (uint32_t*)carve(c * 4);
        const size_t words = (c + 31) / 32;
        s.free_bits = (uint32_t*)carve(words * 4);
        s.free_scan = (uint32_t*)carve(words * 4);
        s.free_block = (uint32_t*)carve(((words + 1023) / 1024 + 1) * 4);
    } else {
        s.scene = nullptr;
        s.free_bits = s.free_scan = s.free_block = nullptr;
    }
    return (size_t)(p - base);
}

static int alloc_path_state(void** mem, uint32_t* capacity, Paths* ps, uint32_t cap, bool batch) {
    if (*capacity >= cap) return PB2_OK;
    cudaFree(*mem);
    *mem = nullptr;
    *capacity = 0;
    Paths probe{};
    const size_t bytes = carve_paths(nullptr, cap, batch, probe);
    cudaError_t e = cudaMalloc(mem, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc path state");
    carve_paths(static_cast<char*>(*mem), cap, batch, *ps);
    *capacity = cap;
    return PB2_OK;
}

static int alloc_paths(pb2_pipeline* pl, uint32_t cap) {
    // with the refill arrays (per-slot path index, free-slot bitmap)
    return alloc_path_state(&pl->state, &pl->capacity, &pl->ps, cap, true);
}

// The scene's textures and the materials' references to them: kinds, channels (a color takes 4, a roughness 1, as
// the reference's loadTexture(desc, 4 / 1) demands, Surface/Classic/Classic.cpp), image sizes and texels.
static int check_textures(const pb2_scene* scene) {
    if (scene->texture_count && !scene->textures) return fail(PB2_ERR_INVALID_ARGUMENT, "textures: null array");
    for (uint32_t i = 0; i < scene->texture_count; ++i) {
        const pb2_texture& t = scene->textures[i];
        const std::string name = "texture " + std::to_string(i);
        if (t.channel != 1 && t.channel != 2 && t.channel != 4)
            return fail(PB2_ERR_INVALID_ARGUMENT, name + ": channel must be 1, 2 or 4");
        if (t.kind == PB2_TEXTURE_IMAGE) {
            if (!t.width || !t.height || !t.texels || t.wrap > PB2_WRAP_MIRROR)
                return fail(PB2_ERR_INVALID_ARGUMENT, name + ": an image needs a size, texels and a wrap mode");
            if ((uint64_t)t.width * t.height * t.channel > 0xFFFFFFFFull)
                return fail(PB2_ERR_NOT_SUPPORTED, name + ": more than 2^32 bytes of texels");
        } else if (t.kind != PB2_TEXTURE_CHECKERBOARD) {
            return fail(PB2_ERR_INVALID_ARGUMENT, name + ": unknown kind");
        }
    }
    static const char* params[4] = { "color0", "color1", "roughness[0]", "roughness[1]" };
    for (uint32_t m = 0; m < scene->material_count; ++m)
        for (int k = 0; k < 4; ++k) {
            const uint32_t ti = scene->materials[m].texture[k];
            if (!ti) continue;
            const std::string where = "material " + std::to_string(m) + " " + params[k];
            if (ti > scene->texture_count) return fail(PB2_ERR_INVALID_ARGUMENT, where + ": texture index out of range");
            const uint32_t want = k < 2 ? 4u : 1u;
            if (scene->textures[ti - 1].channel != want)
                return fail(PB2_ERR_INVALID_ARGUMENT, where + ": mismatched channel, expect " + std::to_string(want) +
                                                          ", but get " + std::to_string(scene->textures[ti - 1].channel));
        }
    return PB2_OK;
}

static float remap_roughness(float roughness) {
    const float x = std::log(std::fmax(1e-3f, roughness));
    return std::fmax(1e-3f, 1.62142f + (0.819955f + (0.1734f + (0.0171201f + 0.000640711f * x) * x) * x) * x);
}

// Textures (texels pooled in one device buffer) and, when a material samples one, each triangle's three texture
// coordinates in index order ((0, 0) for a mesh without texcoords).  The upload is stream-ordered; the caller
// synchronises before the host vectors go out of scope.
static int upload_textures(pb2_pipeline* pl, const pb2_scene* scene, cudaStream_t stream) {
    bool textured = false;
    for (uint32_t m = 0; m < scene->material_count; ++m)
        for (int k = 0; k < 4; ++k) textured |= scene->materials[m].texture[k] != 0;
    if (!textured) return PB2_OK;
    size_t bytes = 0;
    std::vector<size_t> offset(scene->texture_count, 0);
    for (uint32_t i = 0; i < scene->texture_count; ++i) {
        const pb2_texture& t = scene->textures[i];
        if (t.kind != PB2_TEXTURE_IMAGE) continue;
        offset[i] = bytes;
        bytes += ((size_t)t.width * t.height * t.channel + 15) & ~(size_t)15;
    }
    cudaError_t e;
    if (bytes && (e = cudaMalloc(&pl->texels, bytes))) return cuda_fail(e, "texel upload");
    std::vector<DevTexture> dev(scene->texture_count ? scene->texture_count : 1);
    for (uint32_t i = 0; i < scene->texture_count; ++i) {
        const pb2_texture& t = scene->textures[i];
        DevTexture& d = dev[i];
        std::memset(&d, 0, sizeof(d));
        d.kind = t.kind;
        d.channel = t.channel;
        d.wrap = t.wrap;
        d.width = t.width;
        d.height = t.height;
        d.scale = t.scale;
        for (int k = 0; k < 4; ++k) { d.black[k] = t.black[k]; d.white[k] = t.white[k]; }
        if (t.kind == PB2_TEXTURE_IMAGE) {
            d.texels = pl->texels + offset[i];
            if ((e = cudaMemcpyAsync(pl->texels + offset[i], t.texels, (size_t)t.width * t.height * t.channel,
                                     cudaMemcpyHostToDevice, stream)))
                return cuda_fail(e, "texel upload");
        }
    }
    uint64_t ntri = 0;
    for (uint32_t m = 0; m < scene->mesh_count; ++m) ntri += scene->meshes[m].tri_count;
    std::vector<float2> uv(3 * (ntri ? ntri : 1), make_float2(0.0f, 0.0f));
    size_t k = 0;
    for (uint32_t m = 0; m < scene->mesh_count; ++m) {
        const pb2_mesh& me = scene->meshes[m];
        for (uint32_t i = 0; i < me.tri_count; ++i, k += 3)
            if (me.texcoords)
                for (int j = 0; j < 3; ++j) {
                    const uint32_t vi = me.indices[3 * i + j];
                    uv[k + j] = make_float2(me.texcoords[2 * vi], me.texcoords[2 * vi + 1]);
                }
    }
    if ((e = cudaMalloc(&pl->textures, sizeof(DevTexture) * dev.size())) ||
        (e = cudaMalloc(&pl->tri_uv, sizeof(float2) * uv.size())) ||
        (e = cudaMemcpyAsync(pl->textures, dev.data(), sizeof(DevTexture) * dev.size(), cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemcpyAsync(pl->tri_uv, uv.data(), sizeof(float2) * uv.size(), cudaMemcpyHostToDevice, stream)) ||
        (e = cudaStreamSynchronize(stream)))
        return cuda_fail(e, "texture upload");
    return PB2_OK;
}

extern "C" {

int pb2_sobol_generate(const uint64_t* idx, const uint32_t* dim, uint32_t n, float* out, void* stream) {
    if (n == 0) return PB2_OK;
    if (!idx || !dim || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_sobol_generate: null argument");
    k_sobol_generate<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(idx, dim, n, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "k_sobol_generate");
}

int pb2_sobol_start(uint32_t log2_resolution, const uint32_t* pixel_sample, uint32_t n, uint64_t* index, float* offset,
                    void* stream) {
    if (n == 0) return PB2_OK;
    if (!pixel_sample || !index || !offset) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_sobol_start: null argument");
    if (log2_resolution > PB2_SOBOL_VDC_LEVELS) return fail(PB2_ERR_NOT_SUPPORTED, "pb2_sobol_start: resolution > 2^25");
    k_sobol_start<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(log2_resolution, pixel_sample, n, index,
                                                                                   offset);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "k_sobol_start");
}

int pb2_pipeline_create(const pb2_scene* scene, const pb2_render_settings* st, void* stream_ptr, pb2_pipeline** out) {
    if (!scene || !st || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_create: null argument");
    *out = nullptr;
    if (st->scramble > 1)
        return fail(PB2_ERR_INVALID_ARGUMENT, "scramble must be 0 (none, the reference's sampler) or 1 (Owen)");
    if (st->width == 0 || st->height == 0) return fail(PB2_ERR_INVALID_ARGUMENT, "empty film");
    if (st->samples_per_pixel == 0 || (st->samples_per_pixel & (st->samples_per_pixel - 1)))
        return fail(PB2_ERR_INVALID_ARGUMENT, "samples_per_pixel must be a power of two (the sampler rounds it up)");
    if (5ull + 8ull * st->max_depth > PB2_SOBOL_DIMS)
        return fail(PB2_ERR_NOT_SUPPORTED, "max_depth would use Sobol dimensions past 1023 (the reference's "
                                           "mt19937_64 tail is not reproduced)");
    if (st->filter > PB2_FILTER_GAUSSIAN) return fail(PB2_ERR_INVALID_ARGUMENT, "unknown filter");
    for (uint32_t m = 0; m < scene->material_count; ++m)
        if (scene->materials[m].type > PB2_SURFACE_CONDUCTOR) return fail(PB2_ERR_INVALID_ARGUMENT, "unknown surface type");
    if (int rc = check_textures(scene)) return rc;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    auto* pl = new pb2_pipeline();
    int rc = pb2_accel_create(scene, stream_ptr, &pl->accel);
    if (rc) {
        delete pl;
        return rc;
    }
    pl->settings = *st;
    rc = pb2_calc_render_rect(st->width, st->height, st->camera.sensor_size[0] / st->camera.sensor_size[1], st->fit_mode,
                              &pl->ndc, &pl->full);
    if (rc) {
        pb2_pipeline_destroy(pl);
        return rc;
    }
    const uint32_t mx = pl->full.width > pl->full.height ? pl->full.width : pl->full.height;
    pl->log2res = (uint32_t)std::ceil(std::log2((double)mx));
    if (pl->log2res > PB2_SOBOL_VDC_LEVELS) {
        pb2_pipeline_destroy(pl);
        return fail(PB2_ERR_NOT_SUPPORTED, "film larger than 2^25");
    }
    pl->gauss_sub = std::exp(-st->gaussian_alpha);
    {
        float lo[3] = { INFINITY, INFINITY, INFINITY }, hi[3] = { -INFINITY, -INFINITY, -INFINITY };
        for (uint32_t m = 0; m < scene->mesh_count; ++m) {
            const pb2_mesh& me = scene->meshes[m];
            for (uint32_t v = 0; v < me.vert_count; ++v) {
                float x[3];
                pb2_mesh_vertex(me.transform, me.translation, me.vertices + 3 * v, x);
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::fmin(lo[k], x[k]);
                    hi[k] = std::fmax(hi[k], x[k]);
                }
            }
        }
        for (uint32_t i = 0; i < scene->plane_count; ++i) {
            const pb2_plane& pp = scene->planes[i];
            for (int c = 0; c < 4; ++c)
                for (int k = 0; k < 3; ++k) {
                    const float x = pp.origin[k] + ((c & 1) ? pp.u[k] : 0.0f) + ((c & 2) ? pp.v[k] : 0.0f);
                    lo[k] = std::fmin(lo[k], x);
                    hi[k] = std::fmax(hi[k], x);
                }
        }
        for (int k = 0; k < 3; ++k) {
            if (!(lo[k] <= hi[k])) lo[k] = hi[k] = 0.0f;
            const float ext = std::fmax(hi[k] - lo[k], 1e-6f);
            pl->bmin[k] = lo[k] - 1e-3f * ext;
            pl->binv[k] = 1.0f / (ext * 1.002f);
        }
    }
    // materials
    std::vector<DevMaterial> mats(scene->material_count ? scene->material_count : 1);
    for (uint32_t m = 0; m < scene->material_count; ++m) {
        const pb2_material& s = scene->materials[m];
        DevMaterial& d = mats[m];
        std::memset(&d, 0, sizeof(d));
        d.type = s.type;
        for (int k = 0; k < 3; ++k) { d.c0[k] = s.color0[k]; d.c1[k] = s.color1[k]; }
        d.valid0 = s.color0[0] > 0.0f || s.color0[1] > 0.0f || s.color0[2] > 0.0f;
        d.valid1 = s.color1[0] > 0.0f || s.color1[1] > 0.0f || s.color1[2] > 0.0f;
        d.roughness0 = s.roughness[0];
        d.roughness1 = s.roughness[1];
        for (int k = 0; k < 4; ++k) d.tex[k] = s.texture[k];
        if (s.type == PB2_SURFACE_CONDUCTOR) {
            d.ax = d.ay = s.roughness[0];
        } else if (s.type == PB2_SURFACE_PLASTIC) {
            d.ax = d.ay = remap_roughness(s.roughness[0]);
        } else {
            d.ax = remap_roughness(s.roughness[0]);
            d.ay = remap_roughness(s.roughness[1]);
        }
        // OrenNayar (Classic/Kernel.cpp:103-109)
        const float sigma = s.roughness[0] * 3.14159265358979323846f;
        const float sigma2 = sigma * sigma;
        d.on_a = 1.0f - (sigma2 / (2.0f * (sigma2 + 0.33f)));
        d.on_b = 0.45f * sigma2 / (sigma2 + 0.09f);
    }
    // lights (AreaLight.cpp, BasicShapes.cpp:76-94)
    std::vector<DevLight> lights(scene->area_light_count ? scene->area_light_count : 1);
    std::vector<float> cdf(scene->plane_count ? scene->plane_count : 1, 0.0f), pdf(cdf.size(), 0.0f);
    for (uint32_t l = 0; l < scene->area_light_count; ++l) {
        const pb2_area_light& al = scene->area_lights[l];
        DevLight& L = lights[l];
        for (int k = 0; k < 3; ++k) { L.radiance[k] = al.radiance[k]; L.translation[k] = al.translation[k]; }
        L.first_plane = al.first_plane;
        L.plane_count = al.plane_count;
        float total = 0.0f;
        for (uint32_t i = 0; i < al.plane_count; ++i) {
            const pb2_plane& p = scene->planes[al.first_plane + i];
            const float d0 = p.u[1] * p.v[2] - p.u[2] * p.v[1];
            const float d1 = p.u[2] * p.v[0] - p.u[0] * p.v[2];
            const float d2 = p.u[0] * p.v[1] - p.u[1] * p.v[0];
            const float area = std::sqrt(std::fmax(d0 * d0 + d1 * d1 + d2 * d2, 0.0f));
            total = total + area;
            cdf[al.first_plane + i] = total;
            pdf[al.first_plane + i] = area;
        }
        for (uint32_t i = 0; i < al.plane_count; ++i) {
            cdf[al.first_plane + i] = cdf[al.first_plane + i] / total;
            pdf[al.first_plane + i] = pdf[al.first_plane + i] / total;
        }
        L.area = total;
        L.inverse_area = 1.0f / total;
    }
    pl->num_lights = scene->area_light_count;
    pl->material_count = scene->material_count;
    for (uint32_t m = 0; m < scene->material_count; ++m) pl->type_mask |= 1u << scene->materials[m].type;
    if (scene->material_count == 0) pl->type_mask = (1u << kNumSurfaceTypes) - 1u;
    for (int k = 0; k < 3; ++k) pl->env[k] = scene->env_radiance[k];
    cudaError_t e;
    if (int rt = upload_textures(pl, scene, stream)) {
        pb2_pipeline_destroy(pl);
        return rt;
    }
    if ((e = cudaMalloc(&pl->materials, sizeof(DevMaterial) * mats.size())) ||
        (e = cudaMalloc(&pl->lights, sizeof(DevLight) * lights.size())) ||
        (e = cudaMalloc(&pl->plane_cdf, sizeof(float) * cdf.size())) ||
        (e = cudaMalloc(&pl->plane_pdf, sizeof(float) * pdf.size())) ||
        (e = cudaMemcpyAsync(pl->materials, mats.data(), sizeof(DevMaterial) * mats.size(), cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemcpyAsync(pl->lights, lights.data(), sizeof(DevLight) * lights.size(), cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemcpyAsync(pl->plane_cdf, cdf.data(), sizeof(float) * cdf.size(), cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemcpyAsync(pl->plane_pdf, pdf.data(), sizeof(float) * pdf.size(), cudaMemcpyHostToDevice, stream))) {
        pb2_pipeline_destroy(pl);
        return cuda_fail(e, "pipeline upload");
    }
    // the Sobol byte tables of this device (same values on every fill, so a fill may overlap other
    // pipelines' renders)
    k_sobol_byte_tables<<<256, 256, 0, stream>>>();
    if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(stream))) {
        pb2_pipeline_destroy(pl);
        return cuda_fail(e, "pipeline set-up");
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&pl->sms, cudaDevAttrMultiProcessorCount, dev);
    *out = pl;
    return PB2_OK;
}

int pb2_pipeline_destroy(pb2_pipeline* pl) {
    if (!pl) return PB2_OK;
    pb2_accel_destroy(pl->accel);
    cudaFree(pl->materials);
    cudaFree(pl->textures);
    cudaFree(pl->texels);
    cudaFree(pl->tri_uv);
    cudaFree(pl->lights);
    cudaFree(pl->plane_cdf);
    cudaFree(pl->plane_pdf);
    cudaFree(pl->state);
    cudaFree(pl->refill);
    cudaFree(pl->trace_counters);
    cudaFree(pl->guide_state);
    cudaFree(pl->g_train);
    cudaFree(pl->g_batch);
    cudaFree(pl->g_count);
    for (cudaGraphExec_t& x : pl->gexec)
        if (x) cudaGraphExecDestroy(x);
    if (pl->cap_stream) cudaStreamDestroy(pl->cap_stream);
    delete pl;
    return PB2_OK;
}

int pb2_pipeline_set_graphs(pb2_pipeline* pl, int enabled) {
    if (!pl) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_graphs: null pipeline");
    pl->use_graphs = enabled != 0;
    return PB2_OK;
}

int pb2_pipeline_get_rect(const pb2_pipeline* pl, pb2_rect* full, pb2_ndc_transform* ndc) {
    if (!pl) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_get_rect: null pipeline");
    if (full) *full = pl->full;
    if (ndc) *ndc = pl->ndc;
    return PB2_OK;
}

static LaunchParams make_params(const pb2_pipeline* pl, const pb2_rect& rect, uint32_t sb, uint32_t sc) {
    LaunchParams lp{};
    lp.rect = rect;
    lp.full = pl->full;
    lp.ndc = pl->ndc;
    lp.width = pl->settings.width;
    lp.height = pl->settings.height;
    lp.log2res = pl->log2res;
    lp.sample_begin = sb;
    lp.sample_count = sc;
    lp.max_depth = pl->settings.max_depth;
    lp.min_rr_depth = pl->settings.min_rr_depth;
    lp.filter = pl->settings.filter;
    lp.gauss_neg_alpha = -pl->settings.gaussian_alpha;
    lp.gauss_sub = pl->gauss_sub;
    lp.cam = pl->settings.camera;
    lp.num_lights = pl->num_lights;
    for (int k = 0; k < 3; ++k) lp.env[k] = pl->env[k];
    lp.path_count = rect.width * rect.height * sc;
    lp.scramble = pl->settings.scramble;
    lp.scramble_seed = pl->settings.scramble_seed;
    static const bool checks = [] {
        const char* v = std::getenv("PB2_DEBUG_CHECKS");
        return v && v[0] == '1';
    }();
    lp.checks = checks ? 1u : 0u;
    return lp;
}

static bool rect_inside(const pb2_rect& r, const pb2_rect& full) {
    return r.width && r.height && r.left >= full.left && r.top >= full.top &&
           (uint64_t)r.left + r.width <= (uint64_t)full.left + full.width &&
           (uint64_t)r.top + r.height <= (uint64_t)full.top + full.height;
}

int pb2_pipeline_camera_rays(pb2_pipeline* pl, const pb2_rect* rect, uint32_t sample, pb2_ray* rays, float* points,
                             void* stream) {
    if (!pl || !rect || !rays || !points) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_camera_rays: null");
    if (!rect_inside(*rect, pl->full)) return fail(PB2_ERR_INVALID_ARGUMENT, "rect outside the render rectangle");
    const LaunchParams lp = make_params(pl, *rect, sample, 1);
    const uint32_t n = rect->width * rect->height;
    k_camera_rays<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(lp, sample, reinterpret_cast<float4*>(rays),
                                                                                   reinterpret_cast<float2*>(points));
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "k_camera_rays");
}

int pb2_pipeline_launch(pb2_pipeline* pl, const pb2_rect* rect, uint32_t sample_begin, uint32_t sample_count,
                        float* rgbw, float* sample_out, void* stream_ptr) {
    if (!pl || !rect) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_launch: null argument");
    if (!rect_inside(*rect, pl->full)) return fail(PB2_ERR_INVALID_ARGUMENT, "rect outside the render rectangle");
    if (sample_count == 0) return PB2_OK;
    if ((uint64_t)sample_begin + sample_count > (1ull << 31))
        return fail(PB2_ERR_INVALID_ARGUMENT, "sample range too large");
    const uint64_t paths = (uint64_t)rect->width * rect->height * sample_count;
    if (paths > 0x7FFFFFFFull) return fail(PB2_ERR_INVALID_ARGUMENT, "launch has more than 2^31 paths");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    // path slots in flight: the whole launch, or at most pl->path_slots (then refilled as paths finish)
    const uint32_t slots = (uint32_t)std::min<uint64_t>(paths, pl->path_slots);
    int rc = alloc_paths(pl, slots);
    if (rc) return rc;
    if (!pl->refill) {
        const cudaError_t ea = cudaMalloc(&pl->refill, sizeof(BatchState));
        if (ea != cudaSuccess) return cuda_fail(ea, "cudaMalloc refill state");
    }
    LaunchParams lp = make_params(pl, *rect, sample_begin, sample_count);
    GuideState gs{};
    if (pl->guide) {
        if (5ull + 9ull * pl->settings.max_depth > PB2_SOBOL_DIMS)
            return fail(PB2_ERR_NOT_SUPPORTED, "guided sampling uses 9 Sobol dimensions per bounce: max_depth too large");
        if ((rc = alloc_guide_slots(pl, slots))) return rc;
        gs.enabled = 1;
        gs.sel_prob = pl->guide_settings.selection_prob;
        gs.types = pl->guide_settings.guided_types;
        gs.max_depth = pl->guide_settings.max_guided_depth ? pl->guide_settings.max_guided_depth : 0xFFFFFFFFu;
        gs.dump = pl->g_dump;
        gs.dump_count = pl->g_dump_count;
        gs.dump_cap = pl->g_dump_cap;
        gs.net = pl->guide->view();
        gs.mix = pl->g_mix;
        gs.rec = pl->g_rec;
        gs.nrec = pl->g_nrec;
        gs.cap = pl->guide_cap;
        gs.train = pl->g_train;
        gs.train_count = pl->g_count;
        gs.train_capacity = pl->g_train_capacity;
        // keep about `capacity` of the records the launches offer between two training calls: the expected
        // count of this launch is estimated from the previous ones (all records are kept at first)
        const double expect = (double)pl->g_offered + (double)paths * 1.5;
        gs.accept_prob = expect > pl->g_train_capacity ? (float)(pl->g_train_capacity / expect) : 1.0f;
        gs.salt = ++pl->g_salt;
        for (int k = 0; k < 3; ++k) { gs.bmin[k] = pl->bmin[k]; gs.binv[k] = pl->binv[k]; }
        static std::atomic<int> attr[kMaxDevices];
        const cudaError_t ea = smem_attr_once((const void*)k_guide_infer, infer_smem(), attr);
        if (ea != cudaSuccess) return cuda_fail(ea, "k_guide_infer shared-memory limit");
    }
    SceneView sv;
    sv.materials = pl->materials;
    sv.textures = pl->textures;
    sv.tri_uv = pl->tri_uv;
    sv.prim_material = pl->accel->prim_material;
    sv.lights = pl->lights;
    sv.plane_cdf = pl->plane_cdf;
    sv.plane_pdf = pl->plane_pdf;
    sv.bvh = pl->accel->view;
    sv.material_count = pl->material_count;
    Paths ps = pl->ps;
    float4* film = reinterpret_cast<float4*>(rgbw);
    cudaError_t e;
    // every slot starts free; each bounce first refills the slots freed by the previous one from the launch's
    // remaining paths (k_batch_claim + k_single_regen), so the wavefront stays full until the paths run out
    lp.path_count = slots;
    lp.refill = slots < paths ? 1u : 0u;
    if ((e = cudaMemsetAsync(ps.counts, 0, sizeof(uint32_t) * C_COUNT, stream))) return cuda_fail(e, "memset counts");
    k_batch_init<<<(slots + 255) / 256, 256, 0, stream>>>(ps, slots, pl->refill, paths);
    const int grid = pl->sms * 8;
    uint32_t* work = pl->accel->work;
    unsigned long long* stats = reinterpret_cast<unsigned long long*>(ps.counts + C_STAT_CLOSEST);
    unsigned long long* sstats = reinterpret_cast<unsigned long long*>(ps.counts + C_STAT_SHADOW);
    static std::atomic<int> qcache[kMaxDevices], qcache_any[kMaxDevices];
    const int qblocks = resident_grid_cached((const void*)k_trace_queue<Q_EXTEND, SingleCtx>, kQThreads, 0, qcache);
    const int qblocks_any =
        resident_grid_cached((const void*)k_trace_queue<Q_SHADOW, SingleCtx>, kQThreads, 0, qcache_any);
    // generous bound: every path needs at most (max depth + light pass-throughs) bounces, and a slot serves
    // about paths / slots of them one after another
    const uint64_t max_bounces = (paths / slots + 2) * (4ull * (pl->settings.max_depth + 2) + 64);
    // PB2_DEBUG_SYNC=1: synchronise after every kernel and name the one that failed
    static const bool debug_sync = [] {
        const char* v = std::getenv("PB2_DEBUG_SYNC");
        return v && v[0] == '1';
    }();
    const char* failed = nullptr;
    auto checked = [&](const char* name) {
        if (!debug_sync || failed) return;
        cudaError_t err = cudaGetLastError();
        if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
        if (err != cudaSuccess) {
            failed = name;
            e = err;
        }
    };
    checked("k_batch_init");
    SingleCtx ctx;
    ctx.lp = lp;
    ctx.sv = sv;
    ctx.film = film;
    ctx.sample_out = sample_out;
    // The bounce kernels read their queue sizes on the device, so the host checks for completion only
    // every kCheckEvery bounces (a bounce with empty queues costs only its launches) and the launches of
    // the bounces between checks queue up without a host round trip.
    constexpr int kCheckEvery = 4;
    // one bounce on stream `s` with extend-queue parity `c`; `refill_step` first starts the launch's next paths in
    // the slots the previous bounce freed
    auto bounce = [&](cudaStream_t s, bool refill_step, uint32_t c) {
        if (refill_step) {
            k_batch_claim<<<1, 1, 0, s>>>(ps, pl->refill, work);  // also clears the trace work counters
            k_free_scan<<<(slots + 32767) / 32768, 1024, 0, s>>>(ps, (slots + 31) / 32, pl->refill);
            k_free_scan_blocks<<<1, 1024, 0, s>>>(ps, (slots + 32767) / 32768, pl->refill);
            k_single_regen<<<grid, 256, 0, s>>>(lp, ps, gs, pl->refill, c);
            checked("k_single_regen");
        } else {
            cudaMemsetAsync(work, 0, sizeof(uint32_t) * 3, s);
        }
        // the persistent trace blocks stop when the queue is drained
        const int qgrid = qblocks;
        if (pl->trace_counters)
            k_trace_queue<Q_EXTEND, SingleCtx, true><<<qgrid, kQThreads, 0, s>>>(
                ctx, ps, ps.ext[c], ps.counts + C_EXT_CUR, work, stats, pl->trace_counters);
        else
            k_trace_queue<Q_EXTEND><<<qgrid, kQThreads, 0, s>>>(ctx, ps, ps.ext[c], ps.counts + C_EXT_CUR, work,
                                                                     stats);
        checked("k_trace_queue<extend>");
        k_classify<<<grid, 256, 0, s>>>(ctx, ps, gs, c);
        checked("k_classify");
        if (gs.enabled)
            k_guide_infer<<<pl->sms, guide::TcLayout<guide::kTcGroupsInfer>::kThreads, infer_smem(), s>>>(sv, ps, gs);
        checked("k_guide_infer");
        // one shading kernel per surface type the scene's materials use (the others' queues stay empty)
        const uint32_t tm = pl->type_mask;
        if (tm & (1u << PB2_SURFACE_MATTE)) {
            k_shade<PB2_SURFACE_MATTE><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            if (gs.enabled && ((gs.types >> PB2_SURFACE_MATTE) & 1u))
                k_shade<PB2_SURFACE_MATTE, SingleCtx, true><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<matte>");
        }
        if (tm & (1u << PB2_SURFACE_PLASTIC)) {
            k_shade<PB2_SURFACE_PLASTIC><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<plastic>");
        }
        if (tm & (1u << PB2_SURFACE_GLASS)) {
            k_shade<PB2_SURFACE_GLASS><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<glass>");
        }
        if (tm & (1u << PB2_SURFACE_MIRROR)) {
            k_shade<PB2_SURFACE_MIRROR><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<mirror>");
        }
        if (tm & (1u << PB2_SURFACE_SUBSTRATE)) {
            k_shade<PB2_SURFACE_SUBSTRATE><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<substrate>");
        }
        if (tm & (1u << PB2_SURFACE_CONDUCTOR)) {
            k_shade<PB2_SURFACE_CONDUCTOR><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            if (gs.enabled && ((gs.types >> PB2_SURFACE_CONDUCTOR) & 1u))
                k_shade<PB2_SURFACE_CONDUCTOR, SingleCtx, true><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<conductor>");
        }
        if (tm & (1u << PB2_SURFACE_BLACKBODY)) {
            k_shade<PB2_SURFACE_BLACKBODY><<<grid, 128, 0, s>>>(ctx, ps, gs, c);
            checked("k_shade<blackbody>");
        }
        if (pl->trace_counters)
            k_trace_queue<Q_SHADOW, SingleCtx, true><<<qblocks_any, kQThreads, 0, s>>>(
                ctx, ps, ps.shadow_q, ps.counts + C_SHADOW, work + 1, sstats, pl->trace_counters);
        else
            k_trace_queue<Q_SHADOW><<<qblocks_any, kQThreads, 0, s>>>(ctx, ps, ps.shadow_q, ps.counts + C_SHADOW,
                                                                           work + 1, sstats);
        checked("k_trace_queue<shadow>");
        if (pl->trace_counters)
            k_trace_queue<Q_MIS, SingleCtx, true><<<qblocks_any, kQThreads, 0, s>>>(
                ctx, ps, ps.mis_q, ps.counts + C_MIS, work + 2, stats, pl->trace_counters);
        else
            k_trace_queue<Q_MIS><<<qblocks_any, kQThreads, 0, s>>>(ctx, ps, ps.mis_q, ps.counts + C_MIS, work + 2,
                                                                        stats);
        checked("k_trace_queue<mis>");
        k_finish<<<grid, 256, 0, s>>>(ctx, ps, gs, c);
        checked("k_finish");
        k_advance<<<1, 1, 0, s>>>(ps.counts);
        checked("k_advance");
    };
    // CUDA graphs of kCheckEvery bounces (parities 0, 1, 0, 1; graph 0 refills, graph 1 drains), captured on the
    // pipeline's own stream for this launch's parameters and updated in place when the pipeline already holds a
    // graph of the same shape.  The first kCheckEvery bounces run as plain launches, and the graph the next ones
    // need is captured while the device runs them.
    const bool graphs = pl->use_graphs && !debug_sync;
    bool captured[2] = { false, false };
    auto capture = [&](int mode) -> cudaError_t {
        cudaError_t err;
        if (!pl->cap_stream && (err = cudaStreamCreateWithFlags(&pl->cap_stream, cudaStreamNonBlocking))) return err;
        if ((err = cudaStreamBeginCapture(pl->cap_stream, cudaStreamCaptureModeThreadLocal))) return err;
        for (int k = 0; k < kCheckEvery; ++k) bounce(pl->cap_stream, mode == 0, (uint32_t)(k & 1));
        const cudaError_t le = cudaGetLastError();
        cudaGraph_t g = nullptr;
        err = cudaStreamEndCapture(pl->cap_stream, &g);
        if (le != cudaSuccess || err != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return le != cudaSuccess ? le : err;
        }
        if (pl->gexec[mode]) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(pl->gexec[mode], g, &info) != cudaSuccess) {
                cudaGetLastError();  // a graph of another shape: instantiate anew
                cudaGraphExecDestroy(pl->gexec[mode]);
                pl->gexec[mode] = nullptr;
            }
        }
        err = pl->gexec[mode] ? cudaSuccess : cudaGraphInstantiate(&pl->gexec[mode], g, 0);
        cudaGraphDestroy(g);
        if (err == cudaSuccess) captured[mode] = true;
        return err;
    };
    bool refilling = true;
    for (uint64_t group = 0; !failed; ++group) {
        if (group > 0) {
            uint32_t active = 0;
            unsigned long long next = paths;  // once every path has started, only the queue is read
            if ((e = cudaMemcpyAsync(&active, ps.counts + C_EXT_CUR, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                     stream)) ||
                (refilling &&
                 (e = cudaMemcpyAsync(&next, &pl->refill->next, sizeof(next), cudaMemcpyDeviceToHost, stream))) ||
                (e = cudaStreamSynchronize(stream)))
                return cuda_fail(e, "read queue size");
            if (active == 0 && next == paths) break;
            if (next == paths) refilling = false;  // every path has been started
        }
        if (group * kCheckEvery > max_bounces) return fail(PB2_ERR_DEVICE_TIMEOUT, "path loop did not terminate");
        const int mode = refilling ? 0 : 1;
        if (graphs && group > 0) {
            if (!captured[mode] && (e = capture(mode))) return cuda_fail(e, "capture of the bounce graph");
            if ((e = cudaGraphLaunch(pl->gexec[mode], stream))) return cuda_fail(e, "bounce graph launch");
            continue;
        }
        for (int k = 0; k < kCheckEvery && !failed; ++k) {
            bounce(stream, refilling, (uint32_t)(k & 1));
            // all paths fit the slots: the first claim started every one of them
            if (slots == paths) refilling = false;
            if (!failed && (e = cudaGetLastError())) return cuda_fail(e, "bounce launch");
        }
        if (graphs && group == 0 && (e = capture(refilling ? 0 : 1))) return cuda_fail(e, "capture of the bounce graph");
    }
    if (failed) return fail(PB2_ERR_CUDA, std::string(failed) + ": " + cudaGetErrorString(e));
    uint32_t counts[C_COUNT];
    if ((e = cudaMemcpyAsync(counts, ps.counts, sizeof(counts), cudaMemcpyDeviceToHost, stream)) ||
        (e = cudaStreamSynchronize(stream)))
        return cuda_fail(e, "read stats");
    unsigned long long v;
    std::memcpy(&v, counts + C_STAT_CLOSEST, 8);
    pl->stats.closest_rays += v;
    std::memcpy(&v, counts + C_STAT_SHADOW, 8);
    pl->stats.shadow_rays += v;
    std::memcpy(&v, counts + C_STAT_VERTICES, 8);
    pl->stats.path_vertices += v;
    pl->stats.paths += paths;
    if (counts[C_CHECK])
        return fail(PB2_ERR_CUDA, "index check " + std::to_string(counts[C_CHECK]) + " failed in kernel " +
                                      std::to_string(counts[C_CHECK + 1]) + " at slot " +
                                      std::to_string(counts[C_CHECK + 2]) + ", value " +
                                      std::to_string(counts[C_CHECK + 3]));
    if (counts[C_ERROR]) return fail(PB2_ERR_QUEUE_OVERFLOW, "traversal stack overflow");
    if (counts[C_TC_ERROR]) return fail(PB2_ERR_DEVICE_TIMEOUT, "guide inference: a tensor-core wait timed out");
    if (gs.enabled) {
        uint32_t tc[2];
        if ((e = cudaMemcpyAsync(tc, pl->g_count, sizeof(tc), cudaMemcpyDeviceToHost, stream)) ||
            (e = cudaStreamSynchronize(stream)))
            return cuda_fail(e, "read record count");
        pl->g_offered = tc[1];
    }
    return PB2_OK;
}

int pb2_pipeline_set_guide_dump(pb2_pipeline* pl, float* rows_dev, uint32_t capacity, uint32_t* count_dev) {
    if (!pl) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_guide_dump: null pipeline");
    if (rows_dev && (!count_dev || capacity == 0))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_guide_dump: rows need a capacity and a counter");
    pl->g_dump = rows_dev;
    pl->g_dump_count = rows_dev ? count_dev : nullptr;
    pl->g_dump_cap = rows_dev ? capacity : 0;
    return PB2_OK;
}

int pb2_pipeline_set_counting(pb2_pipeline* pl, int enable) {
    if (!pl) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_counting: null pipeline");
    cudaError_t e;
    if (!enable) {
        if ((e = cudaDeviceSynchronize())) return cuda_fail(e, "pb2_pipeline_set_counting");
        cudaFree(pl->trace_counters);
        pl->trace_counters = nullptr;
        return PB2_OK;
    }
    if (!pl->trace_counters && (e = cudaMalloc(&pl->trace_counters, 9 * sizeof(unsigned long long))))
        return cuda_fail(e, "cudaMalloc trace counters");
    if ((e = cudaMemset(pl->trace_counters, 0, 9 * sizeof(unsigned long long)))) return cuda_fail(e, "clear counters");
    return PB2_OK;
}

int pb2_pipeline_get_trace_counters(const pb2_pipeline* pl, uint64_t* counters, void* stream) {
    if (!pl || !counters) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_get_trace_counters: null argument");
    if (!pl->trace_counters) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_get_trace_counters: counting is off");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(counters, pl->trace_counters, 9 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return cuda_fail(e, "read trace counters");
    return PB2_OK;
}

int pb2_pipeline_set_path_slots(pb2_pipeline* pl, uint32_t slots) {
    if (!pl) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_path_slots: null pipeline");
    if (slots < 256 || slots > (1u << 30)) return fail(PB2_ERR_INVALID_ARGUMENT, "path slots must lie in [256, 2^30]");
    pl->path_slots = slots;
    if (pl->capacity > slots) {  // give back path state above the new bound
        cudaFree(pl->state);
        pl->state = nullptr;
        pl->capacity = 0;
        cudaFree(pl->guide_state);
        pl->guide_state = nullptr;
        pl->guide_cap = 0;
    }
    return PB2_OK;
}

int pb2_pipeline_set_guide(pb2_pipeline* pl, pb2_guide* guide, const pb2_guide_settings* settings) {
    if (!pl) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_guide: null pipeline");
    if (!guide) {
        pl->guide = nullptr;
        return PB2_OK;
    }
    if (!settings) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_set_guide: null settings");
    if (!(settings->selection_prob > 0.0f && settings->selection_prob < 1.0f))
        return fail(PB2_ERR_INVALID_ARGUMENT, "selection_prob must lie in (0, 1): the BxDF keeps the estimator unbiased");
    if (settings->record_capacity == 0 || settings->record_capacity > (1u << 26))
        return fail(PB2_ERR_INVALID_ARGUMENT, "record_capacity must lie in [1, 2^26]");
    if (!(settings->weight_quantile >= 0.0f && settings->weight_quantile <= 1.0f))
        return fail(PB2_ERR_INVALID_ARGUMENT, "weight_quantile must lie in [0, 1]");
    if (settings->spatial_cells > 16)
        return fail(PB2_ERR_INVALID_ARGUMENT, "spatial_cells must lie in [0, 16] per axis");
    {
        uint32_t allowed = 0;
        for (int t = 0; t < kNumSurfaceTypes; ++t)
            if (guided_type(t)) allowed |= 1u << t;
        if (settings->guided_types & ~allowed)
            return fail(PB2_ERR_INVALID_ARGUMENT, "guided_types: only Matte and Conductor vertices can be guided "
                                                  "(their BxDFs report their samplers' true density)");
    }
    if (5ull + 9ull * pl->settings.max_depth > PB2_SOBOL_DIMS)
        return fail(PB2_ERR_NOT_SUPPORTED, "guided sampling uses 9 Sobol dimensions per bounce: max_depth too large");
    cudaError_t e;
    if (settings->record_capacity > pl->g_train_capacity) {
        cudaFree(pl->g_train);
        pl->g_train = nullptr;
        pl->g_train_capacity = 0;
        if ((e = cudaMalloc(&pl->g_train, (size_t)settings->record_capacity * 64))) return cuda_fail(e, "cudaMalloc records");
        pl->g_train_capacity = settings->record_capacity;
    }
    if (!pl->g_count) {
        if ((e = cudaMalloc(&pl->g_count, 2 * sizeof(uint32_t)))) return cuda_fail(e, "cudaMalloc record count");
    }
    if ((e = cudaMemset(pl->g_count, 0, 2 * sizeof(uint32_t)))) return cuda_fail(e, "memset record count");
    pl->g_offered = 0;
    pl->guide = guide;
    pl->guide_settings = *settings;
    // default: Matte only.  A glossy conductor's visible-normal sampler is already close to its product with
    // the incident light, and sending half of its samples to a broad guide lobe doubles its variance
    // (measured on the hard-indirect room: relMSE at 128 spp 0.36 guiding both types, 0.27 Matte only).
    if (pl->guide_settings.guided_types == 0) pl->guide_settings.guided_types = 1u << PB2_SURFACE_MATTE;
    return PB2_OK;
}

int pb2_pipeline_train_guide(pb2_pipeline* pl, uint32_t steps, uint32_t batch, float lr, float* loss_host,
                             void* stream_ptr) {
    if (!pl || !pl->guide) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_train_guide: no guide attached");
    if (batch == 0 || batch > (1u << 22)) return fail(PB2_ERR_INVALID_ARGUMENT, "batch must lie in [1, 2^22]");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    cudaError_t e;
    uint32_t tc[2];
    if ((e = cudaMemcpyAsync(tc, pl->g_count, sizeof(tc), cudaMemcpyDeviceToHost, stream)) ||
        (e = cudaStreamSynchronize(stream)))
        return cuda_fail(e, "read record count");
    const uint32_t count = std::min(tc[0], pl->g_train_capacity);
    float loss = 0.0f;
    if (count > 0 && steps > 0) {
        if (batch > pl->g_batch_capacity) {
            cudaFree(pl->g_batch);
            pl->g_batch = nullptr;
            pl->g_batch_capacity = 0;
            if ((e = cudaMalloc(&pl->g_batch, (size_t)batch * 64 + 64 * sizeof(uint32_t) + kMaxCells * 8)))
                return cuda_fail(e, "cudaMalloc batch");
            pl->g_batch_capacity = batch;
        }
        const uint32_t res = pl->guide_settings.spatial_cells;
        if (res > 0) {
            float* csum = reinterpret_cast<float*>(pl->g_batch + (size_t)batch * 16 + 64);
            uint32_t* ccnt = reinterpret_cast<uint32_t*>(csum + kMaxCells);
            if ((e = cudaMemsetAsync(csum, 0, kMaxCells * 8, stream))) return cuda_fail(e, "memset cells");
            k_cell_sums<<<pl->sms * 4, 256, 0, stream>>>(pl->g_train, count, res, csum, ccnt);
            k_cell_normalize<<<pl->sms * 4, 256, 0, stream>>>(pl->g_train, count, res, csum, ccnt);
            if ((e = cudaGetLastError())) return cuda_fail(e, "cell normalisation");
        }
        // weight clamp at the configured quantile of this call's records (log2 bins): a few extreme
        // radiance samples must not dominate a batch's self-normalised loss
        float clamp = 3.0e38f;
        const float q = pl->guide_settings.weight_quantile;
        if (q > 0.0f && q < 1.0f) {
            uint32_t* hist = reinterpret_cast<uint32_t*>(pl->g_batch + (size_t)batch * 16);
            uint32_t h[64];
            if ((e = cudaMemsetAsync(hist, 0, sizeof(h), stream))) return cuda_fail(e, "memset histogram");
            k_weight_hist<<<pl->sms, 256, 0, stream>>>(pl->g_train, count, hist);
            if ((e = cudaMemcpyAsync(h, hist, sizeof(h), cudaMemcpyDeviceToHost, stream)) ||
                (e = cudaStreamSynchronize(stream)))
                return cuda_fail(e, "weight histogram");
            uint64_t cum = 0;
            const uint64_t target = (uint64_t)std::ceil((double)q * count);
            for (int b = 0; b < 64; ++b) {
                cum += h[b];
                if (cum >= target) {
                    clamp = std::ldexp(1.0f, b - 32 + 1);
                    break;
                }
            }
        }
        for (uint32_t s = 0; s < steps; ++s) {
            k_gather_batch<<<(batch + 255) / 256, 256, 0, stream>>>(pl->g_train, count, pl->g_batch, batch,
                                                                    ++pl->g_salt * 0x85ebca6bu, clamp);
            if ((e = cudaGetLastError())) return cuda_fail(e, "k_gather_batch");
            const int rc = pb2_guide_train(pl->guide, pl->g_batch, batch, lr, s + 1 == steps ? &loss : nullptr, stream_ptr);
            if (rc) return rc;
        }
    }
    if ((e = cudaMemsetAsync(pl->g_count, 0, 2 * sizeof(uint32_t), stream)) || (e = cudaStreamSynchronize(stream)))
        return cuda_fail(e, "reset record count");
    pl->g_offered = 0;
    if (loss_host) *loss_host = loss;
    return PB2_OK;
}

int pb2_film_resolve(const float* rgbw, uint32_t n, float* rgb, void* stream) {
    if (n == 0) return PB2_OK;
    if (!rgbw || !rgb) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_film_resolve: null argument");
    k_resolve<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const float4*>(rgbw), n, rgb);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PB2_OK : cuda_fail(e, "k_resolve");
}

int pb2_pipeline_get_stats(const pb2_pipeline* pl, pb2_launch_stats* stats, void*) {
    if (!pl || !stats) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_pipeline_get_stats: null argument");
    *stats = pl->stats;
    return PB2_OK;
}

}  // extern "C"

// ====================================================================================================
// batched multi-scene rendering
// ====================================================================================================

struct pb2_batch {
    std::vector<pb2_pipeline*> pipes;
    std::vector<BatchScene> host_scenes;
    std::vector<size_t> film_offset;  // float4 elements
    BatchScene* scenes = nullptr;
    uint32_t* remaining = nullptr;
    unsigned long long* done_ns = nullptr;
    BatchState* state = nullptr;
    uint32_t* work = nullptr;
    float4* films = nullptr;
    size_t film_elems = 0;
    unsigned long long total_paths = 0;
    // path state
    void* mem = nullptr;
    uint32_t allocated = 0;  // slots the path state was carved for
    uint32_t capacity = 0;   // slots the current config may use (<= allocated)
    Paths ps{};
    pb2_batch_config config{};
    int sms = 0;
    int trace_blocks_max = 0;
    uint32_t type_mask = 0;  // surface types of all scenes' materials
    // the batch's own non-blocking stream: graphs cannot be captured on the legacy default stream
    cudaStream_t own = nullptr;
    // captured graph of two wavefront iterations (cur = 0 then 1) for `graph_config`
    cudaGraphExec_t graph = nullptr;
    pb2_batch_config graph_config{};
    // results of the last render
    std::vector<float> scene_ms;
    float total_ms = 0.0f;
    uint32_t iterations = 0;
    pb2_launch_stats stats{};
};

static void batch_release_graph(pb2_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

static BatchCtx batch_ctx(const pb2_batch* b) {
    BatchCtx c;
    c.scenes = b->scenes;
    c.scene_count = (uint32_t)b->pipes.size();
    c.cap = b->capacity;
    c.check = make_params(b->pipes[0], b->pipes[0]->full, 0, 1).checks;
    c.remaining = b->remaining;
    c.done_ns = b->done_ns;
    c.state = b->state;
    c.scene_of = b->ps.scene;
    return c;
}

// One wavefront iteration over every scene: regenerate freed slots, then one bounce.
static cudaError_t batch_iteration(pb2_batch* b, uint32_t cur, cudaStream_t stream) {
    const BatchCtx ctx = batch_ctx(b);
    const Paths& ps = b->ps;
    GuideState gs{};
    const int grid = b->sms * 8;
    const int sb = (int)b->config.shade_block;
    const int tb = b->sms * (int)b->config.trace_blocks_per_sm;
    unsigned long long* stats = reinterpret_cast<unsigned long long*>(ps.counts + C_STAT_CLOSEST);
    unsigned long long* sstats = reinterpret_cast<unsigned long long*>(ps.counts + C_STAT_SHADOW);
    k_batch_claim<<<1, 1, 0, stream>>>(ps, b->state, b->work);
    k_free_scan<<<(b->capacity + 32767) / 32768, 1024, 0, stream>>>(ps, (b->capacity + 31) / 32, b->state);
    k_free_scan_blocks<<<1, 1024, 0, stream>>>(ps, (b->capacity + 32767) / 32768, b->state);
    k_batch_regen<<<grid, 256, 0, stream>>>(ctx, ps, cur);
    k_trace_queue<Q_EXTEND><<<tb, kQThreads, 0, stream>>>(ctx, ps, ps.ext[cur], ps.counts + C_EXT_CUR, b->work, stats);
    k_classify<<<grid, 256, 0, stream>>>(ctx, ps, gs, cur);
    // shading kernels of the surface types some scene of the batch uses
    const uint32_t tm = b->type_mask;
    if (tm & (1u << PB2_SURFACE_MATTE)) k_shade<PB2_SURFACE_MATTE><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    if (tm & (1u << PB2_SURFACE_PLASTIC)) k_shade<PB2_SURFACE_PLASTIC><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    if (tm & (1u << PB2_SURFACE_GLASS)) k_shade<PB2_SURFACE_GLASS><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    if (tm & (1u << PB2_SURFACE_MIRROR)) k_shade<PB2_SURFACE_MIRROR><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    if (tm & (1u << PB2_SURFACE_SUBSTRATE))
        k_shade<PB2_SURFACE_SUBSTRATE><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    if (tm & (1u << PB2_SURFACE_CONDUCTOR))
        k_shade<PB2_SURFACE_CONDUCTOR><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    if (tm & (1u << PB2_SURFACE_BLACKBODY))
        k_shade<PB2_SURFACE_BLACKBODY><<<grid, sb, 0, stream>>>(ctx, ps, gs, cur);
    k_trace_queue<Q_SHADOW><<<tb, kQThreads, 0, stream>>>(ctx, ps, ps.shadow_q, ps.counts + C_SHADOW, b->work + 1, sstats);
    k_trace_queue<Q_MIS><<<tb, kQThreads, 0, stream>>>(ctx, ps, ps.mis_q, ps.counts + C_MIS, b->work + 2, stats);
    k_finish<<<grid, 256, 0, stream>>>(ctx, ps, gs, cur);
    k_advance<<<1, 1, 0, stream>>>(ps.counts);
    return cudaGetLastError();
}

static bool same_config(const pb2_batch_config& a, const pb2_batch_config& b) {
    return a.capacity == b.capacity && a.shade_block == b.shade_block &&
           a.trace_blocks_per_sm == b.trace_blocks_per_sm;
}

// Resets films, counters and the path index space for a render with the current config.
static int batch_reset(pb2_batch* b, cudaStream_t stream) {
    if (b->allocated < b->config.capacity) {
        batch_release_graph(b);  // the graph holds pointers into the old path state
        const int rc = alloc_path_state(&b->mem, &b->allocated, &b->ps, b->config.capacity, true);
        if (rc) return rc;
    }
    if (b->capacity != b->config.capacity) batch_release_graph(b);
    b->capacity = b->config.capacity;
    cudaError_t e;
    std::vector<uint32_t> rem(b->pipes.size());
    for (size_t i = 0; i < b->pipes.size(); ++i) rem[i] = (uint32_t)b->host_scenes[i].path_count;
    if ((e = cudaMemsetAsync(b->films, 0, sizeof(float4) * b->film_elems, stream)) ||
        (e = cudaMemsetAsync(b->ps.counts, 0, sizeof(uint32_t) * C_COUNT, stream)) ||
        (e = cudaMemsetAsync(b->done_ns, 0, sizeof(unsigned long long) * b->pipes.size(), stream)) ||
        (e = cudaMemcpyAsync(b->remaining, rem.data(), sizeof(uint32_t) * rem.size(), cudaMemcpyHostToDevice, stream)))
        return cuda_fail(e, "batch reset");
    k_batch_init<<<(b->capacity + 255) / 256, 256, 0, stream>>>(b->ps, b->capacity, b->state, b->total_paths);
    if ((e = cudaGetLastError())) return cuda_fail(e, "k_batch_init");
    // the host copy of `rem` must outlive the asynchronous copy
    if ((e = cudaStreamSynchronize(stream))) return cuda_fail(e, "batch reset sync");
    return PB2_OK;
}

// Runs iterations until every path of every scene is splatted (or `max_iterations` when non-zero).
static int batch_run(pb2_batch* b, cudaStream_t stream, uint32_t max_iterations, float* ms_out) {
    cudaError_t e;
    const bool use_graph = b->config.use_graph != 0;
    if (use_graph && !(b->graph && same_config(b->graph_config, b->config))) {
        batch_release_graph(b);
        cudaGraph_t g;
        if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal))) return cuda_fail(e, "begin capture");
        cudaError_t le = batch_iteration(b, 0, stream);
        if (le == cudaSuccess) le = batch_iteration(b, 1, stream);
        e = cudaStreamEndCapture(stream, &g);
        if (le != cudaSuccess || e != cudaSuccess) return cuda_fail(le != cudaSuccess ? le : e, "capture batch iteration");
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e) {
            b->graph = nullptr;
            return cuda_fail(e, "instantiate batch graph");
        }
        b->graph_config = b->config;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto done_events = [&]() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    };
    cudaEventRecord(e0, stream);
    k_batch_clock<<<1, 1, 0, stream>>>(b->state);
    uint32_t it = 0;
    const uint32_t check_every = 8;  // iterations between host checks of completion
    // generous bound: every path needs at most (max depth + light pass-throughs) bounces
    uint64_t per_path = 0;
    for (auto* p : b->pipes) per_path = std::max<uint64_t>(per_path, 4ull * (p->settings.max_depth + 2) + 64);
    const uint64_t max_it = (b->total_paths / std::max<uint32_t>(1u, b->capacity) + 2) * per_path;
    for (;;) {
        for (uint32_t k = 0; k < check_every; k += 2) {
            if (use_graph) {
                if ((e = cudaGraphLaunch(b->graph, stream))) {
                    done_events();
                    return cuda_fail(e, "graph launch");
                }
            } else if ((e = batch_iteration(b, 0, stream)) || (e = batch_iteration(b, 1, stream))) {
                done_events();
                return cuda_fail(e, "batch iteration");
            }
            it += 2;
        }
        uint32_t active = 0;
        unsigned long long next = 0;
        if ((e = cudaMemcpyAsync(&active, b->ps.counts + C_EXT_CUR, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) ||
            (e = cudaMemcpyAsync(&next, &b->state->next, sizeof(next), cudaMemcpyDeviceToHost, stream)) ||
            (e = cudaStreamSynchronize(stream))) {
            done_events();
            return cuda_fail(e, "batch progress");
        }
        if (active == 0 && next == b->total_paths) break;
        if (max_iterations && it >= max_iterations) break;
        if (it > max_it) {
            done_events();
            return fail(PB2_ERR_DEVICE_TIMEOUT, "batch did not finish");
        }
    }
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    done_events();
    b->iterations = it;
    if (ms_out) *ms_out = ms;
    uint32_t counts[C_COUNT];
    if ((e = cudaMemcpy(counts, b->ps.counts, sizeof(counts), cudaMemcpyDeviceToHost))) return cuda_fail(e, "batch stats");
    if (counts[C_CHECK])
        return fail(PB2_ERR_CUDA, "index check " + std::to_string(counts[C_CHECK]) + " failed in kernel " +
                                      std::to_string(counts[C_CHECK + 1]) + " at slot " +
                                      std::to_string(counts[C_CHECK + 2]) + ", value " +
                                      std::to_string(counts[C_CHECK + 3]));
    if (counts[C_ERROR]) return fail(PB2_ERR_QUEUE_OVERFLOW, "traversal stack overflow");
    std::memcpy(&b->stats.closest_rays, counts + C_STAT_CLOSEST, 8);
    std::memcpy(&b->stats.shadow_rays, counts + C_STAT_SHADOW, 8);
    std::memcpy(&b->stats.path_vertices, counts + C_STAT_VERTICES, 8);
    return PB2_OK;
}

// Orders the batch's stream after the caller's stream; the batch then works on its own stream and
// synchronises it before returning.
static int batch_stream(pb2_batch* b, void* stream_ptr, cudaStream_t* out) {
    cudaError_t e;
    if (!b->own && (e = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking))) return cuda_fail(e, "batch stream");
    if ((e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream_ptr)))) return cuda_fail(e, "caller stream");
    *out = b->own;
    return PB2_OK;
}

extern "C" {

int pb2_batch_create(const pb2_scene* scenes, const pb2_render_settings* settings, uint32_t count, void* stream_ptr,
                     pb2_batch** out) {
    if (!scenes || !settings || !out || count == 0) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_create: bad argument");
    *out = nullptr;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    auto* b = new pb2_batch();
    auto cleanup = [&](int code) {
        pb2_batch_destroy(b);
        return code;
    };
    for (uint32_t i = 0; i < count; ++i) {
        pb2_pipeline* pl = nullptr;
        const int rc = pb2_pipeline_create(&scenes[i], &settings[i], stream_ptr, &pl);
        if (rc) return cleanup(rc);
        b->pipes.push_back(pl);
        b->type_mask |= pl->type_mask;
    }
    size_t film = 0;
    unsigned long long path = 0;
    for (uint32_t i = 0; i < count; ++i) {
        pb2_pipeline* pl = b->pipes[i];
        BatchScene sc{};
        sc.lp = make_params(pl, pl->full, 0, pl->settings.samples_per_pixel);
        sc.sv.materials = pl->materials;
        sc.sv.textures = pl->textures;
        sc.sv.tri_uv = pl->tri_uv;
        sc.sv.prim_material = pl->accel->prim_material;
        sc.sv.lights = pl->lights;
        sc.sv.plane_cdf = pl->plane_cdf;
        sc.sv.plane_pdf = pl->plane_pdf;
        sc.sv.bvh = pl->accel->view;
        sc.sv.material_count = pl->material_count;
        const unsigned long long n = (unsigned long long)pl->full.width * pl->full.height * pl->settings.samples_per_pixel;
        if (n >= 0xFFFFFFFFull) return cleanup(fail(PB2_ERR_INVALID_ARGUMENT, "a batched scene has 2^32 paths or more"));
        sc.path_begin = path;
        sc.path_count = n;
        path += n;
        b->film_offset.push_back(film);
        film += (size_t)pl->settings.width * pl->settings.height;
        b->host_scenes.push_back(sc);
    }
    b->film_elems = film;
    b->total_paths = path;
    cudaError_t e;
    if ((e = cudaMalloc(&b->films, sizeof(float4) * film)) || (e = cudaMalloc(&b->scenes, sizeof(BatchScene) * count)) ||
        (e = cudaMalloc(&b->remaining, sizeof(uint32_t) * count)) ||
        (e = cudaMalloc(&b->done_ns, sizeof(unsigned long long) * count)) ||
        (e = cudaMalloc(&b->state, sizeof(BatchState))) || (e = cudaMalloc(&b->work, sizeof(uint32_t) * 4)))
        return cleanup(cuda_fail(e, "pb2_batch_create"));
    for (uint32_t i = 0; i < count; ++i) b->host_scenes[i].film = b->films + b->film_offset[i];
    if ((e = cudaMemcpyAsync(b->scenes, b->host_scenes.data(), sizeof(BatchScene) * count, cudaMemcpyHostToDevice,
                             stream)) ||
        (e = cudaStreamSynchronize(stream)))
        return cleanup(cuda_fail(e, "upload batch scenes"));
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace_queue<Q_EXTEND, BatchCtx>, kQThreads, 0);
    b->trace_blocks_max = per > 0 ? per : 1;
    b->config.capacity = (uint32_t)std::max<unsigned long long>(1024ull, std::min<unsigned long long>(path, 1ull << 22));
    b->config.shade_block = 128;
    b->config.trace_blocks_per_sm = (uint32_t)b->trace_blocks_max;
    b->config.use_graph = 1;
    b->scene_ms.assign(count, 0.0f);
    *out = b;
    return PB2_OK;
}

int pb2_batch_destroy(pb2_batch* b) {
    if (!b) return PB2_OK;
    batch_release_graph(b);
    if (b->own) {
        cudaStreamSynchronize(b->own);
        cudaStreamDestroy(b->own);
    }
    for (auto* p : b->pipes) pb2_pipeline_destroy(p);
    cudaFree(b->films);
    cudaFree(b->scenes);
    cudaFree(b->remaining);
    cudaFree(b->done_ns);
    cudaFree(b->state);
    cudaFree(b->work);
    cudaFree(b->mem);
    delete b;
    return PB2_OK;
}

int pb2_batch_get_config(const pb2_batch* b, pb2_batch_config* config) {
    if (!b || !config) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_get_config: null argument");
    *config = b->config;
    return PB2_OK;
}

int pb2_batch_set_config(pb2_batch* b, const pb2_batch_config* c) {
    if (!b || !c) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_set_config: null argument");
    if (c->capacity < 1024 || c->capacity > (1u << 26))
        return fail(PB2_ERR_INVALID_ARGUMENT, "capacity must lie in [1024, 2^26] paths");
    if (c->shade_block != 64 && c->shade_block != 128 && c->shade_block != 256 && c->shade_block != 512)
        return fail(PB2_ERR_INVALID_ARGUMENT, "shade_block must be 64, 128, 256 or 512");
    if (c->trace_blocks_per_sm < 1 || c->trace_blocks_per_sm > (uint32_t)b->trace_blocks_max)
        return fail(PB2_ERR_INVALID_ARGUMENT, "trace_blocks_per_sm must lie in [1, resident blocks per SM]");
    b->config = *c;
    return PB2_OK;
}

int pb2_batch_render(pb2_batch* b, void* stream_ptr) {
    if (!b) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_render: null batch");
    cudaStream_t stream;
    int rc = batch_stream(b, stream_ptr, &stream);
    if (rc) return rc;
    if ((rc = batch_reset(b, stream))) return rc;
    float ms = 0.0f;
    if ((rc = batch_run(b, stream, 0, &ms))) return rc;
    std::vector<unsigned long long> done(b->pipes.size());
    BatchState st{};
    cudaError_t e;
    if ((e = cudaMemcpy(done.data(), b->done_ns, sizeof(unsigned long long) * done.size(), cudaMemcpyDeviceToHost)) ||
        (e = cudaMemcpy(&st, b->state, sizeof(st), cudaMemcpyDeviceToHost)))
        return cuda_fail(e, "batch timing");
    for (size_t i = 0; i < done.size(); ++i)
        b->scene_ms[i] = done[i] >= st.t_start ? (float)((double)(done[i] - st.t_start) * 1e-6) : -1.0f;
    b->total_ms = ms;
    b->stats.paths = b->total_paths;
    return PB2_OK;
}

int pb2_batch_autotune(pb2_batch* b, void* stream_ptr, pb2_batch_config* chosen, float* tune_ms) {
    if (!b) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_autotune: null batch");
    cudaStream_t stream;
    if (const int rc = batch_stream(b, stream_ptr, &stream)) return rc;
    const pb2_batch_config base = b->config;
    // Candidates are scored by path vertices shaded per ms over 24 iterations after 16 from a fresh start: the
    // wavefront has filled and holds paths of as many scenes as the capacity lets in, as through most of a render
    // (a score over the fill alone favours the largest capacity, whose full wavefront then mixes more scenes'
    // trees in the cache and renders slower).  Capacity first, then the launch shapes.
    auto score = [&](const pb2_batch_config& c, double* out) -> int {
        b->config = c;
        int rc = batch_reset(b, stream);
        if (rc) return rc;
        float ms = 0.0f;
        if ((rc = batch_run(b, stream, 16, &ms))) return rc;
        const unsigned long long v0 = b->stats.path_vertices;
        if ((rc = batch_run(b, stream, 24, &ms))) return rc;
        *out = ms > 0.0f ? (double)(b->stats.path_vertices - v0) / ms : 0.0;
        return PB2_OK;
    };
    const auto t0 = std::chrono::steady_clock::now();
    pb2_batch_config best = base;
    double best_s = -1.0;
    auto consider = [&](const pb2_batch_config& c) -> int {
        double s = 0.0;
        const int rc = score(c, &s);
        if (rc) return rc;
        if (s > best_s) {
            best_s = s;
            best = c;
        }
        return PB2_OK;
    };
    const uint32_t caps[] = { 1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23 };
    for (uint32_t cap : caps) {
        if (cap > std::max<unsigned long long>(b->total_paths, 1u << 20)) break;
        pb2_batch_config c = base;
        c.capacity = cap;
        if (const int rc = consider(c)) return rc;
    }
    for (uint32_t sb : { 64u, 256u }) {
        pb2_batch_config c = best;
        c.shade_block = sb;
        if (const int rc = consider(c)) return rc;
    }
    for (uint32_t tb = (uint32_t)b->trace_blocks_max / 2; tb >= 1; tb /= 2) {
        pb2_batch_config c = best;
        c.trace_blocks_per_sm = tb;
        if (const int rc = consider(c)) return rc;
    }
    b->config = best;
    batch_release_graph(b);
    if (chosen) *chosen = best;
    if (tune_ms)
        *tune_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return PB2_OK;
}

int pb2_batch_film(const pb2_batch* b, uint32_t scene, float** rgbw_dev, uint32_t* width, uint32_t* height) {
    if (!b || scene >= b->pipes.size()) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_film: bad scene index");
    if (rgbw_dev) *rgbw_dev = reinterpret_cast<float*>(b->films + b->film_offset[scene]);
    if (width) *width = b->pipes[scene]->settings.width;
    if (height) *height = b->pipes[scene]->settings.height;
    return PB2_OK;
}

int pb2_batch_timing(const pb2_batch* b, float* scene_ms, uint32_t count, float* total_ms, uint32_t* iterations) {
    if (!b || (scene_ms && count != b->pipes.size()))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_timing: count must equal the scene count");
    if (scene_ms) std::memcpy(scene_ms, b->scene_ms.data(), sizeof(float) * count);
    if (total_ms) *total_ms = b->total_ms;
    if (iterations) *iterations = b->iterations;
    return PB2_OK;
}

int pb2_batch_get_stats(const pb2_batch* b, pb2_launch_stats* stats) {
    if (!b || !stats) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_batch_get_stats: null argument");
    *stats = b->stats;
    return PB2_OK;
}

}  // extern "C"
