/*
 * piper2_b200.h -- C ABI of the B200 path-tracing accelerator and tracer for Piper2.
 *
 * Plain C: fixed-width integers, floats, pointers and sizes.  No CUDA, C++ or torch types cross this
 * boundary; streams are passed as `void*` (a cudaStream_t, NULL = the legacy default stream).
 * Every function returns PB2_OK (0) or a PB2_ERR_* code; pb2_last_error() returns the message of
 * the last failure on the calling thread.  This replaces the reference's error path, which logs and
 * calls std::abort() (Src/PiperCore.cpp:533-538).
 *
 * Device pointers ("_dev") must stay valid until the work queued on `stream` completes.  Host
 * pointers ("_host") are read or written before the call returns.
 *
 * Layouts follow the reference's POD payloads where the reference has one, cited per type.
 */
#ifndef PIPER2_B200_H
#define PIPER2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB2_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------------------------- */
#define PB2_OK 0
#define PB2_ERR_INVALID_ARGUMENT 1
#define PB2_ERR_CUDA 2
#define PB2_ERR_OUT_OF_MEMORY 3
#define PB2_ERR_NOT_SUPPORTED 4
#define PB2_ERR_DEVICE_TIMEOUT 5 /* a bounded device-side wait gave up (see the call's doc) */
#define PB2_ERR_QUEUE_OVERFLOW 6

/* ---- rays and hits (Src/Kernel/Protocol.hpp:31-35 RayInfo; Embree.cpp:281-295 ray/hit) ------ */
typedef struct pb2_ray {
    float org[3];
    float tmin; /* hit accepted only for tmin < t */
    float dir[3];
    float tmax; /* ... and t < tmax */
} pb2_ray; /* 32 bytes */

#define PB2_INVALID_PRIM 0xFFFFFFFFu
typedef struct pb2_hit {
    float t;
    uint32_t prim; /* global triangle index, PB2_INVALID_PRIM on a miss */
    float u, v;    /* barycentrics weighting vertex index[1] and index[2] (Embree convention,
                      Src/BuiltinComponent/Tracer/Embree/Kernel.cpp:175-178) */
} pb2_hit; /* 16 bytes */

/* ---- scene description ----------------------------------------------------------------------- */

/* One triangle mesh placed in the scene.  Mirrors TriangleIndexedGeometryDesc
 * (Src/Interface/BuiltinComponent/Tracer.hpp:51-63) plus the GSM instance (geometry + surface,
 * Tracer.hpp:146-147) and its node transform (Tracer.hpp:148).  A vertex lands in world space as
 * transform * vertex + translation.  `transform` NULL is the reference's translation-only instance.  A
 * non-NULL transform (rotation, scale, skew: pb2_srt_matrix) is a divergence: the reference inverts instance
 * transforms with calcInverse (Src/Kernel/Transform.hpp:344-362), which is wrong for any rotation or scale;
 * here the instance is flattened into world space when the acceleration structure is built, so its hits,
 * normals and shading are those of the transformed geometry. */
typedef struct pb2_mesh {
    const float* vertices;    /* vert_count * 3 floats */
    const uint32_t* indices;  /* tri_count * 3 */
    const float* texcoords;   /* vert_count * 2 floats, or NULL */
    uint32_t vert_count;
    uint32_t tri_count;
    uint32_t material;        /* index into pb2_scene.materials */
    float translation[3];
    const float* transform;   /* NULL, or a row-major 3x4 local-to-world matrix [L | t] (12 floats) */
} pb2_mesh;

/* TransformSRT (Src/Kernel/Transform.hpp:390-393), the reference's instance transform: Embree's
 * RTCQuaternionDecomposition, local-to-world = T * R * S (S = scale with skew and shift, R = the rotation of
 * the quaternion, T = translation). */
typedef struct pb2_srt {
    float scale[3];       /* scaleX, scaleY, scaleZ */
    float skew[3];        /* skewXY, skewXZ, skewYZ */
    float shift[3];       /* shiftX, shiftY, shiftZ */
    float quat[4];        /* quatW, quatX, quatY, quatZ (normalised on use) */
    float translation[3]; /* transX, transY, transZ */
} pb2_srt; /* 64 bytes */

/* Parallelogram primitive of the BasicShapes "Plane" geometry: PerPlaneData
 * (Src/BuiltinComponent/Geometry/BasicShapes/Shared.hpp:22-28), byte-compatible (64 bytes).
 * Fill it with pb2_plane_make(). */
typedef struct pb2_plane {
    float origin[3];
    float u[3];
    float v[3];
    float normal[3];
    float tangent[3];
    uint32_t max_det_comp;
} pb2_plane;

/* A "Diffuse" area light over a Plane geometry (Src/BuiltinComponent/Light/AreaLight/Shared.hpp:22-26,
 * AreaLight.cpp:36-57).  Its planes are pb2_scene.planes[first_plane .. first_plane+plane_count). */
typedef struct pb2_area_light {
    float radiance[3];
    uint32_t first_plane;
    uint32_t plane_count;
    float translation[3];
} pb2_area_light;

/* Surfaces of the "Classic" module (Src/BuiltinComponent/Surface/Classic/Classic.cpp:30-199) with
 * constant textures (Src/BuiltinComponent/Texture/ProceduralTexture/Kernel.cpp:21-26). */
enum pb2_surface_type {
    PB2_SURFACE_BLACKBODY = 0, /* no fields */
    PB2_SURFACE_MATTE = 1,     /* color0 = Diffuse, roughness[0] = Roughness (0 -> Lambert) */
    PB2_SURFACE_PLASTIC = 2,   /* color0 = Diffuse, color1 = Specular, roughness[0] = Roughness */
    PB2_SURFACE_GLASS = 3,     /* color0 = Reflection, color1 = Transmission, roughness = X, Y */
    PB2_SURFACE_MIRROR = 4,    /* color0 = Reflection */
    PB2_SURFACE_SUBSTRATE = 5, /* color0 = Diffuse, color1 = Specular, roughness = X, Y */
    PB2_SURFACE_CONDUCTOR = 6  /* extension, no reference counterpart: GGX reflection with the
                                  Schlick Fresnel of color1 as F0, roughness[0] = alpha */
};
typedef struct pb2_material {
    uint32_t type;
    float color0[4];
    float color1[4];
    float roughness[2];
    /* Per parameter (color0, color1, roughness[0], roughness[1]): 0 takes the constant above (ConstantTexture),
     * k > 0 samples pb2_scene.textures[k - 1] at the hit's texture coordinate instead.  A color takes a 4-channel
     * texture, a roughness a 1-channel one (the reference's loadTexture(desc, 4 / 1), Surface/Classic/Classic.cpp). */
    uint32_t texture[4];
} pb2_material; /* 60 bytes */

/* Textures a material parameter can sample.  The texture coordinate of a triangle hit is the barycentric blend of
 * its mesh's texcoords (calcTriangleMeshSurface, Src/BuiltinComponent/Tracer/Embree/Kernel.cpp:170-192), (0, 0)
 * for a mesh without them. */
enum pb2_texture_kind {
    PB2_TEXTURE_CHECKERBOARD = 1, /* CheckBoard (Texture/ProceduralTexture/Kernel.cpp:27-38): `scale`, `black`, `white` */
    PB2_TEXTURE_IMAGE = 2         /* SampledTexture (Texture/SampledTexture/Kernel.cpp:59-83): bilinear over 8-bit texels */
};
enum pb2_texture_wrap { PB2_WRAP_REPEAT = 0, PB2_WRAP_MIRROR = 1 };
typedef struct pb2_texture {
    uint32_t kind;
    uint32_t channel;        /* 1, 2 or 4 */
    uint32_t wrap;           /* image: pb2_texture_wrap */
    uint32_t width, height;  /* image: texels, rows of width * channel bytes, top row first */
    const uint8_t* texels;   /* image: host memory, copied to the device when the pipeline is created */
    float scale;             /* checkerboard */
    float black[4], white[4];
} pb2_texture;

/* Perspective camera (Src/BuiltinComponent/Sensor/PerspectiveCamera/Shared.hpp:22-29, config parse
 * PerspectiveCamera.cpp:35-46).  `position` is the camera node's translation (the reference reads it
 * from the node transform, Kernel.cpp:26-29).  Sizes in metres: the reference's config is in mm and
 * is scaled by 1e-3f on load; pb2_camera_from_config() does the same conversion. */
typedef struct pb2_camera {
    float position[3];
    float look_at[3];
    float up[3];          /* normalised */
    float sensor_size[2]; /* metres */
    float focal_length;   /* metres */
    float aperture_radius;/* metres = focal_length / (2 FStop) */
} pb2_camera;

typedef struct pb2_scene {
    const pb2_mesh* meshes;
    uint32_t mesh_count;
    const pb2_plane* planes;
    uint32_t plane_count;
    const pb2_area_light* area_lights;
    uint32_t area_light_count;
    const pb2_material* materials;
    uint32_t material_count;
    float env_radiance[3]; /* the single "SampledEnvironment" light, lights[0] (Embree.cpp:1174-1188) */
    const pb2_texture* textures;
    uint32_t texture_count;
} pb2_scene;

/* ---- render settings (component configs) -------------------------------------------------- */
enum pb2_filter_type { PB2_FILTER_BOX = 0, PB2_FILTER_TRIANGLE = 1, PB2_FILTER_GAUSSIAN = 2 };
enum pb2_fit_mode { PB2_FIT_FILL = 0, PB2_FIT_OVERSCAN = 1 };

typedef struct pb2_render_settings {
    uint32_t width, height;   /* film resolution */
    uint32_t fit_mode;        /* pb2_fit_mode, Src/Interface/BuiltinComponent/Sensor.hpp:36-75 */
    uint32_t samples_per_pixel;/* ScrambledSobolSampler "SamplesPerPixel": rounded up to a power of 2
                                  (ScrambledSobolSampler.cpp:43-50) */
    uint32_t scramble;        /* 0: unscrambled, the reference's only mode ("Scramble" is notImplemented,
                                  :51-53).  1: Owen scrambling of dimensions >= 2 (extension, see
                                  scramble_seed); dimensions 0/1 place the sample in its pixel and stay */
    uint32_t max_depth;       /* PathTracing "MaxTraceDepth" (PathTracing.cpp:38) */
    uint32_t min_rr_depth;    /* PathTracing "MinRussianRouletteDepth" (PathTracing.cpp:39) */
    uint32_t filter;          /* pb2_filter_type (FixedSampler.cpp:38-45) */
    float gaussian_alpha;     /* "Alpha" of the gaussian filter */
    pb2_camera camera;
    uint32_t scramble_seed;   /* seed of the Owen scrambling (scramble = 1) */
} pb2_render_settings;

/* Render rectangle (Tracer.hpp:96-98 RenderRECT). */
typedef struct pb2_rect {
    uint32_t left, top, width, height;
} pb2_rect;

/* The NDC transform of calcRenderRECT (Protocol.hpp:113-115 SensorNDCAffineTransform). */
typedef struct pb2_ndc_transform {
    float ox, oy, sx, sy;
} pb2_ndc_transform;

/* Per-launch statistics, the counters the reference's EmbreeProfiler collects
 * (Embree.cpp:1266-1271, PathTracing.cpp:48-54) reduced once per launch. */
typedef struct pb2_launch_stats {
    uint64_t closest_rays;  /* camera + continuation + pass-through + MIS-BSDF rays */
    uint64_t shadow_rays;
    uint64_t paths;
    uint64_t path_vertices;
    uint32_t depth_histogram[32];
} pb2_launch_stats;

/* ---- library --------------------------------------------------------------------------------- */
const char* pb2_last_error(void);
int pb2_abi_version(void);
/* Selects the CUDA device for the calling thread (cuCtxSetCurrent analogue of
 * Src/Infrastructure/Accelerator/CUDA/CUDA.cpp:204-210). */
int pb2_set_device(int device);

/* ---- component helpers (host) -------------------------------------------------------------- */
/* Plane primitive from Origin/U/V (BasicShapes.cpp:70-89). */
int pb2_plane_make(const float origin[3], const float u[3], const float v[3], pb2_plane* out);
/* The row-major 3x4 local-to-world matrix of an SRT transform; PB2_ERR_INVALID_ARGUMENT for a zero or non-finite
 * quaternion or a non-finite entry. */
int pb2_srt_matrix(const pb2_srt* srt, float matrix[12]);
/* A plane mapped by a 3x4 local-to-world matrix: origin as a point, u and v as vectors, then pb2_plane_make (the
 * normal of the mapped parallelogram is the correctly transformed normal). */
int pb2_plane_transform(const pb2_plane* in, const float matrix[12], pb2_plane* out);
/* Camera from the PerspectiveCamera config keys in their config units (mm, FStop)
 * (PerspectiveCamera.cpp:39-44). */
int pb2_camera_from_config(const float position[3], const float look_at[3], const float up[3],
                           const float sensor_size_mm[2], float focal_length_mm, float fstop,
                           pb2_camera* out);
/* calcRenderRECT (Src/Interface/BuiltinComponent/Sensor.hpp:38-75). */
int pb2_calc_render_rect(uint32_t width, uint32_t height, float device_aspect, uint32_t fit_mode,
                         pb2_ndc_transform* transform, pb2_rect* rect);

/* ---- Sobol sampler (Src/BuiltinComponent/Sampler/ScrambledSobolSampler/Kernel.cpp) ----------- */
/* sobolGenerate (:65-67) for n (index, dimension) pairs, on the device. */
int pb2_sobol_generate(const uint64_t* index_dev, const uint32_t* dim_dev, uint32_t n, float* out_dev,
                       void* stream);
/* sobolStart (:52-62) for n (px, py, sample) triples: writes the global index and pixel offset. */
int pb2_sobol_start(uint32_t log2_resolution, const uint32_t* pixel_sample_dev, uint32_t n,
                    uint64_t* index_dev, float* offset_dev, void* stream);
/* SHA-256 (hex) of the generated Sobol tables compiled into the library. */
const char* pb2_sobol_table_digest(void);

/* ---- acceleration structure and traversal (replaces Tracer::buildAcceleration and Embree's
 *      rtcIntersect1/rtcOccluded1, Embree.cpp:267-391, 497-655) ------------------------------- */
typedef struct pb2_accel pb2_accel;

typedef struct pb2_accel_info {
    uint32_t triangle_count;
    uint32_t node_count;       /* 8-wide nodes */
    uint32_t leaf_triangle_slots;
    uint32_t plane_count;
    uint64_t device_bytes;
    float build_ms;            /* device time of the build */
} pb2_accel_info;

/* Builds the LBVH -> 8-wide quantised BVH over all scene meshes on the device.  Host scene
 * arrays are copied during the call. */
int pb2_accel_create(const pb2_scene* scene, void* stream, pb2_accel** out);
int pb2_accel_destroy(pb2_accel* accel);
int pb2_accel_get_info(const pb2_accel* accel, pb2_accel_info* info);
/* Host-side structural check of the built BVH (copies it out of device memory): child and triangle
 * indices in range, every node and triangle reached exactly once, every triangle inside the dequantised
 * box of its child slot.  PB2_OK or PB2_ERR_INVALID_ARGUMENT naming the first violation.  No
 * counterpart in the reference (Embree's BVH is opaque). */
int pb2_accel_validate(const pb2_accel* accel);

/* Closest hit over triangles and area-light planes (planes reported with prim =
 * PB2_PLANE_FLAG | plane index).  Ties in t resolve to the lowest prim. */
#define PB2_PLANE_FLAG 0x80000000u
int pb2_trace_closest(const pb2_accel* accel, const pb2_ray* rays_dev, uint32_t n, pb2_hit* hits_dev,
                      void* stream);
/* Any hit over triangles only (planes never occlude: mask = GSM only, Embree.cpp:378).
 * occluded_dev[i] = 1 if some triangle has tmin < t < tmax. */
int pb2_trace_any(const pb2_accel* accel, const pb2_ray* rays_dev, uint32_t n, uint32_t* occluded_dev,
                  void* stream);
/* The same two calls with host arrays: copies in, traces, copies out, synchronises `stream`.  Batches
 * of more than 2^20 rays are cut into chunks of 2^20 (from 2^21 rays on with a quarter and a half chunk at
 * either end) that three internal streams (created on the first such call, kept until pb2_accel_destroy)
 * upload, trace and download in turn, so the copies of one chunk overlap the traversal of another; host
 * arrays should be pinned for the copies to overlap. */
int pb2_trace_closest_host(const pb2_accel* accel, const pb2_ray* rays_host, uint32_t n,
                           pb2_hit* hits_host, void* stream);
int pb2_trace_any_host(const pb2_accel* accel, const pb2_ray* rays_host, uint32_t n,
                       uint32_t* occluded_host, void* stream);
/* Traversal work counters of the last trace call on this accel (node visits, triangle tests),
 * summed over the batch; only filled when counting is enabled. */
int pb2_accel_set_counting(pb2_accel* accel, int enable);
int pb2_accel_get_counters(const pb2_accel* accel, uint64_t* node_visits, uint64_t* tri_tests,
                           void* stream);

/* Closest hit for callers that cannot allocate device memory (a fixed memory budget owned by their own
 * allocator, or no room for the implicit device synchronisation of cudaMalloc/cudaFree).  No counterpart
 * in the reference.  Builds the 8-wide BVH over `triangles_dev` (tri_count * 9 floats: v0, v1, v2 per
 * triangle, world space; prim = triangle index) and writes the closest hit of each ray to hits_dev,
 * with every intermediate buffer in one 8 MiB file-scope device array that every GPU loading the library
 * holds until exit -- at most 16384 triangles (larger inputs return PB2_ERR_INVALID_ARGUMENT).  Hits
 * equal those of pb2_accel_create + pb2_trace_closest on the same triangles.  The first call on a device
 * looks the array's device address up (cudaGetSymbolAddress) and should come before any stream
 * capture; the address is kept per device, so the call must not be used across a cudaDeviceReset of a
 * device it ran on.  The call synchronises `stream` and returns when its hits are written; a ray whose
 * traversal stack overflowed makes it return PB2_ERR_QUEUE_OVERFLOW.  All calls share the array and it
 * keeps the last call's contents: calls that overlap on the GPU (other threads or streams) race and
 * must be serialised by the caller. */
int pb2_trace_closest_nalloc(const float* triangles_dev, uint32_t tri_count, const pb2_ray* rays_dev, uint32_t n,
                             pb2_hit* hits_dev, void* stream);

/* ---- Piper component payloads -> scene (Tracer::buildPipeline's materialize step) ----------------------
 * A Piper tracer plugin receives each component's materialized program as a symbol name plus POD payload
 * bytes (Tracer::buildProgram, MaterializeContext::registerCall / registerResource; Tracer.hpp:86-91,
 * 121-133).  The builder takes exactly those, byte for byte in the reference's layouts, dispatches on the
 * symbol, and assembles the pb2_scene and pb2_render_settings of a pipeline.  Supported symbols (the
 * components of the render path):
 *   sensor         "rayGen"          PCData (PerspectiveCamera/Shared.hpp:22-29)
 *   integrator     "trace"           Data (PathTracing/Shared.hpp:22-29)
 *   render driver  "accumulate"      RDData (FixedSampler/Shared.hpp) -> a call to "box", "triangle" or
 *                                    "gaussian" (GaussianFilterData)
 *   sampler        "sobolStart"      no payload (SobolData is made per frame)
 *   light sampler  "uniformSelect"   no payload
 *   surface        "blackBodyInit", "matteInit", "plasticInit", "glassInit", "mirrorInit", "substrateInit"
 *                                    with MatteData / PlasticData / GlassData / MirrorData / SubstrateData
 *                                    (Surface/Classic/Shared.hpp), their textures calls to
 *                                    "constantTexture" (ConstantData, ProceduralTexture/Shared.hpp)
 *   light          "SEInit"          SampledEnvironmentData (BasicLight/Shared.hpp)
 *                  "diffuseInit"     DiffuseAreaLightData (AreaLight/Shared.hpp) -> a call to "planeSample"
 *                                    (CDFData, BasicShapes/Shared.hpp) over a resource of PerPlaneData
 * Any other symbol fails with PB2_ERR_NOT_SUPPORTED naming it, as the reference's pipeline build would
 * fail on a program it cannot link.  Handles inside payloads (Call<...>, TraversalHandle) are the 64-bit
 * values this builder returned (pb2_builder_register_call) or was given (pb2_builder_add_node). */
typedef struct pb2_builder pb2_builder;
enum pb2_program_kind {
    PB2_PROGRAM_SENSOR = 0,
    PB2_PROGRAM_INTEGRATOR = 1,
    PB2_PROGRAM_RENDER_DRIVER = 2,
    PB2_PROGRAM_SAMPLER = 3,
    PB2_PROGRAM_LIGHT_SAMPLER = 4,
    PB2_PROGRAM_SURFACE = 5,
    PB2_PROGRAM_LIGHT = 6
};
int pb2_builder_create(pb2_builder** out);
int pb2_builder_destroy(pb2_builder* builder);
/* MaterializeContext::registerResource: a buffer later payloads name by the returned index. */
int pb2_builder_register_resource(pb2_builder* builder, const void* data, size_t bytes, uint32_t* index);
/* MaterializeContext::registerCall: a program and its payload; *handle is the CallHandle value that other
 * payloads hold in their Call<...> fields. */
int pb2_builder_register_call(pb2_builder* builder, const char* symbol, const void* payload, size_t bytes,
                              uint64_t* handle);
/* A scene node (Tracer::buildNode) by the TraversalHandle value payloads use for it, with its
 * translation. */
int pb2_builder_add_node(pb2_builder* builder, uint64_t traversal, const float translation[3]);
/* A scene node with a full local-to-world transform (row-major 3x4, e.g. from pb2_srt_matrix).  A light on it has
 * its planes mapped into world space (pb2_plane_transform) unless the linear part is the identity, in which case
 * it is the translation-only node of pb2_builder_add_node; a camera on it stands at the transform's origin, as the
 * reference's rayGen reads only the origin of its node (PerspectiveCamera/Kernel.cpp:25-28). */
int pb2_builder_add_node_transform(pb2_builder* builder, uint64_t traversal, const float matrix[12]);
/* A component's materialized program of the given pb2_program_kind: its (first) symbol and payload.
 * *index (may be NULL) is the material index of a surface, the light index of a light, else 0. */
int pb2_builder_add_program(pb2_builder* builder, uint32_t kind, const char* symbol, const void* payload,
                            size_t bytes, uint32_t* index);
/* A triangle mesh GSM instance (Tracer::buildAcceleration + buildGSMInstance + buildNode); mesh->material is
 * a surface index from pb2_builder_add_program.  The arrays are copied. */
int pb2_builder_add_mesh(pb2_builder* builder, const pb2_mesh* mesh);
/* Pipeline::prepare's inputs: the film, the fit mode and the sampler's samples per pixel.  Fills *scene
 * and *settings (their arrays belong to the builder and live until it is destroyed); fails if a required
 * component (sensor, integrator, render driver, sampler, light sampler, the environment as light 0) is
 * missing. */
int pb2_builder_build(pb2_builder* builder, uint32_t width, uint32_t height, uint32_t fit_mode,
                      uint32_t samples_per_pixel, pb2_scene* scene, pb2_render_settings* settings);

/* ---- render pipeline (Tracer::buildPipeline, Pipeline::prepare, TraceLauncher::launch;
 *      Tracer.hpp:100-119, 153-155; Embree.cpp:978-1304) --------------------------------------- */
typedef struct pb2_pipeline pb2_pipeline;

int pb2_pipeline_create(const pb2_scene* scene, const pb2_render_settings* settings, void* stream,
                        pb2_pipeline** out);
int pb2_pipeline_destroy(pb2_pipeline* pipeline);
/* Film resolution and full render rectangle (TraceLauncher::getFilmResolution/getRenderRECT). */
int pb2_pipeline_get_rect(const pb2_pipeline* pipeline, pb2_rect* full_rect, pb2_ndc_transform* ndc);
/* Renders samples [sample_begin, sample_begin + sample_count) of every pixel of `rect` (a sub-rect of
 * the full rect) and adds them to the RGBW film `rgbw_dev` (width * height float4, the
 * FixedSampler film, FixedSampler/Kernel.cpp:22-52).  If `sample_out_dev` is not NULL it receives
 * per (pixel, sample) the film point and radiance, 5 floats each, in (y, x, sample) order. */
int pb2_pipeline_launch(pb2_pipeline* pipeline, const pb2_rect* rect, uint32_t sample_begin,
                        uint32_t sample_count, float* rgbw_dev, float* sample_out_dev, void* stream);
/* Counting build of the render's traversal (for the render path's byte model; slower, off by default):
 * while on, the closest-hit, MIS and shadow queries of every launch add their rays, node visits and triangle
 * tests to nine counters (extend rays/visits/tests, MIS ..., shadow ...), cleared when counting is switched
 * on; pb2_pipeline_get_trace_counters reads them (synchronising `stream`). */
int pb2_pipeline_set_counting(pb2_pipeline* pipeline, int enable);
int pb2_pipeline_get_trace_counters(const pb2_pipeline* pipeline, uint64_t* counters9_host, void* stream);
/* Bounds the path slots of a single-scene launch (default 2^24, in [256, 2^30]).  A launch keeps at most
 * `slots` paths (rect pixels x sample_count) in flight: every bounce first refills the slots that finished
 * paths freed with the launch's next paths, so the wavefront stays full until they run out, and the path
 * state (about 260 bytes per slot, plus about 400 with a guide attached) stays bounded.  The samples and
 * the film are those of the same launch without the bound.  Shrinking the bound frees the larger state. */
int pb2_pipeline_set_path_slots(pb2_pipeline* pipeline, uint32_t slots);
/* The bounce loop of a single-scene launch as CUDA graphs (on by default; no reference counterpart, the
 * reference runs one CPU task per pixel and sample): after the first four bounces, every four bounces
 * (between two host checks of the extend queue) replay one graph, captured for the launch's parameters on
 * the pipeline's own stream and updated in place from launch to launch.  Off: plain launches (the form
 * PB2_DEBUG_SYNC=1 always uses).  Samples and films are the same either way. */
int pb2_pipeline_set_graphs(pb2_pipeline* pipeline, int enabled);
/* Resolve radiance = rgb / w (FixedSampler.cpp:122-131) into rgb_dev (width * height * 3). */
int pb2_film_resolve(const float* rgbw_dev, uint32_t pixel_count, float* rgb_dev, void* stream);
int pb2_pipeline_get_stats(const pb2_pipeline* pipeline, pb2_launch_stats* stats, void* stream);
/* Camera rays of one sample index for every pixel of `rect` (piperMain + rayGen,
 * Tracer/Embree/Kernel.cpp:47-90, PerspectiveCamera/Kernel.cpp:22-48): rays_dev gets the ray, and
 * points_dev the film point (2 floats), in (y, x) order. */
int pb2_pipeline_camera_rays(pb2_pipeline* pipeline, const pb2_rect* rect, uint32_t sample,
                             pb2_ray* rays_dev, float* points_dev, void* stream);

/* ---- learned path guiding (no counterpart in the reference, which samples BxDFs only) ------------
 * A 96-64-64-64-64-48 MLP (BF16 tensor-core tiles, FP32 accumulation) maps the encoded hit position,
 * shading normal and outgoing direction to a mixture of 8 von Mises-Fisher lobes.  Guided pipelines draw
 * each non-specular continuation direction from 0.5 BxDF + 0.5 mixture (one-sample MIS, pdf = the
 * mixture of both), which keeps the estimator unbiased; NEE + MIS is unchanged.  The network is trained
 * online on the radiance samples the integrator produces, with the Monte-Carlo KL divergence and Adam. */
typedef struct pb2_guide pb2_guide;

uint32_t pb2_guide_param_count(void);
/* He-uniform weights from `seed`, zero biases, zeroed Adam state. */
int pb2_guide_create(uint32_t seed, pb2_guide** out);
int pb2_guide_destroy(pb2_guide* guide);
/* Flat fp32 parameters: per layer W[out][in] then b[out]; setting them resets the Adam state. */
int pb2_guide_set_params(pb2_guide* guide, const float* params_host, uint32_t count);
int pb2_guide_get_params(const pb2_guide* guide, float* params_host, uint32_t count);
/* features_dev (16-byte aligned): n rows of 12 floats (position in the unit cube xyz, normal xyz, outgoing dir xyz, unused);
 * out_dev (16-byte aligned): n rows of 48 raw outputs (8 x (weight logit, mean xyz, concentration), 8 unused).
 * Runs on the tcgen05 tensor cores (one CTA per SM of seven independent 128-row warp groups, TMEM
 * accumulators); synchronises `stream` to check that no tensor-core wait timed out (PB2_ERR_DEVICE_TIMEOUT). */
int pb2_guide_forward(const pb2_guide* guide, const float* features_dev, uint32_t n, float* out_dev, void* stream);
/* pb2_guide_forward without the host synchronisation, for work queued on a stream or captured in a CUDA graph
 * (no reference counterpart): a tensor-core wait that timed out sets *status_dev (a device word) to 1; the
 * caller clears it beforehand and reads it after synchronising.  Nothing is allocated. */
int pb2_guide_forward_async(const pb2_guide* guide, const float* features_dev, uint32_t n, float* out_dev,
                            uint32_t* status_dev, void* stream);
/* The same forward pass on mma.sync tiles (16 rows per warp), asynchronous; the cross-check of the tcgen05
 * path. */
int pb2_guide_forward_mma(const pb2_guide* guide, const float* features_dev, uint32_t n, float* out_dev,
                          void* stream);
/* records_dev: n rows of 16 floats (position xyz, normal xyz, outgoing xyz, sampled direction xyz, weight =
 * target / sampling pdf, unused x3).  Gradient of the batch loss into grad_host (pb2_guide_param_count
 * floats, may be NULL) and the loss; parameters unchanged. */
int pb2_guide_gradient(pb2_guide* guide, const float* records_dev, uint32_t n, float* grad_host, float* loss_host,
                       void* stream);
/* The same gradient on mma.sync tiles (16 records per warp, staged layer inputs and deltas, batch-K weight
 * GEMMs); the cross-check of the tcgen05 training kernel that pb2_guide_gradient and pb2_guide_train use. */
int pb2_guide_gradient_mma(pb2_guide* guide, const float* records_dev, uint32_t n, float* grad_host, float* loss_host,
                           void* stream);
/* One Adam step (beta1 0.9, beta2 0.99) on the batch.  The gradient runs on the tcgen05 tensor cores; a
 * tensor-core wait that timed out is reported (PB2_ERR_DEVICE_TIMEOUT) by the next call that synchronises
 * (pb2_guide_gradient, pb2_guide_train with loss_host, pb2_pipeline_train_guide). */
int pb2_guide_train(pb2_guide* guide, const float* records_dev, uint32_t n, float learning_rate, float* loss_host,
                    void* stream);
/* Called by every training step (pb2_guide_train, pb2_pipeline_train_guide) between the gradient and the
 * Adam update, with the step's gradient on the device (grad_dev, `count` = pb2_guide_param_count() floats)
 * and the stream the step runs on; the hook may rewrite the gradient in place -- e.g. average it over the
 * ranks of a multi-GPU render with an all-reduce queued on `stream` -- and returns PB2_OK or an error code,
 * which fails the step.  NULL removes the hook. */
typedef int (*pb2_gradient_hook)(float* grad_dev, uint32_t count, void* stream, void* user);
int pb2_guide_set_gradient_hook(pb2_guide* guide, pb2_gradient_hook hook, void* user);

typedef struct pb2_guide_settings {
    float selection_prob;      /* probability of sampling the guide at a guided vertex (0.5) */
    uint32_t record_capacity;  /* training records kept between two training calls (e.g. 2^20) */
    float weight_quantile;     /* training weights are clamped at this quantile of the call's records
                                  (e.g. 0.99; 0 or 1 = no clamp) */
    uint32_t spatial_cells;    /* before clamping, each record's weight is divided by the mean weight of its
                                  cell in a spatial_cells^3 grid over the scene box (0 = off, at most 16) */
    uint32_t guided_types;     /* bit t set: vertices of surface type t (PB2_SURFACE_*) sample the guide; only
                                  Matte and Conductor may be set.  0 = Matte only: a glossy conductor's own
                                  sampler is already close to the product with the incident light */
    uint32_t max_guided_depth; /* only vertices at path depth < max_guided_depth (0 = every depth) sample the
                                  guide; the others keep plain BxDF sampling and skip its evaluation */
} pb2_guide_settings;

/* Attaches `guide` (not owned; NULL detaches) to the pipeline: later launches sample and record with it. */
int pb2_pipeline_set_guide(pb2_pipeline* pipeline, pb2_guide* guide, const pb2_guide_settings* settings);
/* Verification copy of the in-render inference: while set, every guided launch appends one row of 52
 * floats per vertex whose mixture it inferred -- the vertex's 9 network inputs (position in the unit scene
 * box, shading normal, outgoing direction) and the 40 mixture parameters it used (8 lobe weights, 8 unit
 * means xyz, 8 concentrations), 3 unused -- to rows_dev, at most `capacity` rows; *count_dev (device
 * memory, cleared by the caller) counts the vertices offered.  rows_dev = NULL stops it. */
int pb2_pipeline_set_guide_dump(pb2_pipeline* pipeline, float* rows_dev, uint32_t capacity, uint32_t* count_dev);
/* Runs `steps` Adam steps of `batch` records drawn uniformly from the records of the launches since the
 * last call (weights clamped per pb2_guide_settings.weight_quantile), then clears them.  Writes the last
 * step's loss. */
int pb2_pipeline_train_guide(pb2_pipeline* pipeline, uint32_t steps, uint32_t batch, float learning_rate,
                             float* loss_host, void* stream);

/* ---- batched multi-scene rendering (no reference counterpart: the reference renders one scene per
 * pipeline and frame, FixedSampler.cpp:68-133) -----------------------------------------------------
 * All scenes share one wavefront of path slots: a slot whose path is splatted is refilled from one global
 * (scene, pixel, sample) index space, so scenes and films of uneven size keep every launch full.  Each path
 * is the one a single-scene launch of the full frame traces for that (pixel, sample); films match per-scene
 * renders within accumulation rounding.  Two wavefront iterations run as one captured CUDA graph on the
 * batch's own stream, ordered after the caller's stream. */
typedef struct pb2_batch pb2_batch;
typedef struct pb2_batch_config {
    uint32_t capacity;            /* path slots in flight, [1024, 2^26] */
    uint32_t shade_block;         /* threads per block of the shading kernels (64/128/256/512) */
    uint32_t trace_blocks_per_sm; /* resident blocks per SM of the persistent traversal kernels */
    uint32_t use_graph;           /* 1: replay the captured iteration graph, 0: plain launches */
} pb2_batch_config;

/* One pipeline per (scene, settings) pair; spp per scene as in pb2_render_settings. */
int pb2_batch_create(const pb2_scene* scenes, const pb2_render_settings* settings, uint32_t count, void* stream,
                     pb2_batch** out);
int pb2_batch_destroy(pb2_batch* batch);
int pb2_batch_get_config(const pb2_batch* batch, pb2_batch_config* config);
int pb2_batch_set_config(pb2_batch* batch, const pb2_batch_config* config);
/* Times short runs of candidate configurations (capacity, then shading block, then traversal blocks per
 * SM) and keeps the fastest; writes it and the tuning time. */
int pb2_batch_autotune(pb2_batch* batch, void* stream, pb2_batch_config* chosen, float* tune_ms);
/* Clears the films and renders every scene's samples; returns when they are done. */
int pb2_batch_render(pb2_batch* batch, void* stream);
/* Device pointer of scene `scene`'s RGBW film (width x height float4) and its size. */
int pb2_batch_film(const pb2_batch* batch, uint32_t scene, float** rgbw_dev, uint32_t* width, uint32_t* height);
/* Per-scene completion time (ms after the render started, device clock) of the last render, its total
 * device time and the number of wavefront iterations. */
int pb2_batch_timing(const pb2_batch* batch, float* scene_ms, uint32_t count, float* total_ms,
                     uint32_t* iterations);
int pb2_batch_get_stats(const pb2_batch* batch, pb2_launch_stats* stats);

/* ---- Accelerator: buffers, tiled outputs, resource lookup tables, generic kernel launches ---------
 * The CUDA Accelerator plugin of the reference (Src/Interface/Infrastructure/Accelerator.hpp:130-161,
 * Src/Infrastructure/Accelerator/CUDA/CUDA.cpp:497-927) without its LLVM-IR JIT: a kernel is native sm_100a
 * code compiled against include/piper2_b200_device.cuh and registered by entry name, in place of
 * compileKernel's link of LLVM modules.  One accelerator drives one device (the current device at creation;
 * the reference opens a context per device, CUDA.cpp:718-780) through `streams` CUDA streams (its "Steams"
 * option, CUDA.cpp:723-726; 0 = 4).  Every operation is ordered by futures as in the reference: a buffer's
 * upload, a tiled output's last marked writer and a launch each complete a future, and a launch waits for the
 * futures of every resource its lookup table reaches (CUDA.cpp:817-824).  Resources and futures are
 * reference counted (the reference's SharedPtr): *_release drops one reference; a lookup table holds its
 * entries, a launch holds its kernel, table and resources until it completes. */
typedef struct pb2_accelerator pb2_accelerator;
typedef struct pb2_resource pb2_resource;
typedef struct pb2_kernel pb2_kernel;
typedef struct pb2_future pb2_future;
/* Fills `size` bytes of staging memory at `dst` (the Function<void, Ptr> of createBuffer). */
typedef void (*pb2_fill_fn)(void* dst, size_t size, void* user);

int pb2_acc_create(uint32_t streams, pb2_accelerator** out);
/* Waits for all work and drops the caller's reference; the streams live on until the last resource made by the
 * accelerator is released. */
int pb2_acc_destroy(pb2_accelerator* acc);
/* "NVIDIA CUDA" (getNativePlatform, CUDA.cpp:791-793). */
const char* pb2_acc_native_platform(const pb2_accelerator* acc);
/* Device index of the accelerator's context and its stream count (enumerateContexts). */
int pb2_acc_get_info(const pb2_accelerator* acc, int* device, uint32_t* streams);
/* createBuffer (CUDA.cpp:913-916, CUDABufferInstance :513-566): `fill` writes the initial bytes into pinned
 * staging memory before the call returns (NULL fill = zeros); the upload to the device is asynchronous and
 * completes the buffer's future.  `alignment` is a power of two (the device address is aligned to it). */
int pb2_acc_create_buffer(pb2_accelerator* acc, size_t size, size_t alignment, pb2_fill_fn fill, void* user,
                          pb2_resource** out);
/* createTiledOutput (CUDA.cpp:922-924, CUDATiledBufferInstance :585-640): a zeroed device buffer that kernels
 * write; pb2_tiled_output_mark_dirty names the launch whose writes a download must wait for. */
int pb2_acc_create_tiled_output(pb2_accelerator* acc, size_t size, size_t alignment, pb2_resource** out);
/* createResourceLUT (CUDA.cpp:919-921, ResourceLookUpTableInstance :665-697): entries are buffers, tiled
 * outputs or other tables; a launch flattens the tables (root first, each nested table's entries appended
 * after its parent's, the parent's entry holding the handle index where they start). */
int pb2_acc_create_resource_lut(pb2_accelerator* acc, pb2_resource* const* resources, uint32_t count,
                                pb2_resource** out);
/* ResourceInstance::getHandle: the device address of a buffer or tiled output (tables have none). */
int pb2_resource_get_handle(const pb2_resource* res, uint64_t* handle);
int pb2_resource_release(pb2_resource* res);
/* TiledOutput::markDirty (CUDA.cpp:656-658). */
int pb2_tiled_output_mark_dirty(pb2_resource* output, pb2_future* writer);
/* TiledOutput::download (CUDA.cpp:627-637): waits for the marked writer, copies `size` bytes (at most the
 * output's size) to `dst_host` and returns when they are there. */
int pb2_tiled_output_download(pb2_resource* output, void* dst_host, size_t size);
/* compileKernel without the JIT: `entry` names a kernel registered on this accelerator; unknown names fail
 * with PB2_ERR_NOT_SUPPORTED naming the entry (the reference fails to link an unknown symbol). */
int pb2_acc_compile_kernel(pb2_accelerator* acc, const char* entry, pb2_kernel** out);
/* Registers a generic kernel: `cu_function` is the CUfunction of an entry declared with PB2_KERNEL_ENTRY
 * (from cudaGetFuncBySymbol or cuModuleGetFunction) in the accelerator's device context. */
int pb2_acc_register_kernel(pb2_accelerator* acc, const char* entry, void* cu_function);
int pb2_kernel_release(pb2_kernel* kernel);
/* launchKernel (CUDA.cpp:803-910): packs the flattened handles of `root` and the arguments (`arg_desc` holds
 * arg_count (offset, size) pairs into `arg_data`, the reference's ArgumentPackage) into a launch buffer and
 * launches the kernel over dim[0] x dim[1] x dim[2] tasks on a stream (the first idle one, else round robin)
 * after the futures of every resource reached through `root`.  An empty launch is rejected (CUDA.cpp:
 * 805-806).  *out (optional) is the launch's future. */
int pb2_acc_launch_kernel(pb2_accelerator* acc, const uint32_t dim[3], pb2_kernel* kernel, pb2_resource* root,
                          const void* arg_data, const uint32_t* arg_desc, uint32_t arg_count, pb2_future** out);
/* The launch buffer layout alone (no device): writes it for `handles` and the arguments to `dst` (when
 * dst_size suffices) and its size to *needed.  The layout is documented in piper2_b200_device.cuh. */
int pb2_acc_pack_launch(const uint64_t* handles, uint32_t handle_count, const void* arg_data, const uint32_t* arg_desc,
                        uint32_t arg_count, void* dst, size_t dst_size, size_t* needed);
/* Future<void>: wait, poll, release (the reference's FutureImpl::wait / ready). */
int pb2_future_wait(pb2_future* future);
int pb2_future_ready(pb2_future* future, int* ready);
int pb2_future_release(pb2_future* future);

#ifdef __cplusplus
}
#endif
#endif /* PIPER2_B200_H */
