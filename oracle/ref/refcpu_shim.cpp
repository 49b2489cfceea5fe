/*
 * refcpu_shim.cpp -- host shim that runs the reference's own device code natively on the CPU.
 * TEST INFRASTRUCTURE ONLY: the reference harness pins the C oracle (pb2_oracle.c) and is the CPU
 * baseline of the render path.  It is compiled together with the reference's unmodified Kernel.cpp
 * files (see Makefile) into oracle/_ref/librefcpu.so.
 *
 * In the reference, the Embree tracer links those kernels with a "Native" symbol table and JITs them
 * (Src/BuiltinComponent/Tracer/Embree/Embree.cpp:1030-1274), the Parallel accelerator provides the
 * task runtime (Src/Infrastructure/Accelerator/Parallel/Parallel.cpp:249-253, Kernel.cpp:22-30), and
 * Embree answers the traversal queries (Embree.cpp:267-391).  This shim provides the same symbols:
 *   - the task runtime (piperGetTaskIndex / piperGetArgument / resource lookup),
 *   - the static redirects embree* -> sobol*, trace, accumulate, uniformSelect (Embree.cpp:1171-1237),
 *   - piperTrace / piperOcclude: triangles through the oracle's watertight test, area-light planes
 *     through the reference's own planeIntersect / planeSurface callbacks, and the result assembly of
 *     piperEmbreeTrace (Embree.cpp:302-352) including its calcInverse of the instance transform,
 *   - piperQueryTransform (Embree.cpp:398-413) for translation-only nodes.
 * Everything else -- sampler, camera, integrator, BxDFs, lights, film -- is the reference's code.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "BuiltinComponent/Geometry/BasicShapes/Shared.hpp"
#include "BuiltinComponent/Integrator/PathTracing/Shared.hpp"
#include "BuiltinComponent/Light/AreaLight/Shared.hpp"
#include "BuiltinComponent/Light/BasicLight/Shared.hpp"
#include "BuiltinComponent/RenderDriver/FixedSampler/Shared.hpp"
#include "BuiltinComponent/Sampler/ScrambledSobolSampler/Shared.hpp"
#include "BuiltinComponent/Sensor/PerspectiveCamera/Shared.hpp"
#include "BuiltinComponent/Surface/Classic/Shared.hpp"
#include "BuiltinComponent/Texture/ProceduralTexture/Shared.hpp"
#include "BuiltinComponent/Tracer/Embree/Shared.hpp"

extern "C" {
#include "pb2_oracle.h"
}

using namespace Piper;

/* ---- reference kernel symbols this shim binds (extern "C" in the reference's Kernel.cpp files) -- */
namespace Piper {
extern "C" {
void sobolStart(const void*, uint32_t, uint32_t, uint32_t, uint64_t&, Vector2<float>&);
void sobolGenerate(const void*, uint64_t, uint32_t, float&);
void rayGen(RestrictedContext, const void*, const Vector2<float>&, float, float, RayInfo<FOR::World>&, Dimensionless<float>&);
void trace(FullContext, const void*, RayInfo<FOR::World>&, Spectrum<Radiance>&);
void accumulate(RestrictedContext, const void*, const void*, const Vector2<float>&, const Spectrum<Radiance>&);
void box(RestrictedContext, const void*, float, float, Dimensionless<float>&);
void triangle(RestrictedContext, const void*, float, float, Dimensionless<float>&);
void gaussian(RestrictedContext, const void*, float, float, Dimensionless<float>&);
void uniformSelect(RestrictedContext, const void*, float, LightSelectResult&);
void SEInit(RestrictedContext, const void*, void*);
void SESample(RestrictedContext, const void*, const void*, const Point<Distance, FOR::World>&, float, float, LightSample&);
void SEEvaluate(RestrictedContext, const void*, const void*, const Point<Distance, FOR::World>&, const Normal<float, FOR::World>&,
                const Normal<float, FOR::World>&, Spectrum<Radiance>&);
void SEPdf(RestrictedContext, const void*, const void*, const Point<Distance, FOR::World>&, const Normal<float, FOR::World>&,
           const Normal<float, FOR::World>&, Distance, Dimensionless<float>&);
void diffuseInit(RestrictedContext, const void*, void*);
void diffuseSample(RestrictedContext, const void*, const void*, const Point<Distance, FOR::World>&, float, float, LightSample&);
void diffuseEvaluate(RestrictedContext, const void*, const void*, const Point<Distance, FOR::World>&,
                     const Normal<float, FOR::World>&, const Normal<float, FOR::World>&, Spectrum<Radiance>&);
void diffusePdf(RestrictedContext, const void*, const void*, const Point<Distance, FOR::World>&, const Normal<float, FOR::World>&,
                const Normal<float, FOR::World>&, Distance, Dimensionless<float>&);
void planeIntersect(RestrictedContext, const void*, uint32_t, const RayInfo<FOR::Local>&, float, float&, void*);
void planeSurface(RestrictedContext, const void*, const void*, SurfaceIntersectionInfo&);
void planeSample(RestrictedContext, const void*, const Point<Distance, FOR::World>&, float, float, Point<Distance, FOR::World>&,
                 Normal<float, FOR::World>&, Dimensionless<float>&);
void constantTexture(RestrictedContext, const void*, const Vector2<float>&, Dimensionless<float>*);
void checkBoard(RestrictedContext, const void*, const Vector2<float>&, Dimensionless<float>*);
void sampleTexture(RestrictedContext, const void*, const Vector2<float>&, Dimensionless<float>*);
void calcTriangleMeshSurface(RestrictedContext, const void*, const void*, SurfaceIntersectionInfo&);
void piperMain(TaskContext ctx);
#define SURFACE_DECL(P)                                                                                          \
    void P##Init(RestrictedContext, const void*, const Vector2<float>&, const Normal<float, FOR::Shading>&, Face, \
                 TransportMode, void*, bool&);                                                                   \
    void P##Sample(RestrictedContext, const void*, const void*, const Normal<float, FOR::Shading>&,             \
                   const Normal<float, FOR::Shading>&, BxDFPart, float, float, SurfaceSample&);                 \
    void P##Evaluate(RestrictedContext, const void*, const void*, const Normal<float, FOR::Shading>&,           \
                     const Normal<float, FOR::Shading>&, const Normal<float, FOR::Shading>&, BxDFPart,          \
                     Spectrum<Dimensionless<float>>&);                                                          \
    void P##Pdf(RestrictedContext, const void*, const void*, const Normal<float, FOR::Shading>&,                \
                const Normal<float, FOR::Shading>&, const Normal<float, FOR::Shading>&, BxDFPart, Dimensionless<float>&);
SURFACE_DECL(blackBody)
SURFACE_DECL(matte)
SURFACE_DECL(plastic)
SURFACE_DECL(glass)
SURFACE_DECL(substrate)
void mirrorInit(RestrictedContext, const void*, const Vector2<float>&, const Normal<float, FOR::Shading>&, Face, TransportMode,
                void*, bool&);
void mirrorSample(RestrictedContext, const void*, const void*, const Normal<float, FOR::Shading>&,
                  const Normal<float, FOR::Shading>&, BxDFPart, float, float, SurfaceSample&);
}
}  // namespace Piper

/* ---- task runtime (Parallel/Kernel.cpp:22-30, Parallel.cpp:249-253) -------------------------------- */
namespace Piper {
struct TaskContextReserved {
    Dim3 index;
    const KernelArgument* arg;
};
}  // namespace Piper

struct TraversalNodeShim {
    float translation[3];
};

static std::vector<void*>* g_resources = nullptr;
static thread_local float* t_sample_out = nullptr;

namespace Piper {
extern "C" {
int8_t** piperBuiltinSymbolLUT = nullptr;

void piperGetTaskIndex(TaskContext context, Dim3& index) { index = context->index; }
void piperGetArgument(TaskContext context, uint32_t, void* ptr) { std::memcpy(ptr, context->arg, sizeof(KernelArgument)); }
void piperGetRootResourceLUT(TaskContext, ResourceHandle& handle) { handle = 0; }
void piperLookUpResourceHandle(TaskContext, ResourceHandle, uint32_t index, ResourceHandle& handle) {
    handle = reinterpret_cast<ResourceHandle>((*g_resources)[index]);
}

/* static redirects (Embree.cpp:1171, 1220, 1231, 1236-1237) */
void embreeSampleGenerate(const void* SBTData, uint64_t idx, uint32_t dim, float& val) { sobolGenerate(SBTData, idx, dim, val); }
void embreeSampleStart(const void* SBTData, uint32_t x, uint32_t y, uint32_t s, uint64_t& idx, Vector2<float>& off) {
    sobolStart(SBTData, x, y, s, idx, off);
}
void embreeIntegrate(FullContext context, const void* SBTData, RayInfo<FOR::World>& ray, Spectrum<Radiance>& sample) {
    trace(context, SBTData, ray, sample);
}
void embreeAccumulate(RestrictedContext context, const void* SBTData, const void* launchData, const Vector2<float>& point,
                      const Spectrum<Radiance>& sample) {
    if (t_sample_out) {
        t_sample_out[0] = point.x; t_sample_out[1] = point.y;
        t_sample_out[2] = sample.r.val; t_sample_out[3] = sample.g.val; t_sample_out[4] = sample.b.val;
    }
    accumulate(context, SBTData, launchData, point, sample);
}
void embreeLightSelect(RestrictedContext context, const void* SBTData, float u, LightSelectResult& select) {
    uniformSelect(context, SBTData, u, select);
}

void piperStatisticsUInt(RestrictedContext, StatisticsHandle, uint32_t) {}
void piperStatisticsBool(RestrictedContext, StatisticsHandle, bool) {}
void piperStatisticsFloat(RestrictedContext, StatisticsHandle, float) {}
void piperStatisticsTime(RestrictedContext, StatisticsHandle, uint64_t) {}
void piperGetTime(RestrictedContext, uint64_t& val) { val = 0; }
void piperPrintFloat(RestrictedContext, const char*, float) {}

/* piperEmbreeFloatAtomicAdd (Embree.cpp:420-428) */
void piperFloatAtomicAdd(float& x, float y) {
    auto& a = *reinterpret_cast<std::atomic<float>*>(&x);
    float src = a.load(std::memory_order_relaxed);
    while (!a.compare_exchange_weak(src, src + y, std::memory_order_release, std::memory_order_relaxed)) {
    }
}

/* piperEmbreeQueryTransform (Embree.cpp:398-413) for a single translation-only node */
void piperQueryTransform(RestrictedContext, TraversalHandle traversal, Transform<Distance, FOR::Local, FOR::World>& transform) {
    const auto* node = reinterpret_cast<const TraversalNodeShim*>(traversal);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) transform.A2B[r][c].val = (c == r) ? 1.0f : 0.0f;
    for (int r = 0; r < 3; ++r) transform.A2B[r][3].val = node ? node->translation[r] : 0.0f;
    calcInverse(transform.A2B, transform.B2A);
}
}
}  // namespace Piper

/* ---- scene ------------------------------------------------------------------------------------- */
struct RefScene {
    or_scene* oracle = nullptr;
    std::vector<void*> symbols;
    std::vector<const void*> callInfo;
    std::vector<void*> resources;
    std::vector<std::vector<uint8_t>> payloads;
    std::vector<TraversalNodeShim*> nodes;
    std::vector<GSMInstanceUserData*> gsm;       /* per mesh */
    std::vector<AreaLightUserData*> areaUser;    /* per area light */
    std::vector<uint32_t> meshFirstPrim;
    std::vector<TraversalNodeShim*> meshNode;
    std::vector<BuiltinTriangleBuffer*> meshBuffer;
    std::vector<std::vector<uint32_t>> meshIndex;
    std::vector<uint32_t> lightFirstPlane, lightPlaneCount;
    std::vector<PlaneData*> lightPlaneData;
    std::vector<TraversalNodeShim*> lightNode;
    LightFuncGroup* lights = nullptr;
    KernelArgument arg{};
    uint32_t rgbwResource = 0;
    float* rgbw = nullptr;

    template <typename T>
    T* payload(const T& v) {
        payloads.emplace_back(sizeof(T));
        std::memcpy(payloads.back().data(), &v, sizeof(T));
        return reinterpret_cast<T*>(payloads.back().data());
    }
    template <typename F>
    CallHandle call(F* fn, const void* sbt) {
        symbols.push_back(reinterpret_cast<void*>(fn));
        callInfo.push_back(sbt);
        return reinterpret_cast<CallHandle>(static_cast<ptrdiff_t>(symbols.size() - 1));
    }
    uint32_t resource(void* p) {
        resources.push_back(p);
        return static_cast<uint32_t>(resources.size() - 1);
    }
    CallHandle constant(const float* v, uint32_t channel) {
        ConstantData d{};
        d.channel = channel;
        for (uint32_t i = 0; i < channel; ++i) d.value[i].val = v[i];
        return call(&constantTexture, payload(d));
    }
    /* The payload of the SampledTexture kernel (its Data, Texture/SampledTexture/Shared.hpp:22-30; a struct of the
     * same name in the PathTracing header keeps it from being included beside the others). */
    struct SampledTextureData {
        TextureWrap wrap;
        uint32_t width, height, stride, channel, texel;
        StatisticsHandle profileSample;
    };
    /* A material parameter: its constant, or the scene texture it names (CheckBoard / SampledTexture). */
    CallHandle texture(const pb2_scene* d, uint32_t index, const float* v, uint32_t channel) {
        if (!index) return constant(v, channel);
        const pb2_texture& t = d->textures[index - 1];
        if (t.kind == PB2_TEXTURE_CHECKERBOARD) {
            CheckBoardData c{};
            c.scale = t.scale;
            c.channel = t.channel;
            for (uint32_t i = 0; i < 4; ++i) { c.black[i].val = t.black[i]; c.white[i].val = t.white[i]; }
            return call(&checkBoard, payload(c));
        }
        SampledTextureData sd{};
        sd.wrap = t.wrap ? TextureWrap::Mirror : TextureWrap::Repeat;
        sd.width = t.width;
        sd.height = t.height;
        sd.stride = t.width * t.channel;
        sd.channel = t.channel;
        sd.texel = resource(const_cast<uint8_t*>(t.texels));
        sd.profileSample = nullptr;
        return call(&sampleTexture, payload(sd));
    }
    ~RefScene() {
        if (oracle) or_scene_destroy(oracle);
        for (auto* n : nodes) delete n;
    }
};

static TraversalNodeShim* make_node(RefScene* S, const float t[3]) {
    auto* n = new TraversalNodeShim{ { t[0], t[1], t[2] } };
    S->nodes.push_back(n);
    return n;
}

namespace Piper {
/* piperEmbreeTrace (Embree.cpp:267-355) with Embree replaced */
extern "C" void piperTrace(FullContext context, const RayInfo<FOR::World>& ray, float minT, float maxT, TraceResult& result) {
    const auto* ctx = reinterpret_cast<const PerSampleContext*>(context);
    auto* S = reinterpret_cast<RefScene*>(ctx->argument.scene);
    pb2_ray r{ { ray.origin.x.val, ray.origin.y.val, ray.origin.z.val }, minT,
               { ray.direction.x.val, ray.direction.y.val, ray.direction.z.val }, maxT };
    pb2_hit h;
    const int triHit = or_closest_triangle(S->oracle, &r, &h);
    float tFar = triHit ? h.t : maxT;
    GeometryStorage storage;
    int planeLight = -1;
    for (size_t l = 0; l < S->lightFirstPlane.size(); ++l) {
        const float* t = S->lightNode[l]->translation;
        const RayInfo<FOR::Local> local{
            Point<Distance, FOR::Local>{ { ray.origin.x.val - t[0] }, { ray.origin.y.val - t[1] }, { ray.origin.z.val - t[2] } },
            Normal<float, FOR::Local>{ Vector<Dimensionless<float>, FOR::Local>{
                { ray.direction.x.val }, { ray.direction.y.val }, { ray.direction.z.val } } }
        };
        for (uint32_t p = 0; p < S->lightPlaneCount[l]; ++p) {
            const float old = tFar;
            planeIntersect(decay(context), S->lightPlaneData[l], p, local, minT, tFar, &storage);
            if (tFar < old) planeLight = static_cast<int>(l);
        }
    }
    if (!triHit && planeLight < 0) {
        result.kind = TraceKind::Missing;
        return;
    }
    result.surface.t = Distance{ tFar };
    const float* t = planeLight >= 0 ? S->lightNode[planeLight]->translation : nullptr;
    uint32_t mesh = 0, local = 0;
    if (planeLight < 0) {
        mesh = static_cast<uint32_t>(std::upper_bound(S->meshFirstPrim.begin(), S->meshFirstPrim.end(), h.prim) -
                                     S->meshFirstPrim.begin()) - 1;
        local = h.prim - S->meshFirstPrim[mesh];
        t = S->meshNode[mesh]->translation;
    }
    for (int rr = 0; rr < 3; ++rr)
        for (int c = 0; c < 4; ++c) result.surface.transform.B2A[rr][c].val = (c == rr) ? 1.0f : 0.0f;
    for (int rr = 0; rr < 3; ++rr) result.surface.transform.B2A[rr][3].val = t[rr];
    calcInverse(result.surface.transform.B2A, result.surface.transform.A2B);
    const GeometryUserData* data;
    if (planeLight < 0) {
        const float* v = or_triangle_vertices(S->oracle, h.prim);
        const float e1[3] = { v[3] - v[0], v[4] - v[1], v[5] - v[2] };
        const float e2[3] = { v[6] - v[0], v[7] - v[1], v[8] - v[2] };
        const Vector<Dimensionless<float>, FOR::World> ng{ { e1[1] * e2[2] - e1[2] * e2[1] }, { e1[2] * e2[0] - e1[0] * e2[2] },
                                                          { e1[0] * e2[1] - e1[1] * e2[0] } };
        auto& builtin = *reinterpret_cast<BuiltinHitInfo*>(&storage);
        builtin.Ng = result.surface.transform(Normal<float, FOR::World>{ ng });
        builtin.index = local;
        builtin.barycentric = { h.u, h.v };
        builtin.face = (dot(result.surface.transform(ray.direction), builtin.Ng).val < 0.0f ? Face::Front : Face::Back);
        data = S->gsm[mesh];
    } else {
        data = S->areaUser[planeLight];
    }
    data->calcSurface(reinterpret_cast<RestrictedContext>(context), &storage, result.surface.intersect);
    if (data->usage == GeometryUsage::GSM) {
        result.kind = TraceKind::Surface;
        result.surface.surface = reinterpret_cast<SurfaceHandle>(data);
    } else {
        result.kind = TraceKind::AreaLight;
        result.surface.light = reinterpret_cast<const AreaLightUserData*>(data)->light;
    }
}

/* piperEmbreeOcclude (Embree.cpp:357-391): mask = GSM only, area-light planes never occlude */
extern "C" bool piperOcclude(FullContext context, const RayInfo<FOR::World>& ray, float minT, float maxT) {
    const auto* ctx = reinterpret_cast<const PerSampleContext*>(context);
    auto* S = reinterpret_cast<RefScene*>(ctx->argument.scene);
    pb2_ray r{ { ray.origin.x.val, ray.origin.y.val, ray.origin.z.val }, minT,
               { ray.direction.x.val, ray.direction.y.val, ray.direction.z.val }, maxT };
    return or_any_triangle(S->oracle, &r) != 0;
}
}  // namespace Piper

/* ---- pipeline construction (the materialize steps of EmbreePipeline, Embree.cpp:1055-1274) ------- */
extern "C" void* ref_scene_create(const pb2_scene* d, const pb2_render_settings* st, int use_bvh) {
    auto* S = new RefScene();
    S->oracle = or_scene_create(d, use_bvh);
    S->resources.reserve(1024);
    /* materials -> surface programs (Classic.cpp:70-199) */
    struct SurfaceCalls { CallHandle init, sample, evaluate, pdf; };
    std::vector<SurfaceCalls> surf(d->material_count);
    for (uint32_t m = 0; m < d->material_count; ++m) {
        const pb2_material& mt = d->materials[m];
        SurfaceCalls& c = surf[m];
        switch (mt.type) {
            case PB2_SURFACE_MATTE: {
                const MatteData* p = S->payload(MatteData{ { S->texture(d, mt.texture[0], mt.color0, 4) },
                                                           { S->texture(d, mt.texture[2], mt.roughness, 1) } });
                c = { S->call(&matteInit, p), S->call(&matteSample, p), S->call(&matteEvaluate, p), S->call(&mattePdf, p) };
            } break;
            case PB2_SURFACE_PLASTIC: {
                const PlasticData* p = S->payload(PlasticData{ { S->texture(d, mt.texture[0], mt.color0, 4) },
                                                              { S->texture(d, mt.texture[1], mt.color1, 4) },
                                                              { S->texture(d, mt.texture[2], mt.roughness, 1) } });
                c = { S->call(&plasticInit, p), S->call(&plasticSample, p), S->call(&plasticEvaluate, p),
                      S->call(&plasticPdf, p) };
            } break;
            case PB2_SURFACE_GLASS: {
                const GlassData* p = S->payload(GlassData{ { S->texture(d, mt.texture[0], mt.color0, 4) },
                                                          { S->texture(d, mt.texture[1], mt.color1, 4) },
                                                          { S->texture(d, mt.texture[2], &mt.roughness[0], 1) },
                                                          { S->texture(d, mt.texture[3], &mt.roughness[1], 1) } });
                c = { S->call(&glassInit, p), S->call(&glassSample, p), S->call(&glassEvaluate, p), S->call(&glassPdf, p) };
            } break;
            case PB2_SURFACE_MIRROR: {
                const MirrorData* p = S->payload(MirrorData{ { S->texture(d, mt.texture[0], mt.color0, 4) } });
                c = { S->call(&mirrorInit, p), S->call(&mirrorSample, p), S->call(&blackBodyEvaluate, p),
                      S->call(&blackBodyPdf, p) };
            } break;
            case PB2_SURFACE_SUBSTRATE: {
                const SubstrateData* p = S->payload(SubstrateData{ { S->texture(d, mt.texture[0], mt.color0, 4) },
                                                                  { S->texture(d, mt.texture[1], mt.color1, 4) },
                                                                  { S->texture(d, mt.texture[2], &mt.roughness[0], 1) },
                                                                  { S->texture(d, mt.texture[3], &mt.roughness[1], 1) } });
                c = { S->call(&substrateInit, p), S->call(&substrateSample, p), S->call(&substrateEvaluate, p),
                      S->call(&substratePdf, p) };
            } break;
            default: /* black body; the conductor extension has no reference counterpart */
                c = { S->call(&blackBodyInit, nullptr), S->call(&blackBodySample, nullptr), S->call(&blackBodyEvaluate, nullptr),
                      S->call(&blackBodyPdf, nullptr) };
                break;
        }
    }
    /* meshes -> GSM instances with the builtin triangle surface (Embree.cpp:1142-1150, 1246-1258) */
    uint32_t first = 0;
    for (uint32_t i = 0; i < d->mesh_count; ++i) {
        const pb2_mesh& mesh = d->meshes[i];
        S->meshFirstPrim.push_back(first);
        first += mesh.tri_count;
        S->meshNode.push_back(make_node(S, mesh.translation));
        S->meshIndex.emplace_back(mesh.indices, mesh.indices + 3 * (size_t)mesh.tri_count);
        BuiltinTriangleBuffer buf{ S->meshIndex.back().data(), reinterpret_cast<const Vector2<float>*>(mesh.texcoords), nullptr,
                                   nullptr };
        const auto* bufp = S->payload(buf);
        auto* u = new GSMInstanceUserData{};
        u->kind = HitKind::Builtin;
        u->calcSurface = { S->call(&calcTriangleMeshSurface, bufp) };
        u->usage = GeometryUsage::GSM;
        const SurfaceCalls& c = surf[mesh.material];
        u->init = { c.init }; u->sample = { c.sample }; u->evaluate = { c.evaluate }; u->pdf = { c.pdf };
        S->gsm.push_back(u);
    }
    /* lights: lights[0] = the environment, then the area lights (Embree.cpp:1174-1214) */
    const uint32_t nl = 1 + d->area_light_count;
    S->lights = new LightFuncGroup[nl];
    {
        SampledEnvironmentData env{};
        env.traversal = reinterpret_cast<TraversalHandle>(make_node(S, (const float[3]){ 0, 0, 0 }));
        env.texture = Spectrum<Radiance>{ { d->env_radiance[0] }, { d->env_radiance[1] }, { d->env_radiance[2] } };
        const auto* p = S->payload(env);
        S->lights[0] = { { S->call(&SEInit, p) }, { S->call(&SESample, p) }, { S->call(&SEEvaluate, p) }, { S->call(&SEPdf, p) } };
    }
    for (uint32_t l = 0; l < d->area_light_count; ++l) {
        const pb2_area_light& al = d->area_lights[l];
        auto* node = make_node(S, al.translation);
        S->lightNode.push_back(node);
        /* Plane geometry (BasicShapes.cpp:62-95) */
        auto* planes = new std::vector<PerPlaneData>(al.plane_count);
        std::memcpy(planes->data(), d->planes + al.first_plane, sizeof(PerPlaneData) * al.plane_count);
        static_assert(sizeof(PerPlaneData) == sizeof(pb2_plane), "PerPlaneData layout");
        auto* cdf = new std::vector<float>(al.plane_count);
        auto* pdf = new std::vector<float>(al.plane_count);
        float area = 0.0f;
        for (uint32_t i = 0; i < al.plane_count; ++i) {
            const auto& pl = (*planes)[i];
            const auto det3 = cross(pl.u, pl.v);
            const float a = length(det3).val;
            area = area + a;
            (*cdf)[i] = area;
            (*pdf)[i] = a;
        }
        for (auto& x : *cdf) x = x / area;
        for (auto& x : *pdf) x = x / area;
        const uint32_t planeRes = S->resource(planes->data());
        const uint32_t cdfRes = S->resource(cdf->data());
        const uint32_t pdfRes = S->resource(pdf->data());
        const auto* planeData = S->payload(PlaneData{ planeRes });
        S->lightPlaneData.push_back(const_cast<PlaneData*>(planeData));
        S->lightFirstPlane.push_back(al.first_plane);
        S->lightPlaneCount.push_back(al.plane_count);
        CDFData cd{};
        cd.primitives = planeRes;
        cd.traversal = reinterpret_cast<TraversalHandle>(node);
        cd.cdf = cdfRes;
        cd.pdf = pdfRes;
        cd.inverseArea = Dimensionless<float>{ 1.0f / area };
        cd.size = al.plane_count;
        const auto* cdp = S->payload(cd);
        DiffuseAreaLightData ld{};
        ld.radiance = Spectrum<Radiance>{ { al.radiance[0] }, { al.radiance[1] }, { al.radiance[2] } };
        ld.sample = { S->call(&planeSample, cdp) };
        ld.area = Area<float>{ area };
        const auto* lp = S->payload(ld);
        S->lights[1 + l] = { { S->call(&diffuseInit, lp) }, { S->call(&diffuseSample, lp) }, { S->call(&diffuseEvaluate, lp) },
                             { S->call(&diffusePdf, lp) } };
        auto* au = new AreaLightUserData{};
        au->kind = HitKind::Custom;
        au->calcSurface = { S->call(&planeSurface, planeData) };
        au->usage = GeometryUsage::AreaLight;
        au->light = reinterpret_cast<LightHandle>(S->lights + 1 + l);
        S->areaUser.push_back(au);
    }
    /* light sampler payload: count + delta flags (BasicLight.cpp:91-101) */
    std::vector<uint8_t> ls(sizeof(uint32_t) + nl, 0);
    std::memcpy(ls.data(), &nl, sizeof(uint32_t));
    S->payloads.push_back(ls);
    const void* lsPayload = S->payloads.back().data();

    /* render driver + filter (FixedSampler.cpp:38-54, 135-144) */
    CallHandle filter;
    if (st->filter == PB2_FILTER_TRIANGLE) filter = S->call(&triangle, nullptr);
    else if (st->filter == PB2_FILTER_GAUSSIAN) {
        GaussianFilterData g{ -st->gaussian_alpha, std::exp(-st->gaussian_alpha) };
        filter = S->call(&gaussian, S->payload(g));
    } else filter = S->call(&box, nullptr);
    const auto* rd = S->payload(RDData{ { filter } });

    /* camera (PerspectiveCamera.cpp:35-61) */
    PCData pc{};
    pc.traversal = reinterpret_cast<TraversalHandle>(make_node(S, st->camera.position));
    pc.lookAt = Point<Distance, FOR::World>{ { st->camera.look_at[0] }, { st->camera.look_at[1] }, { st->camera.look_at[2] } };
    pc.size = Vector2<float>{ st->camera.sensor_size[0], st->camera.sensor_size[1] };
    pc.upRef = Normal<float, FOR::World>{ Vector<Dimensionless<float>, FOR::World>{ { st->camera.up[0] }, { st->camera.up[1] },
                                                                                     { st->camera.up[2] } },
                                          Unsafe{} };
    pc.focalLength = Distance{ st->camera.focal_length };
    pc.apertureRadius = Distance{ st->camera.aperture_radius };
    const CallHandle rg = S->call(&rayGen, S->payload(pc));

    /* integrator (PathTracing.cpp:42-56) */
    const auto* tr = S->payload(Data{ st->max_depth, st->min_rr_depth, nullptr, nullptr, nullptr });

    /* prepare (Embree.cpp:1275-1300) */
    pb2_ndc_transform ndc;
    pb2_rect full;
    or_calc_render_rect(st->width, st->height, st->camera.sensor_size[0] / st->camera.sensor_size[1], st->fit_mode, &ndc, &full);
    const uint32_t log2res = static_cast<uint32_t>(std::ceil(std::log2(static_cast<double>(std::max(full.width, full.height)))));
    const auto* sa = S->payload(SobolData{ 1u << log2res, log2res });

    S->rgbwResource = S->resource(nullptr);
    KernelArgument& a = S->arg;
    a.width = st->width;
    a.height = st->height;
    a.fullRect = { full.left, full.top, full.width, full.height };
    a.rect = a.fullRect;
    a.scene = reinterpret_cast<RTCSceneTy*>(S);
    a.rayGen = { rg };
    a.ACPayload = rd;
    a.TRPayload = tr;
    a.lights = S->lights;
    a.LSPayload = lsPayload;
    a.SAPayload = sa;
    a.sampleCount = 1;
    a.maxDimension = numSobolDimensions;
    a.transform = { ndc.ox, ndc.oy, ndc.sx, ndc.sy };
    a.profiler = nullptr;
    a.debug = false;
    a.errorHandler = nullptr;
    return S;
}

extern "C" void ref_scene_destroy(void* p) { delete reinterpret_cast<RefScene*>(p); }

/* TraceLauncher::launch + the Parallel accelerator's loop (Parallel.cpp:457-494): one task per
 * pixel of `rect`, serial over samples.  rgbw: W*H float4 film; sample_out: 5 floats per sample. */
extern "C" int ref_render(void* p, const pb2_rect* rect, uint32_t sample_begin, uint32_t sample_count, float* rgbw,
                          float* sample_out, int threads) {
    auto* S = reinterpret_cast<RefScene*>(p);
    S->resources[S->rgbwResource] = rgbw;
    g_resources = &S->resources;
    piperBuiltinSymbolLUT = reinterpret_cast<int8_t**>(S->symbols.data());
    KernelArgument arg = S->arg;
    arg.rect = { rect->left, rect->top, rect->width, rect->height };
    arg.callInfo = S->callInfo.data();
    arg.sampleCount = sample_begin + sample_count;
    LaunchData ld{ S->rgbwResource, S->arg.width, S->arg.height };
    arg.launchData = &ld;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (int64_t row = 0; row < (int64_t)rect->height; ++row) {
        for (uint32_t col = 0; col < rect->width; ++col) {
            for (uint32_t k = 0; k < sample_count; ++k) {
                TaskContextReserved task{ Dim3{ static_cast<uint32_t>(row), col, sample_begin + k }, &arg };
                t_sample_out = sample_out ? sample_out + 5 * (((size_t)row * rect->width + col) * sample_count + k) : nullptr;
                piperMain(&task);
            }
        }
    }
    t_sample_out = nullptr;
    return 0;
}

extern "C" float ref_sobol_generate(uint64_t index, uint32_t dim) {
    float v;
    sobolGenerate(nullptr, index, dim, v);
    return v;
}

extern "C" void ref_sobol_start(uint32_t log2res, uint32_t px, uint32_t py, uint32_t sample, uint64_t* index, float* offset) {
    SobolData d{ 1u << log2res, log2res };
    Vector2<float> off;
    sobolStart(&d, px, py, sample, *index, off);
    offset[0] = off.x;
    offset[1] = off.y;
}

/* rayGen through the reference camera (PerspectiveCamera/Kernel.cpp:22-48) */
extern "C" void ref_camera_ray(void* p, float ndc_x, float ndc_y, float u1, float u2, float* out6) {
    auto* S = reinterpret_cast<RefScene*>(p);
    g_resources = &S->resources;
    piperBuiltinSymbolLUT = reinterpret_cast<int8_t**>(S->symbols.data());
    const auto idx = reinterpret_cast<ptrdiff_t>(S->arg.rayGen.handle);
    RayInfo<FOR::World> ray;
    Dimensionless<float> w;
    rayGen(nullptr, S->callInfo[idx], Vector2<float>{ ndc_x, ndc_y }, u1, u2, ray, w);
    out6[0] = ray.origin.x.val; out6[1] = ray.origin.y.val; out6[2] = ray.origin.z.val;
    out6[3] = ray.direction.x.val; out6[4] = ray.direction.y.val; out6[5] = ray.direction.z.val;
}
