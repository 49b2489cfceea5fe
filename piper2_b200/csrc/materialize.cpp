// materialize.cpp -- Piper component payloads -> pb2_scene / pb2_render_settings (pb2_builder_*).
//
// A Piper tracer plugin sees the render path's components only through what their materialize() calls
// hand it: a program symbol name (Tracer::buildProgram) with a POD payload, and the calls and resources the
// payloads reference (MaterializeContext::registerCall / registerResource, Tracer.hpp:86-91, 121-133).  The
// reference's Embree tracer links the programs by symbol and copies the payloads into its SBT arena
// (Tracer/Embree/Embree.cpp:1046-1052, 1055-1274).  Here the symbol selects a decoder that reads the payload
// in the reference's byte layout and fills the C ABI's scene description; unknown symbols are an error.
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "pb2_internal.h"

namespace pb2 {
namespace payload {

// Byte layouts of the reference's payload PODs.  Every physical quantity (Distance, Dimensionless, Radiance,
// Area, ...) is one float, Spectrum / Point / Vector / Normal are three, Vector2 two; handles (TraversalHandle,
// CallHandle inside Call<...>, StatisticsHandle) are pointers, 8 bytes.
struct V3 {
    float x, y, z;
};
// PerspectiveCamera/Shared.hpp:22-29
struct PCData {
    uint64_t traversal;
    V3 look_at;
    float size[2];  // metres (the component scales its mm config by 1e-3)
    V3 up;
    float focal_length;
    float aperture_radius;
};
static_assert(sizeof(PCData) == 48, "PCData layout");
// PathTracing/Shared.hpp:22-29
struct PathTracingData {
    uint32_t max_depth;
    uint32_t min_rr_depth;
    uint64_t statistics[3];
};
static_assert(sizeof(PathTracingData) == 32, "PathTracing Data layout");
// FixedSampler/Shared.hpp: RDData and GaussianFilterData
struct RDData {
    uint64_t filter;
};
struct GaussianFilterData {
    float neg_alpha, sub;
};
// ProceduralTexture/Shared.hpp: ConstantData
struct ConstantData {
    uint32_t channel;
    float value[4];
};
static_assert(sizeof(ConstantData) == 20, "ConstantData layout");
// Surface/Classic/Shared.hpp: texture calls of each surface, in declaration order
struct MatteData {
    uint64_t diffuse, roughness;
};
struct PlasticData {
    uint64_t diffuse, specular, roughness;
};
struct MirrorData {
    uint64_t reflection;
};
struct GlassData {
    uint64_t reflection, transmission, roughness_x, roughness_y;
};
struct SubstrateData {
    uint64_t diffuse, specular, roughness_x, roughness_y;
};
// BasicLight/Shared.hpp: SampledEnvironmentData
struct SampledEnvironmentData {
    uint64_t traversal;
    V3 radiance;
};
static_assert(sizeof(SampledEnvironmentData) == 24, "SampledEnvironmentData layout");
// AreaLight/Shared.hpp: DiffuseAreaLightData
struct DiffuseAreaLightData {
    V3 radiance;
    uint64_t sample;  // Call<GeometrySampleFunc>
    float area;
};
static_assert(sizeof(DiffuseAreaLightData) == 32, "DiffuseAreaLightData layout");
// BasicShapes/Shared.hpp: CDFData (the plane geometry's sample call) and PerPlaneData (= pb2_plane)
struct CDFData {
    uint32_t primitives;  // resource index of PerPlaneData[size]
    uint64_t traversal;
    uint32_t cdf, pdf;    // resource indices of the area CDF and pdf
    float inverse_area;
    uint32_t size;
};
static_assert(sizeof(CDFData) == 32, "CDFData layout");
static_assert(sizeof(pb2_plane) == 64, "PerPlaneData layout");

}  // namespace payload
}  // namespace pb2

struct pb2_builder {
    struct Call {
        std::string symbol;
        std::vector<unsigned char> payload;
    };
    std::vector<std::vector<unsigned char>> resources;
    std::vector<Call> calls;  // CallHandle value = index + 1
    struct Node {
        float m[12];    // row-major 3x4 local-to-world
        bool linear;    // the linear part is not the identity (a rotation, scale or skew)
    };
    std::unordered_map<uint64_t, Node> nodes;
    bool sensor = false, integrator = false, driver = false, sampler = false, light_sampler = false, env = false;
    pb2::payload::PCData camera{};
    uint32_t max_depth = 0, min_rr_depth = 0, filter = PB2_FILTER_BOX;
    float gaussian_alpha = 0.0f;
    float env_radiance[3] = { 0, 0, 0 };
    std::vector<pb2_material> materials;
    std::vector<pb2_plane> planes;
    std::vector<pb2_area_light> area_lights;
    struct Mesh {
        std::vector<float> vertices, texcoords, transform;
        std::vector<uint32_t> indices;
        pb2_mesh desc;
    };
    std::vector<Mesh> meshes;
    std::vector<pb2_mesh> mesh_descs;  // filled by pb2_builder_build
};

using namespace pb2;

namespace {

template <class T>
int read_payload(const void* payload, size_t bytes, const char* symbol, T& out) {
    if (bytes != sizeof(T) || !payload)
        return fail(PB2_ERR_INVALID_ARGUMENT, std::string("payload of '") + symbol + "': " + std::to_string(bytes) +
                                                  " bytes, its layout has " + std::to_string(sizeof(T)));
    std::memcpy(&out, payload, sizeof(T));
    return PB2_OK;
}

const pb2_builder::Call* find_call(const pb2_builder* b, uint64_t handle) {
    if (handle == 0 || handle > b->calls.size()) return nullptr;
    return &b->calls[handle - 1];
}

// The value of a texture call (ProceduralTexture "constantTexture"; Texture/ProceduralTexture/Kernel.cpp:21-26).
int texture_value(const pb2_builder* b, uint64_t handle, float (&v)[4]) {
    const pb2_builder::Call* c = find_call(b, handle);
    if (!c) return fail(PB2_ERR_INVALID_ARGUMENT, "texture call handle " + std::to_string(handle) + " is not registered");
    if (c->symbol != "constantTexture")
        return fail(PB2_ERR_NOT_SUPPORTED, "texture program '" + c->symbol + "': only constantTexture is supported");
    payload::ConstantData d;
    if (int rc = read_payload(c->payload.data(), c->payload.size(), "constantTexture", d)) return rc;
    for (int k = 0; k < 4; ++k) v[k] = d.value[k];
    return PB2_OK;
}

int surface(pb2_builder* b, const std::string& sym, const void* p, size_t n, pb2_material& m) {
    std::memset(&m, 0, sizeof(m));
    float t0[4] = {}, t1[4] = {}, r0[4] = {}, r1[4] = {};
    int rc = PB2_OK;
    if (sym == "blackBodyInit") {
        m.type = PB2_SURFACE_BLACKBODY;
        return PB2_OK;
    } else if (sym == "matteInit") {
        payload::MatteData d;
        if ((rc = read_payload(p, n, sym.c_str(), d)) || (rc = texture_value(b, d.diffuse, t0)) ||
            (rc = texture_value(b, d.roughness, r0)))
            return rc;
        m.type = PB2_SURFACE_MATTE;
    } else if (sym == "plasticInit") {
        payload::PlasticData d;
        if ((rc = read_payload(p, n, sym.c_str(), d)) || (rc = texture_value(b, d.diffuse, t0)) ||
            (rc = texture_value(b, d.specular, t1)) || (rc = texture_value(b, d.roughness, r0)))
            return rc;
        m.type = PB2_SURFACE_PLASTIC;
    } else if (sym == "glassInit") {
        payload::GlassData d;
        if ((rc = read_payload(p, n, sym.c_str(), d)) || (rc = texture_value(b, d.reflection, t0)) ||
            (rc = texture_value(b, d.transmission, t1)) || (rc = texture_value(b, d.roughness_x, r0)) ||
            (rc = texture_value(b, d.roughness_y, r1)))
            return rc;
        m.type = PB2_SURFACE_GLASS;
    } else if (sym == "mirrorInit") {
        payload::MirrorData d;
        if ((rc = read_payload(p, n, sym.c_str(), d)) || (rc = texture_value(b, d.reflection, t0))) return rc;
        m.type = PB2_SURFACE_MIRROR;
    } else if (sym == "substrateInit") {
        payload::SubstrateData d;
        if ((rc = read_payload(p, n, sym.c_str(), d)) || (rc = texture_value(b, d.diffuse, t0)) ||
            (rc = texture_value(b, d.specular, t1)) || (rc = texture_value(b, d.roughness_x, r0)) ||
            (rc = texture_value(b, d.roughness_y, r1)))
            return rc;
        m.type = PB2_SURFACE_SUBSTRATE;
    } else {
        return fail(PB2_ERR_NOT_SUPPORTED, "surface program '" + sym + "' is not supported");
    }
    for (int k = 0; k < 4; ++k) {
        m.color0[k] = t0[k];
        m.color1[k] = t1[k];
    }
    m.roughness[0] = r0[0];
    m.roughness[1] = r1[0];
    return PB2_OK;
}

const pb2_builder::Node* find_node(const pb2_builder* b, uint64_t traversal) {
    auto it = b->nodes.find(traversal);
    return it == b->nodes.end() ? nullptr : &it->second;
}

// The node's origin: its translation, or for a full transform the image of the local origin (the reference's
// rayGen reads only this, Sensor/PerspectiveCamera/Kernel.cpp:25-28).
int node_translation(const pb2_builder* b, uint64_t traversal, float (&t)[3]) {
    const pb2_builder::Node* nd = find_node(b, traversal);
    if (!nd) return fail(PB2_ERR_INVALID_ARGUMENT, "traversal handle " + std::to_string(traversal) + " names no node");
    for (int k = 0; k < 3; ++k) t[k] = nd->m[4 * k + 3];
    return PB2_OK;
}

int light(pb2_builder* b, const std::string& sym, const void* p, size_t n, uint32_t* index) {
    int rc;
    if (sym == "SEInit") {
        // the pipeline needs the environment as lights[0] (Tracer/Embree/Embree.cpp:1174-1188)
        if (b->env || !b->area_lights.empty())
            return fail(PB2_ERR_NOT_SUPPORTED, "the environment light must be the first and only infinite light");
        payload::SampledEnvironmentData d;
        if ((rc = read_payload(p, n, sym.c_str(), d))) return rc;
        b->env_radiance[0] = d.radiance.x;
        b->env_radiance[1] = d.radiance.y;
        b->env_radiance[2] = d.radiance.z;
        b->env = true;
        if (index) *index = 0;
        return PB2_OK;
    }
    if (sym == "diffuseInit") {
        if (!b->env) return fail(PB2_ERR_NOT_SUPPORTED, "the environment light must come first (lights[0])");
        payload::DiffuseAreaLightData d;
        if ((rc = read_payload(p, n, sym.c_str(), d))) return rc;
        const pb2_builder::Call* c = find_call(b, d.sample);
        if (!c) return fail(PB2_ERR_INVALID_ARGUMENT, "area light: its sample call is not registered");
        if (c->symbol != "planeSample")
            return fail(PB2_ERR_NOT_SUPPORTED, "area light geometry '" + c->symbol + "': only planeSample is supported");
        payload::CDFData cdf;
        if ((rc = read_payload(c->payload.data(), c->payload.size(), "planeSample", cdf))) return rc;
        if (cdf.primitives >= b->resources.size())
            return fail(PB2_ERR_INVALID_ARGUMENT, "planeSample: primitive resource out of range");
        const std::vector<unsigned char>& res = b->resources[cdf.primitives];
        if (cdf.size == 0 || res.size() != (size_t)cdf.size * sizeof(pb2_plane))
            return fail(PB2_ERR_INVALID_ARGUMENT, "planeSample: the primitive resource is not size x PerPlaneData");
        pb2_area_light al{};
        if ((rc = node_translation(b, cdf.traversal, al.translation))) return rc;
        const pb2_builder::Node* nd = find_node(b, cdf.traversal);
        if (nd->linear) al.translation[0] = al.translation[1] = al.translation[2] = 0.0f;  // planes mapped below
        al.radiance[0] = d.radiance.x;
        al.radiance[1] = d.radiance.y;
        al.radiance[2] = d.radiance.z;
        al.first_plane = (uint32_t)b->planes.size();
        al.plane_count = cdf.size;
        for (uint32_t i = 0; i < cdf.size; ++i) {
            pb2_plane pl;
            std::memcpy(&pl, res.data() + i * sizeof(pb2_plane), sizeof(pl));
            if (nd->linear) {
                pb2_plane local = pl;
                if ((rc = pb2_plane_transform(&local, nd->m, &pl))) return rc;
            }
            b->planes.push_back(pl);
        }
        b->area_lights.push_back(al);
        if (index) *index = (uint32_t)b->area_lights.size();  // light index: 0 is the environment
        return PB2_OK;
    }
    return fail(PB2_ERR_NOT_SUPPORTED, "light program '" + sym + "' is not supported");
}

}  // namespace

extern "C" {

int pb2_builder_create(pb2_builder** out) {
    if (!out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_create: null argument");
    *out = new pb2_builder();
    return PB2_OK;
}

int pb2_builder_destroy(pb2_builder* b) {
    delete b;
    return PB2_OK;
}

int pb2_builder_register_resource(pb2_builder* b, const void* data, size_t bytes, uint32_t* index) {
    if (!b || !index || (bytes && !data)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_register_resource: null");
    const unsigned char* p = static_cast<const unsigned char*>(data);
    b->resources.emplace_back(p, p + bytes);
    *index = (uint32_t)(b->resources.size() - 1);
    return PB2_OK;
}

int pb2_builder_register_call(pb2_builder* b, const char* symbol, const void* payload, size_t bytes,
                              uint64_t* handle) {
    if (!b || !symbol || !handle || (bytes && !payload))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_register_call: null argument");
    const unsigned char* p = static_cast<const unsigned char*>(payload);
    b->calls.push_back({ std::string(symbol), std::vector<unsigned char>(p, p + bytes) });
    *handle = (uint64_t)b->calls.size();
    return PB2_OK;
}

int pb2_builder_add_node(pb2_builder* b, uint64_t traversal, const float translation[3]) {
    if (!b || !translation) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_node: null argument");
    pb2_builder::Node nd{ { 1, 0, 0, translation[0], 0, 1, 0, translation[1], 0, 0, 1, translation[2] }, false };
    b->nodes[traversal] = nd;
    return PB2_OK;
}

int pb2_builder_add_node_transform(pb2_builder* b, uint64_t traversal, const float matrix[12]) {
    if (!b || !matrix) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_node_transform: null argument");
    pb2_builder::Node nd{};
    for (int i = 0; i < 12; ++i) {
        if (!std::isfinite(matrix[i]))
            return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_node_transform: non-finite entry");
        nd.m[i] = matrix[i];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) nd.linear |= matrix[4 * r + c] != (r == c ? 1.0f : 0.0f);
    b->nodes[traversal] = nd;
    return PB2_OK;
}

int pb2_builder_add_program(pb2_builder* b, uint32_t kind, const char* symbol, const void* p, size_t n,
                            uint32_t* index) {
    if (!b || !symbol) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_program: null argument");
    const std::string sym(symbol);
    if (index) *index = 0;
    int rc;
    switch (kind) {
    case PB2_PROGRAM_SENSOR:  // PerspectiveCamera rayGen (Sensor/PerspectiveCamera/PerspectiveCamera.cpp:51-60)
        if (sym != "rayGen") break;
        if ((rc = read_payload(p, n, symbol, b->camera))) return rc;
        b->sensor = true;
        return PB2_OK;
    case PB2_PROGRAM_INTEGRATOR: {  // PathTracing trace (Integrator/PathTracing/PathTracing.cpp:42-56)
        if (sym != "trace") break;
        payload::PathTracingData d;
        if ((rc = read_payload(p, n, symbol, d))) return rc;
        b->max_depth = d.max_depth;
        b->min_rr_depth = d.min_rr_depth;
        b->integrator = true;
        return PB2_OK;
    }
    case PB2_PROGRAM_RENDER_DRIVER: {  // FixedSampler accumulate + filter call (FixedSampler.cpp:45-55, 135-143)
        if (sym != "accumulate") break;
        payload::RDData d;
        if ((rc = read_payload(p, n, symbol, d))) return rc;
        const pb2_builder::Call* c = find_call(b, d.filter);
        if (!c) return fail(PB2_ERR_INVALID_ARGUMENT, "render driver: its filter call is not registered");
        if (c->symbol == "box") b->filter = PB2_FILTER_BOX;
        else if (c->symbol == "triangle") b->filter = PB2_FILTER_TRIANGLE;
        else if (c->symbol == "gaussian") {
            payload::GaussianFilterData g;
            if ((rc = read_payload(c->payload.data(), c->payload.size(), "gaussian", g))) return rc;
            b->filter = PB2_FILTER_GAUSSIAN;
            b->gaussian_alpha = -g.neg_alpha;
        } else {
            return fail(PB2_ERR_NOT_SUPPORTED, "film filter '" + c->symbol + "' is not supported");
        }
        b->driver = true;
        return PB2_OK;
    }
    case PB2_PROGRAM_SAMPLER:  // ScrambledSobolSampler (ScrambledSobolSampler.cpp:56-64)
        if (sym != "sobolStart" && sym != "sobolGenerate") break;
        b->sampler = true;
        return PB2_OK;
    case PB2_PROGRAM_LIGHT_SAMPLER:  // uniform light selection (Light/BasicLight/BasicLight.cpp:96-104)
        if (sym != "uniformSelect") break;
        b->light_sampler = true;
        return PB2_OK;
    case PB2_PROGRAM_SURFACE: {
        pb2_material m;
        if ((rc = surface(b, sym, p, n, m))) return rc;
        b->materials.push_back(m);
        if (index) *index = (uint32_t)(b->materials.size() - 1);
        return PB2_OK;
    }
    case PB2_PROGRAM_LIGHT:
        return light(b, sym, p, n, index);
    default:
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_program: unknown program kind " + std::to_string(kind));
    }
    return fail(PB2_ERR_NOT_SUPPORTED, "program '" + sym + "' is not supported for its component kind");
}

int pb2_builder_add_mesh(pb2_builder* b, const pb2_mesh* mesh) {
    if (!b || !mesh || (mesh->vert_count && !mesh->vertices) || (mesh->tri_count && !mesh->indices))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_mesh: null argument");
    if (mesh->material >= b->materials.size())
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_add_mesh: material index is not a surface of this builder");
    pb2_builder::Mesh m;
    m.vertices.assign(mesh->vertices, mesh->vertices + 3 * (size_t)mesh->vert_count);
    m.indices.assign(mesh->indices, mesh->indices + 3 * (size_t)mesh->tri_count);
    if (mesh->texcoords) m.texcoords.assign(mesh->texcoords, mesh->texcoords + 2 * (size_t)mesh->vert_count);
    if (mesh->transform) m.transform.assign(mesh->transform, mesh->transform + 12);
    m.desc = *mesh;
    b->meshes.push_back(std::move(m));
    return PB2_OK;
}

int pb2_builder_build(pb2_builder* b, uint32_t width, uint32_t height, uint32_t fit_mode, uint32_t spp,
                      pb2_scene* scene, pb2_render_settings* st) {
    if (!b || !scene || !st) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_builder_build: null argument");
    const char* missing = !b->sensor ? "a sensor (rayGen)" : !b->integrator ? "an integrator (trace)"
                          : !b->driver ? "a render driver (accumulate)" : !b->sampler ? "a sampler (sobolStart)"
                          : !b->light_sampler ? "a light sampler (uniformSelect)" : !b->env ? "an environment light (SEInit)"
                                                                                              : nullptr;
    if (missing) return fail(PB2_ERR_INVALID_ARGUMENT, std::string("pb2_builder_build: the pipeline has no ") + missing);
    float position[3];
    if (int rc = node_translation(b, b->camera.traversal, position)) return rc;
    b->mesh_descs.clear();
    for (pb2_builder::Mesh& m : b->meshes) {
        pb2_mesh d = m.desc;
        d.vertices = m.vertices.data();
        d.indices = m.indices.data();
        d.texcoords = m.texcoords.empty() ? nullptr : m.texcoords.data();
        d.transform = m.transform.empty() ? nullptr : m.transform.data();
        b->mesh_descs.push_back(d);
    }
    std::memset(scene, 0, sizeof(*scene));
    scene->meshes = b->mesh_descs.data();
    scene->mesh_count = (uint32_t)b->mesh_descs.size();
    scene->planes = b->planes.data();
    scene->plane_count = (uint32_t)b->planes.size();
    scene->area_lights = b->area_lights.data();
    scene->area_light_count = (uint32_t)b->area_lights.size();
    scene->materials = b->materials.data();
    scene->material_count = (uint32_t)b->materials.size();
    for (int k = 0; k < 3; ++k) scene->env_radiance[k] = b->env_radiance[k];
    std::memset(st, 0, sizeof(*st));
    st->width = width;
    st->height = height;
    st->fit_mode = fit_mode;
    st->samples_per_pixel = spp;
    st->scramble = 0;  // the reference's Scramble is notImplemented (ScrambledSobolSampler.cpp:51-53)
    st->max_depth = b->max_depth;
    st->min_rr_depth = b->min_rr_depth;
    st->filter = b->filter;
    st->gaussian_alpha = b->gaussian_alpha;
    const payload::PCData& c = b->camera;
    for (int k = 0; k < 3; ++k) st->camera.position[k] = position[k];
    st->camera.look_at[0] = c.look_at.x;
    st->camera.look_at[1] = c.look_at.y;
    st->camera.look_at[2] = c.look_at.z;
    st->camera.up[0] = c.up.x;
    st->camera.up[1] = c.up.y;
    st->camera.up[2] = c.up.z;
    st->camera.sensor_size[0] = c.size[0];
    st->camera.sensor_size[1] = c.size[1];
    st->camera.focal_length = c.focal_length;
    st->camera.aperture_radius = c.aperture_radius;
    return PB2_OK;
}

}  // extern "C"
