// capi.cu -- the C ABI (include/piper2_b200.h): error handling, host-side component helpers, the
// acceleration structure and the batch trace calls.  The render pipeline lives in render.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pb2_internal.h"
#include "sobol_tables_decl.h"

namespace pb2 {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t err, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
    return err == cudaErrorMemoryAllocation ? PB2_ERR_OUT_OF_MEMORY : PB2_ERR_CUDA;
}

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    return dev;
}

cudaError_t smem_attr_once(const void* kernel, size_t bytes, std::atomic<int> (&done)[kMaxDevices]) {
    const int dev = current_device();
    if (dev >= 0 && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess && dev >= 0) done[dev].store(1, std::memory_order_release);
    return e;
}

int resident_grid_cached(const void* kernel, int threads, size_t smem, std::atomic<int> (&cache)[kMaxDevices]) {
    const int dev = current_device();
    if (dev >= 0) {
        const int v = cache[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int sms = 148, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev >= 0 ? dev : 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    if (dev >= 0) cache[dev].store(grid, std::memory_order_relaxed);
    return grid;
}

}  // namespace pb2

using namespace pb2;

#define PB2_CUDA(call, what)                                  \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, (what));  \
    } while (0)

extern "C" {

const char* pb2_last_error(void) { return g_last_error.c_str(); }

int pb2_abi_version(void) { return PB2_ABI_VERSION; }

int pb2_set_device(int device) {
    PB2_CUDA(cudaSetDevice(device), "cudaSetDevice");
    return PB2_OK;
}

/* Plane from Origin/U/V (Src/BuiltinComponent/Geometry/BasicShapes/BasicShapes.cpp:70-89). */
int pb2_plane_make(const float origin[3], const float u[3], const float v[3], pb2_plane* out) {
    if (!origin || !u || !v || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_plane_make: null argument");
    const float d0 = u[1] * v[2] - u[2] * v[1];
    const float d1 = u[2] * v[0] - u[0] * v[2];
    const float d2 = u[0] * v[1] - u[1] * v[0];
    const float area = std::sqrt(std::fmax(d0 * d0 + d1 * d1 + d2 * d2, 0.0f));
    const float ul = std::sqrt(std::fmax(u[0] * u[0] + u[1] * u[1] + u[2] * u[2], 0.0f));
    const float a0 = std::fabs(d0), a1 = std::fabs(d1), a2 = std::fabs(d2);
    uint32_t sel;
    if (a0 >= a1 && a0 >= a2) sel = 0;
    else sel = (a1 >= a0 && a1 >= a2) ? 1 : 2;
    for (int k = 0; k < 3; ++k) {
        out->origin[k] = origin[k];
        out->u[k] = u[k];
        out->v[k] = v[k];
        out->tangent[k] = u[k] / ul;
    }
    out->normal[0] = d0 / area;
    out->normal[1] = d1 / area;
    out->normal[2] = d2 / area;
    out->max_det_comp = sel;
    return PB2_OK;
}

int pb2_srt_matrix(const pb2_srt* srt, float matrix[12]) {
    if (!srt || !matrix) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_srt_matrix: null argument");
    const float* f = reinterpret_cast<const float*>(srt);
    for (int i = 0; i < 16; ++i)
        if (!std::isfinite(f[i])) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_srt_matrix: non-finite entry");
    if (f[9] == 0.0f && f[10] == 0.0f && f[11] == 0.0f && f[12] == 0.0f)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_srt_matrix: zero quaternion");
    pb2_srt_matrix_hd(f, matrix);
    return PB2_OK;
}

int pb2_plane_transform(const pb2_plane* in, const float matrix[12], pb2_plane* out) {
    if (!in || !matrix || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_plane_transform: null argument");
    float o[3], u[3], v[3];
    pb2_xform_point(matrix, in->origin, o);
    pb2_xform_vector(matrix, in->u, u);
    pb2_xform_vector(matrix, in->v, v);
    return pb2_plane_make(o, u, v, out);
}

/* PerspectiveCamera config -> payload (Src/BuiltinComponent/Sensor/PerspectiveCamera/PerspectiveCamera.cpp:39-44) */
int pb2_camera_from_config(const float position[3], const float look_at[3], const float up[3],
                           const float sensor_size_mm[2], float focal_length_mm, float fstop, pb2_camera* out) {
    if (!position || !look_at || !up || !sensor_size_mm || !out)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_camera_from_config: null argument");
    const float ul = std::sqrt(std::fmax(up[0] * up[0] + up[1] * up[1] + up[2] * up[2], 0.0f));
    for (int k = 0; k < 3; ++k) {
        out->position[k] = position[k];
        out->look_at[k] = look_at[k];
        out->up[k] = up[k] / ul;
    }
    out->sensor_size[0] = sensor_size_mm[0] * 1e-3f;
    out->sensor_size[1] = sensor_size_mm[1] * 1e-3f;
    out->focal_length = focal_length_mm * 1e-3f;
    out->aperture_radius = out->focal_length / (2.0f * fstop);
    return PB2_OK;
}

/* calcRenderRECT (Src/Interface/BuiltinComponent/Sensor.hpp:38-75) */
int pb2_calc_render_rect(uint32_t width, uint32_t height, float device_aspect, uint32_t fit_mode,
                         pb2_ndc_transform* tr, pb2_rect* rect) {
    if (!tr || !rect || width == 0 || height == 0 || !(device_aspect > 0.0f))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_calc_render_rect: invalid argument");
    const float iar = (float)width / (float)height;
    const float iiar = 1.0f / iar;
    const float idar = 1.0f / device_aspect;
    if (fit_mode == PB2_FIT_FILL) {
        *rect = { 0, 0, width, height };
        if (iar > device_aspect) *tr = { 0.0f, (idar - iiar) * 0.5f * device_aspect, 1.0f, iiar * device_aspect };
        else *tr = { (device_aspect - iar) * 0.5f * idar, 0.0f, iar * idar, 1.0f };
    } else {
        if (iar > device_aspect) {
            *tr = { -(iar - device_aspect) * 0.5f * idar, 0.0f, iar * idar, 1.0f };
            rect->left = (uint32_t)std::floor(std::fmax(0.0f, (float)width * (iar - device_aspect) * 0.5f * iiar));
            rect->top = 0;
            const uint32_t r = (uint32_t)std::ceil((float)width * (iar + device_aspect) * 0.5f * iiar);
            rect->width = (width < r ? width : r) - rect->left;
            rect->height = height;
        } else {
            *tr = { 0.0f, -(iiar - idar) * 0.5f * device_aspect, 1.0f, device_aspect * iiar };
            rect->left = 0;
            rect->top = (uint32_t)std::floor(std::fmax(0.0f, (float)height * (iiar - idar) * 0.5f * iar));
            rect->width = width;
            rect->height = (uint32_t)std::ceil((float)height * (iiar + idar) * 0.5f * iar) - rect->top;
        }
    }
    return PB2_OK;
}

const char* pb2_sobol_table_digest(void) { return pb2_sobol_table_sha256(); }

/* ---- acceleration structure ------------------------------------------------------------------ */

int pb2_accel_create(const pb2_scene* scene, void* stream_ptr, pb2_accel** out) {
    if (!scene || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_create: null argument");
    *out = nullptr;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    uint64_t n64 = 0;
    for (uint32_t m = 0; m < scene->mesh_count; ++m) {
        const pb2_mesh& mesh = scene->meshes[m];
        if (mesh.tri_count && (!mesh.vertices || !mesh.indices))
            return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_create: mesh without vertices or indices");
        if (mesh.material >= scene->material_count && scene->material_count)
            return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_create: mesh material out of range");
        for (uint64_t i = 0; i < 3ull * mesh.tri_count; ++i)
            if (mesh.indices[i] >= mesh.vert_count)
                return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_create: vertex index out of range");
        if (mesh.transform)
            for (int i = 0; i < 12; ++i)
                if (!std::isfinite(mesh.transform[i]))
                    return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_create: non-finite mesh transform");
        n64 += mesh.tri_count;
    }
    if (n64 >= 0x80000000ull) return fail(PB2_ERR_NOT_SUPPORTED, "pb2_accel_create: more than 2^31 triangles");
    for (uint32_t l = 0; l < scene->area_light_count; ++l) {
        const pb2_area_light& al = scene->area_lights[l];
        if ((uint64_t)al.first_plane + al.plane_count > scene->plane_count || al.plane_count == 0)
            return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_create: area light plane range out of bounds");
    }
    const uint32_t n = (uint32_t)n64;
    std::vector<TriSlot> host(n);
    std::vector<uint32_t> prim_mat(n ? n : 1, 0);
    uint32_t k = 0;
    for (uint32_t m = 0; m < scene->mesh_count; ++m) {
        const pb2_mesh& mesh = scene->meshes[m];
        for (uint32_t i = 0; i < mesh.tri_count; ++i, ++k) {
            float v[9];
            for (int j = 0; j < 3; ++j) {
                const uint32_t vi = mesh.indices[3 * i + j];
                pb2_mesh_vertex(mesh.transform, mesh.translation, mesh.vertices + 3 * vi, v + 3 * j);
            }
            uint32_t id = k;
            float w;
            std::memcpy(&w, &id, 4);
            host[k].v0 = make_float4(v[0], v[1], v[2], w);
            host[k].v1 = make_float4(v[3], v[4], v[5], 0.0f);
            host[k].v2 = make_float4(v[6], v[7], v[8], 0.0f);
            prim_mat[k] = mesh.material;
        }
    }
    std::vector<DevPlane> planes(scene->plane_count);
    for (uint32_t l = 0; l < scene->area_light_count; ++l) {
        const pb2_area_light& al = scene->area_lights[l];
        for (uint32_t i = 0; i < al.plane_count; ++i) {
            DevPlane& d = planes[al.first_plane + i];
            static_assert(sizeof(pb2_plane) == 64, "pb2_plane");
            std::memcpy(&d, &scene->planes[al.first_plane + i], sizeof(pb2_plane));
            for (int a = 0; a < 3; ++a) d.translation[a] = al.translation[a];
            d.light = l;
        }
    }
    auto* acc = new pb2_accel();
    auto cleanup = [&](int code) {
        pb2_accel_destroy(acc);
        return code;
    };
    cudaGetDevice(&acc->device);
    TriSlot* d_in = nullptr;
    void* scratch = nullptr;
    const size_t node_cap = n ? n : 1;
    cudaError_t e;
    if ((e = cudaMalloc(&acc->nodes, sizeof(WideNode) * node_cap))) return cleanup(cuda_fail(e, "cudaMalloc nodes"));
    if ((e = cudaMalloc(&acc->tris, sizeof(TriSlot) * (n ? n : 1)))) return cleanup(cuda_fail(e, "cudaMalloc tris"));
    if ((e = cudaMalloc(&acc->prim_material, sizeof(uint32_t) * (n ? n : 1))))
        return cleanup(cuda_fail(e, "cudaMalloc prim_material"));
    if ((e = cudaMalloc(&acc->planes, sizeof(DevPlane) * (planes.size() ? planes.size() : 1))))
        return cleanup(cuda_fail(e, "cudaMalloc planes"));
    if ((e = cudaMalloc(&acc->work, sizeof(uint32_t) * 8))) return cleanup(cuda_fail(e, "cudaMalloc work"));
    if ((e = cudaMalloc(&acc->counters, sizeof(unsigned long long) * 4)))
        return cleanup(cuda_fail(e, "cudaMalloc counters"));
    if ((e = cudaMalloc(&acc->error_flag, sizeof(uint32_t)))) return cleanup(cuda_fail(e, "cudaMalloc flag"));
    if ((e = cudaMemsetAsync(acc->error_flag, 0, sizeof(uint32_t), stream))) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMemsetAsync(acc->counters, 0, sizeof(unsigned long long) * 4, stream)))
        return cleanup(cuda_fail(e, "memset"));
    if (!planes.empty() && (e = cudaMemcpyAsync(acc->planes, planes.data(), sizeof(DevPlane) * planes.size(),
                                                cudaMemcpyHostToDevice, stream)))
        return cleanup(cuda_fail(e, "upload planes"));
    if ((e = cudaMemcpyAsync(acc->prim_material, prim_mat.data(), sizeof(uint32_t) * prim_mat.size(),
                             cudaMemcpyHostToDevice, stream)))
        return cleanup(cuda_fail(e, "upload materials"));
    BuildResult br{ 0, 0.0f };
    if (n) {
        const size_t sb = build_scratch_bytes(n);
        if ((e = cudaMalloc(&d_in, sizeof(TriSlot) * n))) return cleanup(cuda_fail(e, "cudaMalloc build input"));
        if ((e = cudaMalloc(&scratch, sb))) {
            cudaFree(d_in);
            return cleanup(cuda_fail(e, "cudaMalloc build scratch"));
        }
        e = cudaMemcpyAsync(d_in, host.data(), sizeof(TriSlot) * n, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = build_wide_bvh(d_in, n, acc->nodes, acc->tris, scratch, sb, stream, &br);
        cudaStreamSynchronize(stream);
        cudaFree(d_in);
        cudaFree(scratch);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "BVH build"));
    }
    if ((e = cudaStreamSynchronize(stream))) return cleanup(cuda_fail(e, "accel build sync"));
    acc->view.nodes = acc->nodes;
    acc->view.tris = acc->tris;
    acc->view.planes = acc->planes;
    acc->view.node_count = br.node_count;
    acc->view.tri_count = n;
    acc->view.plane_count = (uint32_t)planes.size();
    acc->view.root_is_leaf = n <= 1;
    acc->info.triangle_count = n;
    acc->info.node_count = br.node_count;
    acc->info.leaf_triangle_slots = n;
    acc->info.plane_count = (uint32_t)planes.size();
    acc->info.device_bytes = sizeof(WideNode) * node_cap + sizeof(TriSlot) * (uint64_t)(n ? n : 1) +
                             sizeof(uint32_t) * (uint64_t)(n ? n : 1) + sizeof(DevPlane) * planes.size();
    acc->info.build_ms = br.ms;
    *out = acc;
    return PB2_OK;
}

int pb2_accel_destroy(pb2_accel* acc) {
    if (!acc) return PB2_OK;
    cudaFree(acc->nodes);
    cudaFree(acc->tris);
    cudaFree(acc->planes);
    cudaFree(acc->prim_material);
    cudaFree(acc->work);
    cudaFree(acc->counters);
    cudaFree(acc->error_flag);
    cudaFree(acc->stage);
    for (cudaStream_t& st : acc->chunk_streams)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t& ev : acc->chunk_events)
        if (ev) cudaEventDestroy(ev);
    delete acc;
    return PB2_OK;
}

// Structural check of the built BVH on the host: every internal child index inside the node array and
// reached exactly once from the root, every leaf triangle range inside the triangle array and every
// triangle slot covered exactly once, every primitive id present once, and every triangle inside the
// dequantised box of the child slot that holds it.
int pb2_accel_validate(const pb2_accel* acc) {
    if (!acc) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_validate: null accel");
    const uint32_t nn = acc->view.node_count, nt = acc->view.tri_count;
    if (nt == 0) return PB2_OK;
    std::vector<WideNode> nodes(nn);
    std::vector<TriSlot> tris(nt);
    cudaError_t e;
    if ((e = cudaMemcpy(nodes.data(), acc->nodes, sizeof(WideNode) * nn, cudaMemcpyDeviceToHost)) ||
        (e = cudaMemcpy(tris.data(), acc->tris, sizeof(TriSlot) * nt, cudaMemcpyDeviceToHost)))
        return cuda_fail(e, "pb2_accel_validate: download");
    if (nn == 0) return fail(PB2_ERR_INVALID_ARGUMENT, "BVH has triangles but no nodes");
    std::vector<uint8_t> node_seen(nn, 0), slot_seen(nt, 0), prim_seen(nt, 0);
    std::vector<uint32_t> stack{ 0 };
    node_seen[0] = 1;
    auto bad = [&](uint32_t node, const std::string& what) {
        return fail(PB2_ERR_INVALID_ARGUMENT, "BVH node " + std::to_string(node) + ": " + what);
    };
    while (!stack.empty()) {
        const uint32_t ni = stack.back();
        stack.pop_back();
        const WideNode& w = nodes[ni];
        float p[3];
        std::memcpy(p, &w.w[0], 12);
        int ex[3];
        for (int a = 0; a < 3; ++a) {
            const uint32_t b = (w.w[0].w >> (8 * a)) & 0xFFu;
            if (b == 0 || b == 255) return bad(ni, "exponent byte out of range");
            ex[a] = (int)b - 127;
        }
        const uint32_t imask = w.w[0].w >> 24, child_base = w.w[1].x, tri_base = w.w[1].y;
        uint8_t meta[8], q[6][8];
        std::memcpy(meta, &w.w[1].z, 8);
        std::memcpy(q[0], &w.w[2].x, 8);  // lo x
        std::memcpy(q[1], &w.w[2].z, 8);  // lo y
        std::memcpy(q[2], &w.w[3].x, 8);  // lo z
        std::memcpy(q[3], &w.w[3].z, 8);  // hi x
        std::memcpy(q[4], &w.w[4].x, 8);  // hi y
        std::memcpy(q[5], &w.w[4].z, 8);  // hi z
        uint32_t rank = 0;
        for (int s = 0; s < 8; ++s) {
            const uint8_t m = meta[s];
            const bool internal = (imask >> s) & 1u;
            if (m == 0) {
                if (internal) return bad(ni, "empty slot marked internal");
                continue;
            }
            double lo[3], hi[3];
            for (int a = 0; a < 3; ++a) {
                lo[a] = (double)p[a] + std::ldexp((double)q[a][s], ex[a]);
                hi[a] = (double)p[a] + std::ldexp((double)q[3 + a][s], ex[a]);
                if (lo[a] > hi[a]) return bad(ni, "inverted child box");
            }
            if (internal) {
                if (m != ((1u << 5) | (24u + s))) return bad(ni, "internal slot meta mismatch");
                const uint64_t c = (uint64_t)child_base + rank++;
                if (c >= nn) return bad(ni, "child index " + std::to_string(c) + " >= node count");
                if (node_seen[c]++) return bad(ni, "child " + std::to_string(c) + " reached twice");
                stack.push_back((uint32_t)c);
            } else {
                const uint32_t unary = m >> 5, off = m & 0x1Fu;
                if (unary != 1u && unary != 3u && unary != 7u) return bad(ni, "leaf count not unary");
                const uint32_t cnt = unary == 1u ? 1u : unary == 3u ? 2u : 3u;
                for (uint32_t k = 0; k < cnt; ++k) {
                    const uint64_t sl = (uint64_t)tri_base + off + k;
                    if (sl >= nt) return bad(ni, "triangle slot " + std::to_string(sl) + " >= triangle count");
                    if (slot_seen[sl]++) return bad(ni, "triangle slot " + std::to_string(sl) + " in two leaves");
                    const TriSlot& t = tris[sl];
                    uint32_t prim;
                    std::memcpy(&prim, &t.v0.w, 4);
                    if (prim >= nt) return bad(ni, "primitive id out of range");
                    if (prim_seen[prim]++) return bad(ni, "primitive " + std::to_string(prim) + " twice");
                    const float* v[3] = { &t.v0.x, &t.v1.x, &t.v2.x };
                    for (int j = 0; j < 3; ++j)
                        for (int a = 0; a < 3; ++a)
                            if (!(v[j][a] >= lo[a] && v[j][a] <= hi[a]))
                                return bad(ni, "triangle outside its child box");
                }
            }
        }
    }
    for (uint32_t i = 0; i < nn; ++i)
        if (!node_seen[i]) return fail(PB2_ERR_INVALID_ARGUMENT, "BVH node " + std::to_string(i) + " unreachable");
    for (uint32_t i = 0; i < nt; ++i)
        if (!slot_seen[i]) return fail(PB2_ERR_INVALID_ARGUMENT, "triangle slot " + std::to_string(i) + " in no leaf");
    return PB2_OK;
}

int pb2_accel_get_info(const pb2_accel* acc, pb2_accel_info* info) {
    if (!acc || !info) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_get_info: null argument");
    *info = acc->info;
    return PB2_OK;
}

int pb2_accel_set_counting(pb2_accel* acc, int enable) {
    if (!acc) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_set_counting: null accel");
    acc->counting = enable != 0;
    return PB2_OK;
}

int pb2_accel_get_counters(const pb2_accel* acc, uint64_t* node_visits, uint64_t* tri_tests, void* stream_ptr) {
    if (!acc || !node_visits || !tri_tests) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_accel_get_counters: null");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    unsigned long long c[2];
    uint32_t flag = 0;
    PB2_CUDA(cudaMemcpyAsync(c, acc->counters, sizeof(c), cudaMemcpyDeviceToHost, stream), "read counters");
    PB2_CUDA(cudaMemcpyAsync(&flag, acc->error_flag, sizeof(flag), cudaMemcpyDeviceToHost, stream), "read flag");
    PB2_CUDA(cudaStreamSynchronize(stream), "sync");
    *node_visits = c[0];
    *tri_tests = c[1];
    if (flag) return fail(PB2_ERR_QUEUE_OVERFLOW, "traversal stack overflow in an earlier trace call");
    return PB2_OK;
}

static int trace_dev(const pb2_accel* acc, const pb2_ray* rays, uint32_t n, pb2_hit* hits, uint32_t* occ, bool closest,
                     cudaStream_t stream) {
    if (acc->counting) PB2_CUDA(cudaMemsetAsync(acc->counters, 0, sizeof(unsigned long long) * 2, stream), "memset");
    PB2_CUDA(launch_trace_api(acc->view, rays, n, hits, occ, closest, acc->counting, acc->work, acc->counters,
                              acc->error_flag, stream),
             closest ? "trace_closest launch" : "trace_any launch");
    return PB2_OK;
}

int pb2_trace_closest(const pb2_accel* acc, const pb2_ray* rays, uint32_t n, pb2_hit* hits, void* stream) {
    if (!acc || (n && (!rays || !hits))) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_trace_closest: null argument");
    return trace_dev(acc, rays, n, hits, nullptr, true, static_cast<cudaStream_t>(stream));
}

int pb2_trace_any(const pb2_accel* acc, const pb2_ray* rays, uint32_t n, uint32_t* occluded, void* stream) {
    if (!acc || (n && (!rays || !occluded))) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_trace_any: null argument");
    return trace_dev(acc, rays, n, nullptr, occluded, false, static_cast<cudaStream_t>(stream));
}

static int ensure_stage(pb2_accel* acc, size_t bytes) {
    if (acc->stage_bytes >= bytes) return PB2_OK;
    cudaFree(acc->stage);
    acc->stage = nullptr;
    acc->stage_bytes = 0;
    PB2_CUDA(cudaMalloc(&acc->stage, bytes), "cudaMalloc staging");
    acc->stage_bytes = bytes;
    return PB2_OK;
}

static int ensure_chunk_streams(pb2_accel* acc) {
    for (cudaStream_t& st : acc->chunk_streams)
        if (!st) PB2_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "create chunk stream");
    for (cudaEvent_t& ev : acc->chunk_events)
        if (!ev) PB2_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "create chunk event");
    return PB2_OK;
}

// Host-array trace: the batch is split into chunks of kHostChunk rays (a quarter and a half chunk at either end),
// dealt round-robin to three streams; each chunk's upload, traversal and download are ordered on its stream, so
// one chunk's copies run on the copy engines while another chunk traverses.  Measured on the stress test's step
// (4M closest-hit + 4M any-hit rays from pinned host memory): uniform 2^19-ray chunks 8.51 ms, ramped 2^19 /
// 2^20 / 2^18 chunks 8.37 / 8.35 / 9.03 ms.  Each stream has its own work counter (accel->work
// slots 4..6; slots 0..2 belong to the render pipeline).  The caller's stream orders the whole call.
#ifndef PB2_HOST_CHUNK_LOG2
#define PB2_HOST_CHUNK_LOG2 20
#endif
static constexpr uint32_t kHostChunk = 1u << PB2_HOST_CHUNK_LOG2;

static int trace_host(const pb2_accel* cacc, const pb2_ray* rays, uint32_t n, void* out, bool closest,
                      cudaStream_t stream) {
    auto* acc = const_cast<pb2_accel*>(cacc);
    const size_t osz = closest ? sizeof(pb2_hit) : sizeof(uint32_t);
    const size_t rb = sizeof(pb2_ray) * (size_t)n;
    const size_t ob = osz * (size_t)n;
    int rc = ensure_stage(acc, rb + ob + 256);
    if (rc) return rc;
    auto* d_rays = static_cast<pb2_ray*>(acc->stage);
    char* d_out = static_cast<char*>(acc->stage) + ((rb + 255) / 256) * 256;
    if (n <= kHostChunk) {
        PB2_CUDA(cudaMemcpyAsync(d_rays, rays, rb, cudaMemcpyHostToDevice, stream), "upload rays");
        rc = trace_dev(acc, d_rays, n, closest ? reinterpret_cast<pb2_hit*>(d_out) : nullptr,
                       closest ? nullptr : reinterpret_cast<uint32_t*>(d_out), closest, stream);
        if (rc) return rc;
        PB2_CUDA(cudaMemcpyAsync(out, d_out, ob, cudaMemcpyDeviceToHost, stream), "download results");
        PB2_CUDA(cudaStreamSynchronize(stream), "trace sync");
        return PB2_OK;
    }
    if ((rc = ensure_chunk_streams(acc))) return rc;
    if (acc->counting) PB2_CUDA(cudaMemsetAsync(acc->counters, 0, sizeof(unsigned long long) * 2, stream), "memset");
    PB2_CUDA(cudaEventRecord(acc->chunk_events[0], stream), "record start");
    for (cudaStream_t st : acc->chunk_streams) PB2_CUDA(cudaStreamWaitEvent(st, acc->chunk_events[0], 0), "wait start");
    // chunk boundaries: kHostChunk rays each, with a quarter and a half chunk first and last (batches of two chunks
    // or more), so that the first traversal starts after a short upload and the last download is short
    std::vector<size_t> bounds{ 0 };
    {
        const size_t q = kHostChunk / 4, h = kHostChunk / 2;
        const bool ramp = n >= 2 * (size_t)kHostChunk;
        if (ramp) { bounds.push_back(q); bounds.push_back(q + h); }
        const size_t body_end = ramp ? n - (q + h) : n;
        while (bounds.back() < body_end) bounds.push_back(std::min(body_end, bounds.back() + kHostChunk));
        if (ramp) { bounds.push_back(n - q); bounds.push_back(n); }
    }
    const uint32_t chunks = (uint32_t)bounds.size() - 1;
    for (uint32_t c = 0; c < chunks; ++c) {
        const int k = (int)(c % 3);
        cudaStream_t st = acc->chunk_streams[k];
        const size_t lo = bounds[c];
        const uint32_t m = (uint32_t)(bounds[c + 1] - lo);
        PB2_CUDA(cudaMemcpyAsync(d_rays + lo, rays + lo, sizeof(pb2_ray) * m, cudaMemcpyHostToDevice, st),
                 "upload rays");
        PB2_CUDA(launch_trace_api(acc->view, d_rays + lo, m,
                                  closest ? reinterpret_cast<pb2_hit*>(d_out) + lo : nullptr,
                                  closest ? nullptr : reinterpret_cast<uint32_t*>(d_out) + lo, closest, acc->counting,
                                  acc->work + 4 + k, acc->counters, acc->error_flag, st),
                 closest ? "trace_closest launch" : "trace_any launch");
        PB2_CUDA(cudaMemcpyAsync(static_cast<char*>(out) + lo * osz, d_out + lo * osz, osz * m, cudaMemcpyDeviceToHost,
                                 st),
                 "download results");
    }
    for (int k = 0; k < 3; ++k) {
        PB2_CUDA(cudaEventRecord(acc->chunk_events[1 + k], acc->chunk_streams[k]), "record chunk");
        PB2_CUDA(cudaStreamWaitEvent(stream, acc->chunk_events[1 + k], 0), "join chunk");
    }
    PB2_CUDA(cudaStreamSynchronize(stream), "trace sync");
    return PB2_OK;
}

int pb2_trace_closest_host(const pb2_accel* acc, const pb2_ray* rays, uint32_t n, pb2_hit* hits, void* stream) {
    if (!acc || (n && (!rays || !hits))) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_trace_closest_host: null");
    return trace_host(acc, rays, n, hits, true, static_cast<cudaStream_t>(stream));
}

int pb2_trace_any_host(const pb2_accel* acc, const pb2_ray* rays, uint32_t n, uint32_t* occluded, void* stream) {
    if (!acc || (n && (!rays || !occluded))) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_trace_any_host: null");
    return trace_host(acc, rays, n, occluded, false, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
