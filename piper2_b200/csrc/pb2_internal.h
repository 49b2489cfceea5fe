// pb2_internal.h -- declarations shared between the library's translation units (not installed).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "../../include/piper2_b200.h"
#include "pb2_bvh.h"
#include "pb2_math.h"

namespace pb2 {

// thread-local last error (pb2_last_error)
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what);

// Per-device launch set-up.  Function attributes and occupancy belong to a device, so a process that
// drives several devices (pb2_set_device) keeps one cache entry per device index.
constexpr int kMaxDevices = 64;
// The calling thread's current device, or -1 if it cannot be read or is >= kMaxDevices.
int current_device();
// Sets a kernel's dynamic shared-memory limit on the current device, once per device.
cudaError_t smem_attr_once(const void* kernel, size_t bytes, std::atomic<int> (&done)[kMaxDevices]);
// Resident blocks per SM x SMs of a kernel on the current device (at least the SM count), cached per
// device in `cache`.
int resident_grid_cached(const void* kernel, int threads, size_t smem, std::atomic<int> (&cache)[kMaxDevices]);

// The guiding network's inference weights (guiding.cu): the padded bf16 weight image and fp32 biases.
struct GuideView {
    const __nv_bfloat16* w16;
    const float* b32;
};
cudaError_t guide_forward(const GuideView& gv, const float* features, uint32_t n, float* out, cudaStream_t stream);
// Batch loss gradient (added to grad) and loss; `workspace` holds guide_workspace_bytes() of staging.
cudaError_t guide_gradient_mma(const GuideView& gv, const float* records, uint32_t n, float* grad, float* scalars,
                               void* workspace, cudaStream_t stream);
// The same gradient on the tcgen05 tensor cores (guiding_train_tc.cu): one fused kernel per batch, each CTA's
// partial gradient in `workspace`, then a reduction; error[0] is set if a tensor-core wait timed out.
cudaError_t guide_gradient_tc(const GuideView& gv, const float* records, uint32_t n, float* grad, float* scalars,
                              void* workspace, uint32_t* error, cudaStream_t stream);
size_t guide_workspace_bytes();
// The same forward pass on the tcgen05 tensor cores (guiding_tc.cu); error[0] is set if a tensor-core
// wait timed out.
cudaError_t guide_forward_tc(const GuideView& gv, const float* features, uint32_t n, float* out, uint32_t* error,
                             cudaStream_t stream);

cudaError_t launch_trace_api(const BvhView& bvh, const pb2_ray* rays, uint32_t n, pb2_hit* hits, uint32_t* occluded,
                             bool closest, bool count, uint32_t* work, unsigned long long* counters,
                             uint32_t* error_flag, cudaStream_t stream);

}  // namespace pb2

struct pb2_accel {
    int device = 0;
    pb2::WideNode* nodes = nullptr;
    pb2::TriSlot* tris = nullptr;
    pb2::DevPlane* planes = nullptr;
    uint32_t* prim_material = nullptr;  // material of each global primitive
    uint32_t* work = nullptr;           // work counters of the trace kernels
    unsigned long long* counters = nullptr;
    uint32_t* error_flag = nullptr;
    bool counting = false;
    pb2::BvhView view{};
    pb2_accel_info info{};
    // staging buffers of the *_host trace calls
    void* stage = nullptr;
    size_t stage_bytes = 0;
    // streams and events of the pipelined *_host trace calls (upload, trace and download of successive
    // chunks overlap); created on first use
    cudaStream_t chunk_streams[3] = { nullptr, nullptr, nullptr };
    cudaEvent_t chunk_events[4] = { nullptr, nullptr, nullptr, nullptr };
};

struct pb2_guide {
    float* params = nullptr;  // fp32 master parameters, flat layout (per layer: W[out][in], then b[out])
    float* m = nullptr;       // Adam moments
    float* v = nullptr;
    float* grad = nullptr;
    __nv_bfloat16* w16 = nullptr;  // padded bf16 weight image used by the tensor-core tiles
    float* b32 = nullptr;
    float* scalars = nullptr;  // [0] weight sum of the batch, [1] loss
    void* workspace = nullptr; // gradient staging (guide_workspace_bytes)
    uint32_t step = 0;
    pb2_gradient_hook hook = nullptr;  // between each step's gradient and its Adam update
    void* hook_user = nullptr;
    pb2::GuideView view() const { return pb2::GuideView{ w16, b32 }; }
};
