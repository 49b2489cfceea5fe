/*
 * piper2_b200_device.cuh -- device-side runtime of the generic kernels launched through pb2_acc_launch_kernel.
 *
 * The reference's accelerators hand every kernel a TaskContext and four runtime calls
 * (Src/Kernel/DeviceRuntime.hpp): piperGetTaskIndex, piperGetArgument, piperGetRootResourceLUT and
 * piperLookUpResourceHandle, implemented for CUDA in Src/Infrastructure/Accelerator/CUDA/Kernel.cpp:36-63
 * over the launch buffer that CUDAAccelerator::launchKernelImpl writes (CUDA.cpp:826-850), and an entry
 * `cudaEntry(maxZ, context)` that runs the kernel for z indices below maxZ (CUDA.cpp:391-414).
 *
 * A generic kernel here is ordinary CUDA C++ compiled by nvcc for sm_100a against this header (the reference
 * JIT-links LLVM IR instead).  Write the body as a __device__ function of a pb2_task_context and declare the
 * entry with PB2_KERNEL_ENTRY; register its CUfunction with pb2_acc_register_kernel.
 *
 * Launch buffer (bytes, 128-byte aligned):
 *   [0]  uint32 offset of the argument table      = 8 + 8 * handle count
 *   [4]  uint32 offset of the argument data       = the above + 8 * argument count
 *   [8]  uint64 resource handles of the flattened lookup tables (root table first)
 *   ...  (uint32 offset, uint32 size) per argument, offsets relative to the argument data
 *   ...  argument bytes
 * The launch grid is (dim.x, dim.y, ceil(dim.z / block)) with block = min(dim.z, the device's thread limit).
 */
#ifndef PIPER2_B200_DEVICE_CUH
#define PIPER2_B200_DEVICE_CUH

#include <stdint.h>

typedef const unsigned char* pb2_task_context;

struct pb2_dim3 {
    uint32_t x, y, z;
};

/* piperGetTaskIndex (CUDA/Kernel.cpp:36-40): x, y = blockIdx.x, .y; z = blockIdx.z * blockDim.x + threadIdx.x. */
__device__ __forceinline__ void pb2_get_task_index(pb2_task_context, pb2_dim3& index) {
    index.x = blockIdx.x;
    index.y = blockIdx.y;
    index.z = blockIdx.z * blockDim.x + threadIdx.x;
}

/* piperGetArgument (CUDA/Kernel.cpp:47-53): copies argument `index` (its packed size) to `ptr`. */
__device__ __forceinline__ void pb2_get_argument(pb2_task_context ctx, uint32_t index, void* ptr) {
    const uint32_t table = reinterpret_cast<const uint32_t*>(ctx)[0];
    const uint32_t data = reinterpret_cast<const uint32_t*>(ctx)[1];
    const uint32_t* desc = reinterpret_cast<const uint32_t*>(ctx + table) + 2 * index;
    const unsigned char* src = ctx + data + desc[0];
    unsigned char* dst = static_cast<unsigned char*>(ptr);
    for (uint32_t i = 0; i < desc[1]; ++i) dst[i] = src[i];
}

/* piperGetRootResourceLUT (CUDA/Kernel.cpp:54-56): the root table starts at handle 0. */
__device__ __forceinline__ void pb2_get_root_resource_lut(pb2_task_context, uint64_t& handle) { handle = 0; }

/* piperLookUpResourceHandle (CUDA/Kernel.cpp:57-62): entry `index` of the table that starts at `lut`: a device
 * address for a buffer or tiled output, the start of the nested table for a lookup table. */
__device__ __forceinline__ void pb2_look_up_resource_handle(pb2_task_context ctx, uint64_t lut, uint32_t index,
                                                            uint64_t& handle) {
    handle = reinterpret_cast<const uint64_t*>(ctx + 8)[lut + index];
}

/* The entry of a generic kernel (cudaEntry, CUDA.cpp:391-414): runs BODY(ctx) for z indices below max_z. */
#define PB2_KERNEL_ENTRY(NAME, BODY)                                                          \
    extern "C" __global__ void NAME(uint32_t max_z, pb2_task_context ctx) {                    \
        if (blockIdx.z * blockDim.x + threadIdx.x < max_z) BODY(ctx);                          \
    }

#endif /* PIPER2_B200_DEVICE_CUH */
