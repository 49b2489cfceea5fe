// generic_kernels.cu -- kernels the accelerator tests launch through pb2_acc_launch_kernel (test infrastructure,
// built by tests/kernels/build_kernels.py into tests/kernels/_build/libpb2_test_kernels.so).
//
// They are written the way a user of the accelerator writes one: a __device__ body over a pb2_task_context using
// the device runtime of include/piper2_b200_device.cuh, an entry declared with PB2_KERNEL_ENTRY, and its
// CUfunction handed to pb2_acc_register_kernel (pb2t_kernel_function below looks it up).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "../../include/piper2_b200_device.cuh"

// The reference's Accelerator test kernel (Src/Test/conv.cpp:22-42 over conv.hpp:22-37): arguments width,
// height, kernelSize; resources X, Y (buffers) and Z (tiled output); one task per pixel, x = row, z = column.
__device__ void conv_body(pb2_task_context ctx) {
    pb2_dim3 idx;
    uint32_t width, height, kernel_size;
    pb2_get_task_index(ctx, idx);
    pb2_get_argument(ctx, 0, &width);
    pb2_get_argument(ctx, 1, &height);
    pb2_get_argument(ctx, 2, &kernel_size);
    uint64_t lut, hx, hy, hz;
    pb2_get_root_resource_lut(ctx, lut);
    pb2_look_up_resource_handle(ctx, lut, 0, hx);
    pb2_look_up_resource_handle(ctx, lut, 1, hy);
    pb2_look_up_resource_handle(ctx, lut, 2, hz);
    const float* X = reinterpret_cast<const float*>(hx);
    const float* Y = reinterpret_cast<const float*>(hy);
    float* Z = reinterpret_cast<float*>(hz);
    const uint32_t i0 = idx.x * width + idx.z;
    const uint32_t half = kernel_size / 2;
    const uint32_t py = i0 / width, px = i0 % width;
    float res = 0.0f;
    for (int32_t i = 0; i < (int32_t)kernel_size; ++i) {
        const int32_t nx = (int32_t)(px + (uint32_t)i - half);
        if (nx >= 0 && nx < (int32_t)width)
            for (int32_t j = 0; j < (int32_t)kernel_size; ++j) {
                const int32_t ny = (int32_t)(py + (uint32_t)j - half);
                if (ny >= 0 && ny < (int32_t)height)
                    res = __fadd_rn(res, __fmul_rn(X[ny * (int32_t)width + nx], Y[i * (int32_t)kernel_size + j]));
            }
    }
    Z[i0] = res;
}
PB2_KERNEL_ENTRY(convEntry, conv_body)

struct Bytes3 {
    unsigned char b[3];
};

// Reads every argument kind and a three-level table.  Arguments: nx, ny, nz (uint32), magic (uint64), f
// (float), three bytes.  Root table: [T (tiled, uint32 per task), H (tiled, uint64 x 16), N1, B0]; N1: [B1, N2];
// N2: [B2].  Every task writes T[task] = B0[task] + B1[0] + B2[0]; task (0, 0, 0) also records in H what it
// looked up.
__device__ void echo_body(pb2_task_context ctx) {
    pb2_dim3 idx;
    pb2_get_task_index(ctx, idx);
    uint32_t nx, ny, nz;
    uint64_t magic;
    float f;
    Bytes3 b3;
    pb2_get_argument(ctx, 0, &nx);
    pb2_get_argument(ctx, 1, &ny);
    pb2_get_argument(ctx, 2, &nz);
    pb2_get_argument(ctx, 3, &magic);
    pb2_get_argument(ctx, 4, &f);
    pb2_get_argument(ctx, 5, &b3);
    uint64_t root, t, h, n1, b0, b1, n2, b2;
    pb2_get_root_resource_lut(ctx, root);
    pb2_look_up_resource_handle(ctx, root, 0, t);
    pb2_look_up_resource_handle(ctx, root, 1, h);
    pb2_look_up_resource_handle(ctx, root, 2, n1);
    pb2_look_up_resource_handle(ctx, root, 3, b0);
    pb2_look_up_resource_handle(ctx, n1, 0, b1);
    pb2_look_up_resource_handle(ctx, n1, 1, n2);
    pb2_look_up_resource_handle(ctx, n2, 0, b2);
    const uint32_t task = (idx.x * ny + idx.y) * nz + idx.z;
    reinterpret_cast<uint32_t*>(t)[task] = reinterpret_cast<const uint32_t*>(b0)[task] +
                                           reinterpret_cast<const uint32_t*>(b1)[0] +
                                           reinterpret_cast<const uint32_t*>(b2)[0];
    if (task == 0) {
        uint64_t* H = reinterpret_cast<uint64_t*>(h);
        H[0] = t;
        H[1] = h;
        H[2] = n1;
        H[3] = b0;
        H[4] = b1;
        H[5] = n2;
        H[6] = b2;
        H[7] = magic;
        H[8] = __float_as_uint(f);
        H[9] = (uint64_t)b3.b[0] | ((uint64_t)b3.b[1] << 8) | ((uint64_t)b3.b[2] << 16);
        H[10] = ((uint64_t)nx << 40) | ((uint64_t)ny << 20) | nz;
        H[11] = gridDim.z;
        H[12] = blockDim.x;
    }
}
PB2_KERNEL_ENTRY(echoEntry, echo_body)

extern "C" int pb2t_kernel_function(const char* name, void** cu_function) {
    const void* sym = nullptr;
    if (strcmp(name, "convEntry") == 0) sym = (const void*)convEntry;
    else if (strcmp(name, "echoEntry") == 0) sym = (const void*)echoEntry;
    else return 1;
    cudaFunction_t f = nullptr;
    if (cudaGetFuncBySymbol(&f, sym) != cudaSuccess) return 2;
    *cu_function = (void*)f;
    return 0;
}
