// pb2_bvh.h -- layout of the 8-wide quantised BVH in device memory, shared by the builder, the
// traversal kernels and the host code.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pb2 {

// One 8-wide node, 80 bytes (five 16-byte words), in the compressed-wide-BVH layout of Ylitie,
// Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs"
// (HPG 2017):
//   w0: origin p (3 floats) | exponent bytes ex, ey, ez (biased +127) | imask (internal-child slots)
//   w1: child_base | tri_base | meta[0..3] | meta[4..7]
//   w2: qlo_x[0..7] | qlo_y[0..7]
//   w3: qlo_z[0..7] | qhi_x[0..7]
//   w4: qhi_y[0..7] | qhi_z[0..7]
// Child box of slot s on axis a: [p_a + qlo_a[s] * 2^e_a, p_a + qhi_a[s] * 2^e_a], rounded outward.
// meta[s] = 0 for an empty slot; (1 << 5) | (24 + s) for an internal child (node
// child_base + popcount(imask below s)); (unary(count) << 5) | offset for a leaf of 1..3
// triangles at tri_base + offset.  Slot s holds the child nearest for rays in octant s.
struct WideNode {
    uint4 w[5];
};
static_assert(sizeof(WideNode) == 80, "WideNode layout");

// Triangle slot in leaf order: three float4, xyz = vertex, w of the first = global primitive id.
struct TriSlot {
    float4 v0, v1, v2;
};
static_assert(sizeof(TriSlot) == 48, "TriSlot layout");

// Area-light plane on the device: PerPlaneData + the light's translation and index.
struct DevPlane {
    float origin[3];
    float u[3];
    float v[3];
    float normal[3];
    float tangent[3];
    uint32_t max_det_comp;
    float translation[3];
    uint32_t light;
};

struct BvhView {
    const WideNode* nodes;
    const TriSlot* tris;
    const DevPlane* planes;
    uint32_t node_count;
    uint32_t tri_count;
    uint32_t plane_count;
    uint32_t root_is_leaf;  // scene with a single triangle or none
};

// Device-side build: `tris_in` holds the flattened scene triangles (world space) in primitive order.
// Fills nodes/tris_out (capacity: max(1, n) nodes, n triangle slots).  Returns a cudaError_t.
struct BuildResult {
    uint32_t node_count;
    float ms;
};
cudaError_t build_wide_bvh(const TriSlot* tris_in, uint32_t n, WideNode* nodes, TriSlot* tris_out, void* scratch,
                           size_t scratch_bytes, cudaStream_t stream, BuildResult* result);
size_t build_scratch_bytes(uint32_t n);
// The same build without CUDA events, into caller-supplied buffers only; writes the node count.
cudaError_t build_wide_bvh_prealloc(const TriSlot* tris_in, uint32_t n, WideNode* nodes, TriSlot* tris_out,
                                    void* scratch, size_t scratch_bytes, cudaStream_t stream, uint32_t* node_count_out);

}  // namespace pb2
