// bvh_build.cu -- device-side build of the 8-wide quantised BVH.
//
//   1. per-triangle bounds and the centroid bounds of the scene,
//   2. 63-bit Morton codes of the centroids (21 bits per axis),
//   3. radix sort of (code, primitive) pairs,
//   4. binary radix tree over the sorted codes (Karras, "Maximizing Parallelism in the Construction of
//      BVHs, Octrees, and k-d Trees", HPG 2012), equal codes ordered by index,
//   5. bottom-up box refit (the second child to arrive at a node computes its box),
//   6. SAH costs of the collapse, bottom-up over the binary tree (Ylitie, Karras, Laine, "Efficient
//      Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017, Sec. 4.1): for every
//      binary node n and i = 1..8, C(n, i) = the least SAH cost of representing n's subtree with at most
//      i children of the enclosing wide node, where one child is either a leaf of <= 3 triangles
//      (cost kCostTri x triangles x area) or a wide node (kCostNode x area + the best distribution of 8
//      children below it); distributions split i between n's two binary children,
//   7. top-down collapse into 8-wide nodes, one frontier level per launch, each wide node taking the
//      children of its optimal distribution; child boxes are quantised to 8 bits relative to the node
//      box (rounded outward) and children are placed in the slot of the ray octant they are nearest for
//      (greedy assignment on the projected centroid offsets).
#include <cub/device/device_radix_sort.cuh>

#include <cfloat>
#include <cmath>

#include "pb2_bvh.h"

namespace pb2 {
namespace {

constexpr int kLeafMax = 3;
// SAH weights of the collapse, per unit of surface area: a wide node against a leaf triangle.  Measured on a
// B200 (1M-triangle soup, closest hit): 0.15 -> 783, 0.3 -> 883, 0.8 -> 964, 1.2 -> 1017, 2.0 -> 1021,
// 3.0 -> 1020 Mrays/s; a triangle weighted above a node makes the collapse favour small leaves, which the
// traversal's per-triangle divergence rewards more than the box count predicts.
#ifndef PB2_SAH_COST_TRI
#define PB2_SAH_COST_TRI 2.0f
#endif
constexpr float kCostNode = 1.0f;
constexpr float kCostTri = PB2_SAH_COST_TRI;

__device__ __forceinline__ int f2key(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float key2f(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

// bounds[0..2] = min keys, bounds[3..5] = max keys of the centroids
__global__ void k_tri_bounds(const TriSlot* __restrict__ tris, uint32_t n, float4* __restrict__ lo,
                             float4* __restrict__ hi, int* __restrict__ cbounds) {
    __shared__ int smin[3], smax[3];
    if (threadIdx.x < 3) { smin[threadIdx.x] = INT_MAX; smax[threadIdx.x] = INT_MIN; }
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const TriSlot t = tris[i];
        const float3 l = make_float3(fminf(t.v0.x, fminf(t.v1.x, t.v2.x)), fminf(t.v0.y, fminf(t.v1.y, t.v2.y)),
                                     fminf(t.v0.z, fminf(t.v1.z, t.v2.z)));
        const float3 h = make_float3(fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x)), fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y)),
                                     fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z)));
        lo[i] = make_float4(l.x, l.y, l.z, 0.0f);
        hi[i] = make_float4(h.x, h.y, h.z, 0.0f);
        const float c[3] = { 0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z) };
        for (int a = 0; a < 3; ++a) {
            atomicMin(&smin[a], f2key(c[a]));
            atomicMax(&smax[a], f2key(c[a]));
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&cbounds[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&cbounds[3 + threadIdx.x], smax[threadIdx.x]);
    }
}

__device__ __forceinline__ uint64_t expand21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                         const int* __restrict__ cbounds, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 l = lo[i], h = hi[i];
    const float c[3] = { 0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z) };
    uint64_t code = 0;
    for (int a = 0; a < 3; ++a) {
        const float mn = key2f(cbounds[a]), mx = key2f(cbounds[3 + a]);
        const float ext = mx - mn;
        float u = ext > 0.0f ? (c[a] - mn) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        const uint32_t q = min((uint32_t)(u * 2097152.0f), 2097151u);
        code |= expand21(q) << (2 - a);
    }
    keys[i] = code;
    vals[i] = i;
}

// Child references: >= 0 internal node, < 0 leaf (sorted position ~ref).
__device__ __forceinline__ int leaf_ref(int i) { return ~i; }
__device__ __forceinline__ bool is_leaf(int r) { return r < 0; }

__device__ __forceinline__ int delta(const uint64_t* keys, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz((uint32_t)(i ^ j));
    return __clzll(a ^ b);
}

struct Internal {
    int left, right;
    uint32_t first, last;
};

__global__ void k_karras(const uint64_t* __restrict__ keys, uint32_t n, Internal* __restrict__ nodes,
                         int* __restrict__ iparent, int* __restrict__ lparent) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)n - 1) return;
    const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int64_t lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t gamma = i + s * d + (d < 0 ? d : 0);
    const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    Internal nd;
    nd.left = (lo == gamma) ? leaf_ref((int)gamma) : (int)gamma;
    nd.right = (hi == gamma + 1) ? leaf_ref((int)(gamma + 1)) : (int)(gamma + 1);
    nd.first = (uint32_t)lo;
    nd.last = (uint32_t)hi;
    nodes[i] = nd;
    if (is_leaf(nd.left)) lparent[~nd.left] = (int)i; else iparent[nd.left] = (int)i;
    if (is_leaf(nd.right)) lparent[~nd.right] = (int)i; else iparent[nd.right] = (int)i;
    if (i == 0) iparent[0] = -1;
}

// Sorted leaf boxes: slo/shi[k] = box of triangle vals[k].
__global__ void k_gather_leaves(const uint32_t* __restrict__ vals, const float4* __restrict__ lo,
                                const float4* __restrict__ hi, uint32_t n, float4* __restrict__ slo,
                                float4* __restrict__ shi) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t t = vals[k];
    slo[k] = lo[t];
    shi[k] = hi[t];
}

__device__ __forceinline__ void child_box(int r, const float4* slo, const float4* shi, const float4* ilo,
                                          const float4* ihi, float4& l, float4& h) {
    if (is_leaf(r)) {
        l = __ldcg(&slo[~r]);
        h = __ldcg(&shi[~r]);
    } else {
        l = __ldcg(&ilo[r]);
        h = __ldcg(&ihi[r]);
    }
}

__global__ void k_refit(const Internal* __restrict__ nodes, const int* __restrict__ iparent,
                        const int* __restrict__ lparent, const float4* __restrict__ slo, const float4* __restrict__ shi,
                        float4* ilo, float4* ihi, uint32_t* flags, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int node = lparent[k];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0) return;
        __threadfence();
        const Internal nd = nodes[node];
        float4 al, ah, bl, bh;
        child_box(nd.left, slo, shi, ilo, ihi, al, ah);
        child_box(nd.right, slo, shi, ilo, ihi, bl, bh);
        const float4 l = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
        const float4 h = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
        __stcg(&ilo[node], l);
        __stcg(&ihi[node], h);
        node = iparent[node];
    }
}

__device__ __forceinline__ float box_area(float4 l, float4 h) {
    const float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
    return dx * dy + dy * dz + dz * dx;
}

// SAH collapse costs (step 6).  cost[8 n + i - 1] = C(n, i); split[8 n + i - 1] = how many of i children go
// to the left binary child in the best distribution D(n, i) (i >= 2); dist[n] bit i set when D(n, i) beats a
// single child for C(n, i); leafy[n] = 1 when that single child is a leaf (possible for <= 3 triangles).
// Bottom-up like the refit.
__global__ void k_sah_costs(const Internal* __restrict__ nodes, const int* __restrict__ iparent,
                            const int* __restrict__ lparent, const float4* __restrict__ slo, const float4* __restrict__ shi,
                            const float4* __restrict__ ilo, const float4* __restrict__ ihi, uint32_t* flags, float* cost,
                            uint8_t* split, uint8_t* dist, uint8_t* leafy, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int node = lparent[k];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0) return;
        __threadfence();
        const Internal nd = nodes[node];
        float cl[8], cr[8];
        if (is_leaf(nd.left)) {
            const float c = kCostTri * box_area(slo[~nd.left], shi[~nd.left]);
            for (int i = 0; i < 8; ++i) cl[i] = c;
        } else {
            for (int i = 0; i < 8; ++i) cl[i] = __ldcg(&cost[8 * (size_t)nd.left + i]);
        }
        if (is_leaf(nd.right)) {
            const float c = kCostTri * box_area(slo[~nd.right], shi[~nd.right]);
            for (int i = 0; i < 8; ++i) cr[i] = c;
        } else {
            for (int i = 0; i < 8; ++i) cr[i] = __ldcg(&cost[8 * (size_t)nd.right + i]);
        }
        float d[9];
        uint8_t sp[9];
        for (int i = 2; i <= 8; ++i) {
            float best = FLT_MAX;
            int arg = 1;
            for (int j = 1; j < i; ++j) {
                const float c = cl[j - 1] + cr[i - j - 1];
                if (c < best) { best = c; arg = j; }
            }
            d[i] = best;
            sp[i] = (uint8_t)arg;
        }
        const float area = box_area(__ldcg(&ilo[node]), __ldcg(&ihi[node]));
        const uint32_t tris = nd.last - nd.first + 1;
        const float c_wide = kCostNode * area + d[8];
        const float c_leaf = tris <= (uint32_t)kLeafMax ? kCostTri * (float)tris * area : FLT_MAX;
        const bool leaf = c_leaf <= c_wide;
        const float c1 = leaf ? c_leaf : c_wide;
        uint8_t dm = 0;
        __stcg(&cost[8 * (size_t)node], c1);
        for (int i = 2; i <= 8; ++i) {
            const bool use = d[i] < c1;
            if (use) dm |= (uint8_t)(1u << i);
            __stcg(&cost[8 * (size_t)node + i - 1], use ? d[i] : c1);
            split[8 * (size_t)node + i - 1] = sp[i];
        }
        dist[node] = dm;
        leafy[node] = leaf ? 1 : 0;
        node = iparent[node];
    }
}

struct Frontier {
    int ref;
    uint32_t wide;
};

__device__ __forceinline__ uint32_t ref_count(int r, const Internal* nodes) {
    if (is_leaf(r)) return 1;
    const Internal nd = nodes[r];
    return nd.last - nd.first + 1;
}
__device__ __forceinline__ uint32_t ref_first(int r, const Internal* nodes) {
    return is_leaf(r) ? (uint32_t)(~r) : nodes[r].first;
}

__device__ int exponent_for(double ext) {
    if (!(ext > 0.0)) return -126;
    int e = (int)ceil(log2(ext / 255.0));
    if (e < -126) e = -126;
    while (e < 127 && ldexp(255.0, e) < ext) ++e;
    while (e > -126 && ldexp(255.0, e - 1) >= ext) --e;
    return e;
}

__global__ void k_collapse(const Frontier* __restrict__ in, uint32_t count, Frontier* __restrict__ out,
                           uint32_t* out_count, uint32_t* node_counter, uint32_t* tri_counter,
                           const Internal* __restrict__ nodes, const float4* __restrict__ slo,
                           const float4* __restrict__ shi, const float4* __restrict__ ilo,
                           const float4* __restrict__ ihi, const uint32_t* __restrict__ vals,
                           const TriSlot* __restrict__ tris_in, WideNode* __restrict__ wnodes,
                           TriSlot* __restrict__ tris_out, const uint8_t* __restrict__ split,
                           const uint8_t* __restrict__ dist, const uint8_t* __restrict__ leafy) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int ref = in[i].ref;
    const uint32_t w = in[i].wide;
    int ch[8];
    int nch = 0;
    if (is_leaf(ref)) {
        ch[nch++] = ref;
    } else {
        // the children of the best distribution of 8 below `ref` (step 6): expand (binary node, slots) pairs
        // until each is one child (a binary leaf, a single-child decision, or a subtree that is a leaf)
        int st_ref[8];
        int st_n[8];
        int sp = 0;
        const Internal nd = nodes[ref];
        const int k8 = split[8 * (size_t)ref + 7];
        st_ref[sp] = nd.right; st_n[sp] = 8 - k8; ++sp;
        st_ref[sp] = nd.left; st_n[sp] = k8; ++sp;
        while (sp > 0 && nch < 8) {
            --sp;
            const int r = st_ref[sp];
            const int slots = st_n[sp];
            if (is_leaf(r) || slots == 1 || !((dist[r] >> slots) & 1u)) {
                ch[nch++] = r;
            } else {
                const Internal c = nodes[r];
                const int k = split[8 * (size_t)r + slots - 1];
                st_ref[sp] = c.right; st_n[sp] = slots - k; ++sp;
                st_ref[sp] = c.left; st_n[sp] = k; ++sp;
            }
        }
    }
    float4 cl[8], chh[8];
    float4 nlo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.0f), nhi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.0f);
    for (int k = 0; k < nch; ++k) {
        if (is_leaf(ch[k]) || !leafy[ch[k]]) {
            if (is_leaf(ch[k])) { cl[k] = slo[~ch[k]]; chh[k] = shi[~ch[k]]; }
            else { cl[k] = ilo[ch[k]]; chh[k] = ihi[ch[k]]; }
        } else {
            cl[k] = ilo[ch[k]];
            chh[k] = ihi[ch[k]];
        }
        nlo.x = fminf(nlo.x, cl[k].x); nlo.y = fminf(nlo.y, cl[k].y); nlo.z = fminf(nlo.z, cl[k].z);
        nhi.x = fmaxf(nhi.x, chh[k].x); nhi.y = fmaxf(nhi.y, chh[k].y); nhi.z = fmaxf(nhi.z, chh[k].z);
    }
    // octant slot assignment
    const float ncx = 0.5f * (nlo.x + nhi.x), ncy = 0.5f * (nlo.y + nhi.y), ncz = 0.5f * (nlo.z + nhi.z);
    int slot_of[8];
    int child_in_slot[8];
    for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
    unsigned used_slots = 0, used_children = 0;
    for (int it = 0; it < nch; ++it) {
        float best = FLT_MAX;
        int bk = 0, bs = 0;
        for (int k = 0; k < nch; ++k) {
            if (used_children & (1u << k)) continue;
            const float ox = 0.5f * (cl[k].x + chh[k].x) - ncx;
            const float oy = 0.5f * (cl[k].y + chh[k].y) - ncy;
            const float oz = 0.5f * (cl[k].z + chh[k].z) - ncz;
            for (int s = 0; s < 8; ++s) {
                if (used_slots & (1u << s)) continue;
                const float c = ((s & 1) ? -ox : ox) + ((s & 2) ? -oy : oy) + ((s & 4) ? -oz : oz);
                if (c < best) { best = c; bk = k; bs = s; }
            }
        }
        used_children |= 1u << bk;
        used_slots |= 1u << bs;
        slot_of[bk] = bs;
        child_in_slot[bs] = bk;
    }
    (void)slot_of;
    uint32_t n_internal = 0, n_tris = 0;
    for (int k = 0; k < nch; ++k) {
        const uint32_t c = ref_count(ch[k], nodes);
        if (!is_leaf(ch[k]) && !leafy[ch[k]]) ++n_internal;
        else n_tris += c;
    }
    const uint32_t child_base = n_internal ? atomicAdd(node_counter, n_internal) : 0u;
    const uint32_t tri_base = n_tris ? atomicAdd(tri_counter, n_tris) : 0u;
    const uint32_t out_base = n_internal ? atomicAdd(out_count, n_internal) : 0u;

    // quantisation frame
    const double ext[3] = { (double)nhi.x - (double)nlo.x, (double)nhi.y - (double)nlo.y, (double)nhi.z - (double)nlo.z };
    int e[3];
    for (int a = 0; a < 3; ++a) e[a] = exponent_for(ext[a]);
    const double p[3] = { nlo.x, nlo.y, nlo.z };
    uint8_t meta[8], qlo[3][8], qhi[3][8];
    uint32_t imask = 0, tri_off = 0, int_idx = 0;
    for (int s = 0; s < 8; ++s) {
        const int k = child_in_slot[s];
        if (k < 0) {
            meta[s] = 0;
            for (int a = 0; a < 3; ++a) { qlo[a][s] = 255; qhi[a][s] = 0; }
            continue;
        }
        const float lo3[3] = { cl[k].x, cl[k].y, cl[k].z }, hi3[3] = { chh[k].x, chh[k].y, chh[k].z };
        for (int a = 0; a < 3; ++a) {
            const double sc = ldexp(1.0, -e[a]);
            double ql = floor(((double)lo3[a] - p[a]) * sc);
            double qh = ceil(((double)hi3[a] - p[a]) * sc);
            ql = fmin(fmax(ql, 0.0), 255.0);
            qh = fmin(fmax(qh, 0.0), 255.0);
            qlo[a][s] = (uint8_t)ql;
            qhi[a][s] = (uint8_t)qh;
        }
        const uint32_t c = ref_count(ch[k], nodes);
        if (!is_leaf(ch[k]) && !leafy[ch[k]]) {
            imask |= 1u << s;
            meta[s] = (uint8_t)((1u << 5) | (24u + s));
            out[out_base + int_idx] = Frontier{ ch[k], child_base + int_idx };
            ++int_idx;
        } else {
            const uint32_t unary = (1u << c) - 1u;
            meta[s] = (uint8_t)((unary << 5) | tri_off);
            const uint32_t first = ref_first(ch[k], nodes);
            for (uint32_t q = 0; q < c; ++q) tris_out[tri_base + tri_off + q] = tris_in[vals[first + q]];
            tri_off += c;
        }
    }
    WideNode wn;
    wn.w[0] = make_uint4(__float_as_uint(nlo.x), __float_as_uint(nlo.y), __float_as_uint(nlo.z),
                         (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)(e[2] + 127) << 16) |
                             (imask << 24));
    auto pack4 = [](const uint8_t* b) {
        return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    wn.w[1] = make_uint4(child_base, tri_base, pack4(meta), pack4(meta + 4));
    wn.w[2] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
    wn.w[3] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
    wn.w[4] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
    wnodes[w] = wn;
}

template <typename T>
T* carve(char*& p, size_t count) {
    T* r = reinterpret_cast<T*>(p);
    p += ((count * sizeof(T) + 255) / 256) * 256;
    return r;
}

size_t cub_bytes(uint32_t n) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0, 63);
    return bytes;
}

}  // namespace

struct ScratchLayout {
    float4 *lo, *hi, *slo, *shi, *ilo, *ihi;
    uint64_t *keys, *keys2;
    uint32_t *vals, *vals2;
    Internal* nodes;
    int *iparent, *lparent;
    uint32_t* flags;
    Frontier *fa, *fb;
    float* cost;
    uint8_t *split, *dist, *leafy;
    int* cbounds;
    uint32_t* counters;
    void* cub_tmp;
    size_t cub_bytes;
    size_t total;
};

// Carves the scratch buffer (base may be null to only measure it).
static ScratchLayout layout(char* base, uint32_t n) {
    const size_t m = n ? n : 1;
    ScratchLayout L;
    char* p = base;
    L.lo = carve<float4>(p, m);
    L.hi = carve<float4>(p, m);
    L.slo = carve<float4>(p, m);
    L.shi = carve<float4>(p, m);
    L.ilo = carve<float4>(p, m);
    L.ihi = carve<float4>(p, m);
    L.keys = carve<uint64_t>(p, m);
    L.keys2 = carve<uint64_t>(p, m);
    L.vals = carve<uint32_t>(p, m);
    L.vals2 = carve<uint32_t>(p, m);
    L.nodes = carve<Internal>(p, m);
    L.iparent = carve<int>(p, m);
    L.lparent = carve<int>(p, m);
    L.flags = carve<uint32_t>(p, m);
    L.fa = carve<Frontier>(p, m);
    L.fb = carve<Frontier>(p, m);
    L.cost = carve<float>(p, 8 * m);
    L.split = carve<uint8_t>(p, 8 * m);
    L.dist = carve<uint8_t>(p, m);
    L.leafy = carve<uint8_t>(p, m);
    L.cbounds = carve<int>(p, 8);
    L.counters = carve<uint32_t>(p, 8);
    L.cub_bytes = cub_bytes((uint32_t)m);
    L.cub_tmp = carve<char>(p, L.cub_bytes);
    L.total = (size_t)(p - base);
    return L;
}

size_t build_scratch_bytes(uint32_t n) { return layout(nullptr, n).total; }

cudaError_t build_wide_bvh(const TriSlot* tris_in, uint32_t n, WideNode* wnodes, TriSlot* tris_out, void* scratch,
                           size_t scratch_bytes, cudaStream_t stream, BuildResult* result) {
    cudaError_t err;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    const size_t m = n ? n : 1;
    const ScratchLayout L = layout(static_cast<char*>(scratch), n);
    if (L.total > scratch_bytes) return cudaErrorInvalidValue;
    float4 *lo = L.lo, *hi = L.hi, *slo = L.slo, *shi = L.shi, *ilo = L.ilo, *ihi = L.ihi;
    uint64_t *keys = L.keys, *keys2 = L.keys2;
    uint32_t *vals = L.vals, *vals2 = L.vals2;
    Internal* nodes = L.nodes;
    int *iparent = L.iparent, *lparent = L.lparent;
    uint32_t* flags = L.flags;
    Frontier *fa = L.fa, *fb = L.fb;
    int* cbounds = L.cbounds;
    uint32_t* counters = L.counters;
    void* cub_tmp = L.cub_tmp;
    const size_t cb = L.cub_bytes;
    uint32_t node_count = 0;
    if (n == 0) {
        result->node_count = 0;
        result->ms = 0.0f;
        return cudaSuccess;
    }
    const int T = 256;
    const unsigned G = (unsigned)((n + T - 1) / T);
    const int init_bounds[8] = { INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN, 0, 0 };
    if ((err = cudaMemcpyAsync(cbounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, stream))) return err;
    k_tri_bounds<<<G, T, 0, stream>>>(tris_in, n, lo, hi, cbounds);
    k_morton<<<G, T, 0, stream>>>(lo, hi, n, cbounds, keys, vals);
    size_t cbb = cb;
    if ((err = cub::DeviceRadixSort::SortPairs(cub_tmp, cbb, keys, keys2, vals, vals2, (int)n, 0, 63, stream))) return err;
    k_gather_leaves<<<G, T, 0, stream>>>(vals2, lo, hi, n, slo, shi);
    if (n > 1) {
        if ((err = cudaMemsetAsync(flags, 0, sizeof(uint32_t) * m, stream))) return err;
        k_karras<<<(unsigned)((n - 1 + T - 1) / T), T, 0, stream>>>(keys2, n, nodes, iparent, lparent);
        k_refit<<<G, T, 0, stream>>>(nodes, iparent, lparent, slo, shi, ilo, ihi, flags, n);
        if ((err = cudaMemsetAsync(flags, 0, sizeof(uint32_t) * m, stream))) return err;
        k_sah_costs<<<G, T, 0, stream>>>(nodes, iparent, lparent, slo, shi, ilo, ihi, flags, L.cost, L.split, L.dist,
                                         L.leafy, n);
    }
    // collapse, one frontier level per launch
    const uint32_t init_counters[8] = { 1u, 0u, 0u, 0u, 0u, 0u, 0u, 0u };  // node_counter, tri_counter, out_count
    if ((err = cudaMemcpyAsync(counters, init_counters, sizeof(init_counters), cudaMemcpyHostToDevice, stream))) return err;
    const Frontier root{ n > 1 ? 0 : ~0, 0u };
    if ((err = cudaMemcpyAsync(fa, &root, sizeof(root), cudaMemcpyHostToDevice, stream))) return err;
    uint32_t count = 1;
    int guard = 0;
    while (count > 0) {
        if ((err = cudaMemsetAsync(counters + 2, 0, sizeof(uint32_t), stream))) return err;
        k_collapse<<<(count + 127) / 128, 128, 0, stream>>>(fa, count, fb, counters + 2, counters + 0, counters + 1,
                                                           nodes, slo, shi, ilo, ihi, vals2, tris_in, wnodes, tris_out,
                                                           L.split, L.dist, L.leafy);
        if ((err = cudaMemcpyAsync(&count, counters + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream))) return err;
        if ((err = cudaStreamSynchronize(stream))) return err;
        Frontier* t = fa; fa = fb; fb = t;
        if (++guard > 256) return cudaErrorUnknown;  // deeper than any tree over 2^32 primitives
    }
    if ((err = cudaMemcpyAsync(&node_count, counters + 0, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream))) return err;
    cudaEventRecord(e1, stream);
    if ((err = cudaStreamSynchronize(stream))) return err;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    result->node_count = node_count;
    result->ms = ms;
    return cudaGetLastError();
}


// The same build for callers that cannot allocate: no CUDA events, every buffer supplied by the caller
// (used by the static-scratch trace entry point in nalloc.cu).
cudaError_t build_wide_bvh_prealloc(const TriSlot* tris_in, uint32_t n, WideNode* wnodes, TriSlot* tris_out,
                                    void* scratch, size_t scratch_bytes, cudaStream_t stream, uint32_t* node_count_out) {
    cudaError_t err;
    const size_t m = n ? n : 1;
    const ScratchLayout L = layout(static_cast<char*>(scratch), n);
    if (L.total > scratch_bytes) return cudaErrorInvalidValue;
    *node_count_out = 0;
    if (n == 0) return cudaSuccess;
    Frontier *fa = L.fa, *fb = L.fb;
    const int T = 256;
    const unsigned G = (unsigned)((n + T - 1) / T);
    const int init_bounds[8] = { INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN, 0, 0 };
    if ((err = cudaMemcpyAsync(L.cbounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, stream))) return err;
    k_tri_bounds<<<G, T, 0, stream>>>(tris_in, n, L.lo, L.hi, L.cbounds);
    k_morton<<<G, T, 0, stream>>>(L.lo, L.hi, n, L.cbounds, L.keys, L.vals);
    size_t cbb = L.cub_bytes;
    if ((err = cub::DeviceRadixSort::SortPairs(L.cub_tmp, cbb, L.keys, L.keys2, L.vals, L.vals2, (int)n, 0, 63, stream)))
        return err;
    k_gather_leaves<<<G, T, 0, stream>>>(L.vals2, L.lo, L.hi, n, L.slo, L.shi);
    if (n > 1) {
        if ((err = cudaMemsetAsync(L.flags, 0, sizeof(uint32_t) * m, stream))) return err;
        k_karras<<<(unsigned)((n - 1 + T - 1) / T), T, 0, stream>>>(L.keys2, n, L.nodes, L.iparent, L.lparent);
        k_refit<<<G, T, 0, stream>>>(L.nodes, L.iparent, L.lparent, L.slo, L.shi, L.ilo, L.ihi, L.flags, n);
        if ((err = cudaMemsetAsync(L.flags, 0, sizeof(uint32_t) * m, stream))) return err;
        k_sah_costs<<<G, T, 0, stream>>>(L.nodes, L.iparent, L.lparent, L.slo, L.shi, L.ilo, L.ihi, L.flags, L.cost,
                                         L.split, L.dist, L.leafy, n);
    }
    const uint32_t init_counters[8] = { 1u, 0u, 0u, 0u, 0u, 0u, 0u, 0u };
    if ((err = cudaMemcpyAsync(L.counters, init_counters, sizeof(init_counters), cudaMemcpyHostToDevice, stream)))
        return err;
    const Frontier root{ n > 1 ? 0 : ~0, 0u };
    if ((err = cudaMemcpyAsync(fa, &root, sizeof(root), cudaMemcpyHostToDevice, stream))) return err;
    uint32_t count = 1;
    int guard = 0;
    while (count > 0) {
        if ((err = cudaMemsetAsync(L.counters + 2, 0, sizeof(uint32_t), stream))) return err;
        k_collapse<<<(count + 127) / 128, 128, 0, stream>>>(fa, count, fb, L.counters + 2, L.counters + 0, L.counters + 1,
                                                           L.nodes, L.slo, L.shi, L.ilo, L.ihi, L.vals2, tris_in, wnodes,
                                                           tris_out, L.split, L.dist, L.leafy);
        if ((err = cudaMemcpyAsync(&count, L.counters + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream))) return err;
        if ((err = cudaStreamSynchronize(stream))) return err;
        Frontier* t = fa;
        fa = fb;
        fb = t;
        if (++guard > 256) return cudaErrorUnknown;
    }
    if ((err = cudaMemcpyAsync(node_count_out, L.counters + 0, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)))
        return err;
    if ((err = cudaStreamSynchronize(stream))) return err;
    return cudaGetLastError();
}

}  // namespace pb2

