// The per-frame deformation of a resident scene, on the device: skin (renderer/shaders/skin.wgsl), leaf gather
// (renderer/shaders/leaf_gather.wgsl), the deforming meshes' trees refit bottom-up (units.rs:251-275 refit), the units'
// world boxes (units.rs:288-300 UnitBox::new) and the top tree built again (units.rs:140-224 build_sah under
// units.rs:303-326 top_tree). The reference does the last three on the CPU each frame; here every stage is a kernel
// and nothing but the palette crosses PCIe.
//
// Arithmetic is in source order under -fmad=false, so each stage rounds as its C++ restatement does: skinned vertices,
// leaves and refit boxes are bit-exact against the oracle, and the top tree is the one trt_prep_build's build_sah makes
// over the same boxes, node for node.
#include "deform.h"

#include <algorithm>
#include <cstring>
#include <unordered_map>

#include "device_common.cuh"

namespace trt {

constexpr uint32_t TOP_DEPTH = 19u;                 // units.rs:30-37: leaves at most TOP_DEPTH - 1 deep
constexpr uint32_t TOP_MAX_DEPTH = TOP_DEPTH - 1u;  // build_sah's max_depth
constexpr uint32_t TOP_LEVELS = TOP_MAX_DEPTH + 1u; // levels 0 .. TOP_MAX_DEPTH
constexpr uint32_t MAX_UNITS = 1u << TOP_MAX_DEPTH;
constexpr uint32_t TOP_BINS = 32u;                  // units.rs:121
// Top-tree nodes of more units than this are built by a CTA each (k_top_big), the rest by a warp each (k_top_level).
constexpr uint32_t TOP_SMALL = 256u, BIG_WARPS = 16u;
// Error bits the kernels record.
constexpr uint32_t E_TREE = 1u, E_DEPTH = 2u, E_ROOT = 4u, E_INDEX = 8u;

struct DMesh { uint32_t first_vertex, n_vertices, first_corner, palette, first_tri, n_tris, root, n_nodes; };
static_assert(sizeof(DMesh) == sizeof(trt_deform_mesh), "DMesh mirrors trt_deform_mesh");

// glam's Vec3A::min / max (SSE minps / maxps): the first operand where it is smaller (larger), else the second.
__host__ __device__ __forceinline__ float gmin(float a, float b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ float gmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ bool finite1(float v) { return (bu(v) & 0x7f800000u) != 0x7f800000u; }

// ---- skin.wgsl ----------------------------------------------------------------------------------------------------

__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 mul4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// skin.wgsl unit: v / |v| where |v| is positive and finite, else zero.
__device__ __forceinline__ V3 unit3(V3 v) {
    float l = sqrtf(dot(v, v));
    if (l > 0.0f && finite1(l)) return V3{v.x / l, v.y / l, v.z / l};
    return v3(0.0f);
}

// skin.wgsl:66-90 place, and main's writes (skin.wgsl:92-113): one thread a vertex, blockIdx.y a mesh.
__global__ void k_skin(const DMesh* __restrict__ meshes, uint32_t n_meshes, const float4* __restrict__ corners,
                       const float4* __restrict__ palette, float4* vertices) {
    for (uint32_t m = blockIdx.y; m < n_meshes; m += gridDim.y) {
        DMesh M = meshes[m];
        for (uint32_t local = blockIdx.x * blockDim.x + threadIdx.x; local < M.n_vertices; local += gridDim.x * blockDim.x) {
            const float4* c = corners + 4ull * (M.first_corner + local);
            float4 cp = c[0], cn = c[1], ct = c[2], cw = c[3];
            uint32_t a = bu(cp.w), b = bu(cn.w), flags = bu(ct.w);
            uint32_t j0 = (M.palette + (a & 0xffffu)) * 3u, j1 = (M.palette + (a >> 16)) * 3u;
            uint32_t j2 = (M.palette + (b & 0xffffu)) * 3u, j3 = (M.palette + (b >> 16)) * 3u;
            float4 r0 = add4(add4(add4(mul4(palette[j0], cw.x), mul4(palette[j1], cw.y)), mul4(palette[j2], cw.z)), mul4(palette[j3], cw.w));
            float4 r1 = add4(add4(add4(mul4(palette[j0 + 1], cw.x), mul4(palette[j1 + 1], cw.y)), mul4(palette[j2 + 1], cw.z)), mul4(palette[j3 + 1], cw.w));
            float4 r2 = add4(add4(add4(mul4(palette[j0 + 2], cw.x), mul4(palette[j1 + 2], cw.y)), mul4(palette[j2 + 2], cw.z)), mul4(palette[j3 + 2], cw.w));
            float4 p = make_float4(cp.x, cp.y, cp.z, 1.0f);
            V3 R0 = xyz(r0), R1 = xyz(r1), R2 = xyz(r2), N = xyz(cn), T = xyz(ct);
            V3 c12 = cross(R1, R2);
            V3 n = V3{dot(c12, N), dot(cross(R2, R0), N), dot(cross(R0, R1), N)};
            if (dot(R0, c12) < 0.0f) n = -n;
            V3 pos = V3{dot4(r0, p), dot4(r1, p), dot4(r2, p)};
            if (!(finite1(pos.x) && finite1(pos.y) && finite1(pos.z))) pos = v3(0.0f);
            uint64_t k = 3ull * (M.first_vertex + local);
            vertices[k] = f4(pos, vertices[k].w);
            if (flags & TRT_CORNER_NORMAL) vertices[k + 1] = f4(unit3(n), vertices[k + 1].w);
            if (flags & TRT_CORNER_TANGENT) vertices[k + 2] = f4(unit3(V3{dot(R0, T), dot(R1, T), dot(R2, T)}), vertices[k + 2].w);
        }
    }
}

// ---- leaf_gather.wgsl ---------------------------------------------------------------------------------------------

// Corner c of triangle t through its index; an index past the mesh's vertices is recorded and read as its first.
__device__ __forceinline__ V3 corner(const float4* vertices, const uint32_t* words, uint32_t w_indices, const DMesh& M,
                                     uint32_t t, uint32_t c, uint32_t* err) {
    uint32_t i = words[w_indices + t * 3u + c];
    if (i >= M.n_vertices) { atomicOr(err, E_INDEX); i = 0u; }
    return xyz(vertices[3ull * (M.first_vertex + i)]);
}

// ---- leaf gather (leaf_gather.wgsl) and refit (units.rs:251-275), one pass ------------------------------------------
//
// The reference refits a tree from its last node back to its root, one node after another, after a separate pass
// has gathered the leaves. Here one CTA takes a mesh's tree a level at a time, deepest first (every node of a level
// at once, a barrier between levels): a leaf gathers its triangles again from the vertices (leaf_gather.wgsl:41-51:
// (v0, keep w), (e1, keep w), (e2, 0)) and folds their corners into its box; an interior node joins its children's
// boxes, written a level before. The level order of each distinct tree shape is made once, at setup.

__device__ __forceinline__ void store_box(uint4* nodes, uint32_t i, V3 lo, V3 hi, uint32_t lf, uint32_t count) {
    nodes[2ull * i] = make_uint4(bu(lo.x), bu(lo.y), bu(lo.z), lf);
    nodes[2ull * i + 1] = make_uint4(bu(hi.x), bu(hi.y), bu(hi.z), count);
}

// A distinct tree shape: its leaves in triangle order, then its interior nodes a level at a time, deepest first
// (level_start[levels_first .. levels_first + n_levels] are offsets into its interior nodes).
struct Shape { uint32_t leaves_first, n_leaves, interior_first, levels_first, n_levels; };

// The leaves of every deforming mesh at once (one thread a leaf, blockIdx.y a mesh), neighbours in triangle order on
// neighbouring threads, whose corners they share.
__global__ void k_refit_leaves(const DMesh* __restrict__ meshes, const uint32_t* __restrict__ shape_of,
                               uint32_t n_meshes, const Shape* __restrict__ shapes,
                               const uint32_t* __restrict__ level_nodes, const float4* __restrict__ vertices,
                               const uint32_t* __restrict__ words, uint32_t w_indices, float4* leaves, uint4* nodes,
                               uint32_t* err) {
    for (uint32_t m = blockIdx.y; m < n_meshes; m += gridDim.y) {
        DMesh M = meshes[m];
        Shape sh = shapes[shape_of[m]];
        for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < sh.n_leaves; j += gridDim.x * blockDim.x) {
            uint32_t i = M.root + level_nodes[sh.leaves_first + j];
            uint4 na = nodes[2ull * i], nb = nodes[2ull * i + 1];
            V3 lo = v3(__uint_as_float(0x7f800000u)), hi = v3(__uint_as_float(0xff800000u));
            for (uint32_t k = na.w; k < na.w + nb.w; ++k) {
                uint32_t t = M.first_tri + k;
                V3 p[3];
                for (uint32_t c = 0; c < 3; ++c) {
                    p[c] = corner(vertices, words, w_indices, M, t, c, err);
                    if (finite1(p[c].x) && finite1(p[c].y) && finite1(p[c].z)) {
                        lo = V3{gmin(lo.x, p[c].x), gmin(lo.y, p[c].y), gmin(lo.z, p[c].z)};
                        hi = V3{gmax(hi.x, p[c].x), gmax(hi.y, p[c].y), gmax(hi.z, p[c].z)};
                    }
                }
                uint64_t q = 3ull * t;
                leaves[q] = f4(p[0], leaves[q].w);
                leaves[q + 1] = f4(p[1] - p[0], leaves[q + 1].w);
                leaves[q + 2] = f4(p[2] - p[0], 0.0f);
            }
            if (lo.x > hi.x) { lo = v3(0.0f); hi = v3(0.0f); }  // a leaf of nothing finite: a point
            store_box(nodes, i, lo, hi, na.w, nb.w);
        }
    }
}

// Then each mesh's interior nodes, a CTA a mesh, a level at a time from the deepest (a barrier between levels).
__global__ void k_refit(const DMesh* __restrict__ meshes, const uint32_t* __restrict__ shape_of, uint32_t n_meshes,
                        const Shape* __restrict__ shapes, const uint32_t* __restrict__ level_start,
                        const uint32_t* __restrict__ level_nodes, uint4* nodes) {
    for (uint32_t m = blockIdx.x; m < n_meshes; m += gridDim.x) {
        DMesh M = meshes[m];
        Shape sh = shapes[shape_of[m]];
        for (uint32_t l = 0; l < sh.n_levels; ++l) {
            uint32_t a = level_start[sh.levels_first + l], b = level_start[sh.levels_first + l + 1];
            for (uint32_t j = a + threadIdx.x; j < b; j += blockDim.x) {
                uint32_t i = M.root + level_nodes[sh.interior_first + j];
                uint4 na = __ldcg(nodes + 2ull * i), nb = __ldcg(nodes + 2ull * i + 1);
                uint64_t c = M.root + na.w;
                uint4 la = __ldcg(nodes + 2 * c), lb = __ldcg(nodes + 2 * c + 1);
                uint4 ra = __ldcg(nodes + 2 * c + 2), rb = __ldcg(nodes + 2 * c + 3);
                V3 lo = V3{gmin(__uint_as_float(la.x), __uint_as_float(ra.x)), gmin(__uint_as_float(la.y), __uint_as_float(ra.y)),
                           gmin(__uint_as_float(la.z), __uint_as_float(ra.z))};
                V3 hi = V3{gmax(__uint_as_float(lb.x), __uint_as_float(rb.x)), gmax(__uint_as_float(lb.y), __uint_as_float(rb.y)),
                           gmax(__uint_as_float(lb.z), __uint_as_float(rb.z))};
                store_box(nodes, i, lo, hi, na.w, nb.w);
            }
            __syncthreads();
        }
        __syncthreads();
    }
}

// ---- the top tree ---------------------------------------------------------------------------------------------------

struct TopBuild {
    float4* box;      // 2 a unit: lo, hi
    float4* centre;   // a unit's box centre
    uint32_t* order[2];
    // A level's nodes, (start, end, final index, interior nodes before it in preorder), in two lists: those of at most
    // TOP_SMALL units (a warp's each) and the larger (a CTA's each); cnt[2 * level + {0, 1}] counts them.
    uint4* tasks[2];
    uint4* big[2];
    uint32_t* cnt;
    uint32_t* err;
    uint4* nodes;
    uint32_t top_first, n_units;
};

// units.rs:288-300 UnitBox::new of each unit's tree root box under its world rows, its centre, and the build's start.
__global__ void k_unit_boxes(const uint4* __restrict__ tables, uint32_t t_instances, uint64_t n_nodes, TopBuild T) {
    uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u == 0) {
        bool large = T.n_units > TOP_SMALL;
        (large ? T.big[0] : T.tasks[0])[0] = make_uint4(0u, T.n_units, 0u, 0u);
        for (uint32_t l = 0; l <= TOP_LEVELS; ++l) T.cnt[2 * l] = T.cnt[2 * l + 1] = 0u;
        T.cnt[large ? 1 : 0] = 1u;
    }
    if (u >= T.n_units) return;
    T.order[0][u] = u;
    uint32_t b = t_instances + u * 10u;
    uint4 m0 = tables[b], m1 = tables[b + 1], m2 = tables[b + 2], n0 = tables[b + 3];
    uint32_t root = n0.w;
    V3 lo = v3(0.0f), hi = v3(0.0f);
    if (root < n_nodes) {
        uint4 na = T.nodes[2ull * root], nb = T.nodes[2ull * root + 1];
        lo = V3{__uint_as_float(na.x), __uint_as_float(na.y), __uint_as_float(na.z)};
        hi = V3{__uint_as_float(nb.x), __uint_as_float(nb.y), __uint_as_float(nb.z)};
    } else {
        atomicOr(T.err, E_ROOT);
    }
    float w[3][4] = {{__uint_as_float(m0.x), __uint_as_float(m0.y), __uint_as_float(m0.z), __uint_as_float(m0.w)},
                     {__uint_as_float(m1.x), __uint_as_float(m1.y), __uint_as_float(m1.z), __uint_as_float(m1.w)},
                     {__uint_as_float(m2.x), __uint_as_float(m2.y), __uint_as_float(m2.z), __uint_as_float(m2.w)}};
    V3 a = v3(__uint_as_float(0x7f800000u)), bb = v3(__uint_as_float(0xff800000u));
    for (int c = 0; c < 8; ++c) {
        V3 q = V3{(c & 1) == 0 ? lo.x : hi.x, (c & 2) == 0 ? lo.y : hi.y, (c & 4) == 0 ? lo.z : hi.z};
        // glam's Mat4 * point: x_axis * x + y_axis * y + z_axis * z + w_axis
        V3 p = V3{w[0][0] * q.x + w[0][1] * q.y + w[0][2] * q.z + w[0][3], w[1][0] * q.x + w[1][1] * q.y + w[1][2] * q.z + w[1][3],
                  w[2][0] * q.x + w[2][1] * q.y + w[2][2] * q.z + w[2][3]};
        a = V3{gmin(a.x, p.x), gmin(a.y, p.y), gmin(a.z, p.z)};
        bb = V3{gmax(bb.x, p.x), gmax(bb.y, p.y), gmax(bb.z, p.z)};
    }
    V3 e = bb - a;
    V3 m = V3{gmax(fabsf(a.x), fabsf(bb.x)), gmax(fabsf(a.y), fabsf(bb.y)), gmax(fabsf(a.z), fabsf(bb.z))};
    float pad = gmax(e.x, gmax(e.y, e.z)) * 1e-4f + gmax(m.x, gmax(m.y, m.z)) * 1e-5f + 1e-6f;
    V3 blo = a - v3(pad), bhi = bb + v3(pad);
    T.box[2ull * u] = f4(blo, 0.0f);
    T.box[2ull * u + 1] = f4(bhi, 0.0f);
    T.centre[u] = f4((blo + bhi) * 0.5f, 0.0f);
}

__device__ __forceinline__ float area3(V3 lo, V3 hi) {
    V3 e = V3{gmax(hi.x - lo.x, 0.0f), gmax(hi.y - lo.y, 0.0f), gmax(hi.z - lo.z, 0.0f)};
    return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
}
__device__ __forceinline__ float comp(float4 v, uint32_t axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
__device__ __forceinline__ float comp3(V3 v, uint32_t axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
// Rust's `f as usize` for the bin (non-negative here), saturating, NaN to 0, then at most TOP_BINS - 1.
__device__ __forceinline__ uint32_t bin_of(float c, float clo, float scale) {
    float f = (c - clo) * scale;
    if (!(f > 0.0f)) return 0u;
    return f >= (float)TOP_BINS ? TOP_BINS - 1u : min((uint32_t)f, TOP_BINS - 1u);
}
// f32::total_cmp's key.
__device__ __forceinline__ int32_t total_key(float f) {
    int32_t b = __float_as_int(f);
    return b ^ (int32_t)(((uint32_t)(b >> 31)) >> 1);
}

// A node's two children onto the next level's lists: the left one's place and preorder count follow from its
// parent's, the right one's from the left side's unit count.
__device__ __forceinline__ void push_children(const TopBuild& T, uint32_t level, uint32_t start, uint32_t mid,
                                              uint32_t end, uint32_t pre) {
    uint4 kids[2] = {make_uint4(start, start + mid, 1u + 2u * pre, pre + 1u),
                     make_uint4(start + mid, end, 2u + 2u * pre, pre + mid)};
    for (int c = 0; c < 2; ++c) {
        bool large = kids[c].y - kids[c].x > TOP_SMALL;
        uint32_t at = atomicAdd(&T.cnt[2 * (level + 1u) + (large ? 1 : 0)], 1u);
        (large ? T.big : T.tasks)[(level + 1u) & 1u][at] = kids[c];
    }
}

// A set of bins in shared memory ([axis][component][bin] boxes, [axis][bin] counts). While the units are added the
// boxes hold f32::total_cmp keys, joined by integer atomic min / max (exact whatever order the lanes and warps come
// in); bins_to_floats turns them back into floats for the sweep.
typedef float BinBoxes[3][TOP_BINS];
__device__ __forceinline__ float key_float(int32_t k) { return __int_as_float(total_key(__int_as_float(k))); }
__device__ __forceinline__ void bins_clear(BinBoxes* blo, BinBoxes* bhi, uint32_t (*bn)[TOP_BINS], uint32_t i0,
                                           uint32_t step) {
    const float lo0 = __int_as_float(total_key(__uint_as_float(0x7f800000u)));
    const float hi0 = __int_as_float(total_key(__uint_as_float(0xff800000u)));
    for (uint32_t i = i0; i < 3u * TOP_BINS; i += step) {
        const uint32_t ax = i / TOP_BINS, b = i % TOP_BINS;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            blo[ax][q][b] = lo0;
            bhi[ax][q][b] = hi0;
        }
        bn[ax][b] = 0u;
    }
}
// A unit into the bins its packed bins name (0xff: none on that axis).
__device__ __forceinline__ void bins_add(BinBoxes* blo, BinBoxes* bhi, uint32_t (*bn)[TOP_BINS], uint32_t packed,
                                         float4 bl, float4 bh) {
#pragma unroll
    for (uint32_t ax = 0; ax < 3; ++ax) {
        const uint32_t b = (packed >> (8u * ax)) & 0xffu;
        if (b >= TOP_BINS) continue;
        atomicMin(reinterpret_cast<int*>(&blo[ax][0][b]), total_key(bl.x));
        atomicMin(reinterpret_cast<int*>(&blo[ax][1][b]), total_key(bl.y));
        atomicMin(reinterpret_cast<int*>(&blo[ax][2][b]), total_key(bl.z));
        atomicMax(reinterpret_cast<int*>(&bhi[ax][0][b]), total_key(bh.x));
        atomicMax(reinterpret_cast<int*>(&bhi[ax][1][b]), total_key(bh.y));
        atomicMax(reinterpret_cast<int*>(&bhi[ax][2][b]), total_key(bh.z));
        atomicAdd(&bn[ax][b], 1u);
    }
}
__device__ __forceinline__ void bins_to_floats(BinBoxes* blo, BinBoxes* bhi, uint32_t i0, uint32_t step) {
    for (uint32_t i = i0; i < 3u * TOP_BINS; i += step) {
        const uint32_t ax = i / TOP_BINS, b = i % TOP_BINS;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            blo[ax][q][b] = key_float(__float_as_int(blo[ax][q][b]));
            bhi[ax][q][b] = key_float(__float_as_int(bhi[ax][q][b]));
        }
    }
}
// A unit's bins on the three axes, 8 bits each (0xff for an invalid unit or an axis not in use).
__device__ __forceinline__ uint32_t pack_bins(bool valid, float4 c, V3 clo, const float scale[3], const bool use[3]) {
    uint32_t p = 0u;
#pragma unroll
    for (uint32_t ax = 0; ax < 3; ++ax)
        p |= (valid && use[ax] ? bin_of(comp(c, ax), comp3(clo, ax), scale[ax]) : 0xffu) << (8u * ax);
    return p;
}

// build_sah's sweep over one set of bins (blo / bhi [axis][component][bin], bn [axis][bin]), a warp at once: lane i
// holds split i (bins 0 .. i-1 to the left). The left sides are an inclusive scan over the bins before, the right
// sides one over the bins from i on (min, max and sums: exact, as the reference's running folds are), each lane then
// computes the split's cost as build_sah does, and the warp takes the first cheapest in build_sah's order (axis, then
// split) among the splits that leave both sides non-empty and within `room`. Every lane gets the result.
__device__ void sah_sweep(const float (*blo)[3][TOP_BINS], const float (*bhi)[3][TOP_BINS], const uint32_t (*bn)[TOP_BINS],
                          const bool use[3], uint32_t count, uint32_t room, float& best_cost, uint32_t& best_axis,
                          uint32_t& best_split, uint32_t& best_left) {
    const uint32_t lane = threadIdx.x & 31u;
    const float pinf = __uint_as_float(0x7f800000u);
    float cost_best = pinf;
    uint32_t key_best = 0xffffffffu, left_best = 0;
    for (uint32_t ax = 0; ax < 3; ++ax) {
        if (!use[ax]) continue;
        // this lane's bin
        float l0 = blo[ax][0][lane], l1 = blo[ax][1][lane], l2 = blo[ax][2][lane];
        float h0 = bhi[ax][0][lane], h1 = bhi[ax][1][lane], h2 = bhi[ax][2][lane];
        uint32_t c = bn[ax][lane];
        // suffix over bins lane .. 31 (the right side of split `lane`)
        float rl0 = l0, rl1 = l1, rl2 = l2, rh0 = h0, rh1 = h1, rh2 = h2;
        // prefix over bins 0 .. lane (the left side of split lane + 1)
        float pl0 = l0, pl1 = l1, pl2 = l2, ph0 = h0, ph1 = h1, ph2 = h2;
        uint32_t pc = c;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            float t;
            t = __shfl_down_sync(~0u, rl0, o); if (lane + o < 32) rl0 = gmin(rl0, t);
            t = __shfl_down_sync(~0u, rl1, o); if (lane + o < 32) rl1 = gmin(rl1, t);
            t = __shfl_down_sync(~0u, rl2, o); if (lane + o < 32) rl2 = gmin(rl2, t);
            t = __shfl_down_sync(~0u, rh0, o); if (lane + o < 32) rh0 = gmax(rh0, t);
            t = __shfl_down_sync(~0u, rh1, o); if (lane + o < 32) rh1 = gmax(rh1, t);
            t = __shfl_down_sync(~0u, rh2, o); if (lane + o < 32) rh2 = gmax(rh2, t);
            t = __shfl_up_sync(~0u, pl0, o); if (lane >= o) pl0 = gmin(pl0, t);
            t = __shfl_up_sync(~0u, pl1, o); if (lane >= o) pl1 = gmin(pl1, t);
            t = __shfl_up_sync(~0u, pl2, o); if (lane >= o) pl2 = gmin(pl2, t);
            t = __shfl_up_sync(~0u, ph0, o); if (lane >= o) ph0 = gmax(ph0, t);
            t = __shfl_up_sync(~0u, ph1, o); if (lane >= o) ph1 = gmax(ph1, t);
            t = __shfl_up_sync(~0u, ph2, o); if (lane >= o) ph2 = gmax(ph2, t);
            uint32_t u = __shfl_up_sync(~0u, pc, o);
            if (lane >= o) pc += u;
        }
        // split i = lane: left = prefix of bins 0 .. i-1 (the lane below's), right = suffix from bin i
        float ql0 = __shfl_up_sync(~0u, pl0, 1), ql1 = __shfl_up_sync(~0u, pl1, 1), ql2 = __shfl_up_sync(~0u, pl2, 1);
        float qh0 = __shfl_up_sync(~0u, ph0, 1), qh1 = __shfl_up_sync(~0u, ph1, 1), qh2 = __shfl_up_sync(~0u, ph2, 1);
        uint32_t nl = __shfl_up_sync(~0u, pc, 1);
        uint32_t nr = count - nl;
        float cost = pinf;
        bool ok = lane >= 1 && nl != 0 && nr != 0 && nl <= room && nr <= room;
        if (ok) cost = area3(V3{ql0, ql1, ql2}, V3{qh0, qh1, qh2}) * (float)nl +
                       area3(V3{rl0, rl1, rl2}, V3{rh0, rh1, rh2}) * (float)nr;
        // a split counts where it is cheaper than the best so far (the reference's `cost < best`)
        bool cand = ok && cost < pinf;
        uint32_t key = cand ? ax * 32u + lane : 0xffffffffu;
        float cv = cand ? cost : pinf;
        // the first cheapest of this axis: min by (cost, key)
#pragma unroll
        for (uint32_t o = 16; o > 0; o >>= 1) {
            float oc = __shfl_xor_sync(~0u, cv, o);
            uint32_t ok2 = __shfl_xor_sync(~0u, key, o);
            uint32_t ol = __shfl_xor_sync(~0u, nl, o);
            if (oc < cv || (oc == cv && ok2 < key)) { cv = oc; key = ok2; nl = ol; }
        }
        if (key != 0xffffffffu && cv < cost_best) { cost_best = cv; key_best = key; left_best = nl; }
    }
    best_cost = cost_best;
    best_axis = key_best == 0xffffffffu ? 0u : key_best / 32u;
    best_split = key_best == 0xffffffffu ? 0u : key_best % 32u;
    best_left = left_best;
}

// The median split's side of unit k: its rank among the node's units by (centre along the axis in f32::total_cmp
// order, then index) against half the count.
__device__ __forceinline__ bool median_left(const TopBuild& T, const uint32_t* order, uint32_t start, uint32_t end,
                                            uint32_t k, uint32_t axis) {
    int32_t kk = total_key(comp(T.centre[k], axis));
    uint32_t rank = 0;
    for (uint32_t q = start; q < end; ++q) {
        uint32_t o = order[q];
        int32_t ko = total_key(comp(T.centre[o], axis));
        rank += (ko < kk || (ko == kk && o < k)) ? 1u : 0u;
    }
    return rank < (end - start) / 2u;
}

// Tasks of more units than this are the CTA kernel's (k_top_big); the rest a warp's (k_top_level).

constexpr uint32_t TOP_WARPS = 8u;

// One level of the build: a warp a node. It takes the node's boxes (order[level & 1][start, end)), picks the split
// build_sah picks (the cheapest binned split along the centres' axes among those the depth allows, else the median
// along the widest axis), writes the node where build_sah's depth-first layout puts it and hands its two children to
// the next level with their items partitioned into order[(level + 1) & 1]. In that layout a node's children sit at
// 1 + 2 * I and 2 + 2 * I, where I counts the interior nodes before it in preorder: a left child's I is its parent's
// plus one, a right child's its parent's plus the left side's item count (a subtree of k items has k - 1 interior
// nodes), so each node's place is known when it is made.
__global__ void __launch_bounds__(TOP_WARPS * 32) k_top_level(TopBuild T, uint32_t level) {
    __shared__ float s_lo[TOP_WARPS][3][3][TOP_BINS], s_hi[TOP_WARPS][3][3][TOP_BINS];
    __shared__ uint32_t s_n[TOP_WARPS][3][TOP_BINS];
    uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    uint32_t n_tasks = T.cnt[2 * level];
    const uint32_t* order = T.order[level & 1u];
    uint32_t* out = T.order[(level + 1u) & 1u];
    const uint4* tasks = T.tasks[level & 1u];
    for (uint32_t ti = blockIdx.x * TOP_WARPS + wib; ti < n_tasks; ti += gridDim.x * TOP_WARPS) {
        uint4 task = tasks[ti];
        uint32_t start = task.x, end = task.y, fin = task.z, pre = task.w, count = end - start;
        V3 lo = v3(__uint_as_float(0x7f800000u)), hi = v3(__uint_as_float(0xff800000u)), clo = lo, chi = hi;
        for (uint32_t j = start + lane; j < end; j += 32u) {
            uint32_t k = order[j];
            float4 bl = T.box[2ull * k], bh = T.box[2ull * k + 1], c = T.centre[k];
            lo = V3{gmin(lo.x, bl.x), gmin(lo.y, bl.y), gmin(lo.z, bl.z)};
            hi = V3{gmax(hi.x, bh.x), gmax(hi.y, bh.y), gmax(hi.z, bh.z)};
            clo = V3{gmin(clo.x, c.x), gmin(clo.y, c.y), gmin(clo.z, c.z)};
            chi = V3{gmax(chi.x, c.x), gmax(chi.y, c.y), gmax(chi.z, c.z)};
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = V3{gmin(lo.x, __shfl_xor_sync(~0u, lo.x, o)), gmin(lo.y, __shfl_xor_sync(~0u, lo.y, o)), gmin(lo.z, __shfl_xor_sync(~0u, lo.z, o))};
            hi = V3{gmax(hi.x, __shfl_xor_sync(~0u, hi.x, o)), gmax(hi.y, __shfl_xor_sync(~0u, hi.y, o)), gmax(hi.z, __shfl_xor_sync(~0u, hi.z, o))};
            clo = V3{gmin(clo.x, __shfl_xor_sync(~0u, clo.x, o)), gmin(clo.y, __shfl_xor_sync(~0u, clo.y, o)), gmin(clo.z, __shfl_xor_sync(~0u, clo.z, o))};
            chi = V3{gmax(chi.x, __shfl_xor_sync(~0u, chi.x, o)), gmax(chi.y, __shfl_xor_sync(~0u, chi.y, o)), gmax(chi.z, __shfl_xor_sync(~0u, chi.z, o))};
        }
        if (fin >= 2u * T.n_units - 1u || count == 0 || end > T.n_units) {  // (a build of n leaves has 2n - 1 nodes)
            if (lane == 0) atomicOr(T.err, E_TREE);
            continue;
        }
        uint32_t node = T.top_first + fin;
        if (count == 1) {
            if (lane == 0) store_box(T.nodes, node, lo, hi, order[start], 1u);
            continue;
        }
        if (level >= TOP_MAX_DEPTH || count > MAX_UNITS) {
            if (lane == 0) atomicOr(T.err, E_DEPTH);
            continue;
        }
        uint32_t room = 1u << (TOP_MAX_DEPTH - level - 1u);
        V3 ext = chi - clo;
        float scale[3] = {(float)TOP_BINS / ext.x, (float)TOP_BINS / ext.y, (float)TOP_BINS / ext.z};
        bool use[3] = {ext.x > 0.0f, ext.y > 0.0f, ext.z > 0.0f};
        bins_clear(s_lo[wib], s_hi[wib], s_n[wib], lane, 32u);
        __syncwarp();
        for (uint32_t base = start; base < end; base += 32u) {
            uint32_t j = base + lane;
            bool valid = j < end;
            uint32_t k = valid ? order[j] : order[start];
            float4 bl = T.box[2ull * k], bh = T.box[2ull * k + 1], c = T.centre[k];
            bins_add(s_lo[wib], s_hi[wib], s_n[wib], pack_bins(valid, c, clo, scale, use), bl, bh);
        }
        __syncwarp();
        bins_to_floats(s_lo[wib], s_hi[wib], lane, 32u);
        __syncwarp();
        float best_cost = 0.0f;
        uint32_t best_axis = 0, best_split = 0, best_left = 0;
        sah_sweep(s_lo[wib], s_hi[wib], s_n[wib], use, count, room, best_cost, best_axis, best_split, best_left);
        bool binned = finite1(best_cost);
        uint32_t med_axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0u : (ext.y >= ext.z ? 1u : 2u);
        uint32_t mid = binned ? best_left : count / 2u;
        // Partition, left side first (stable: the order inside a side does not change the tree).
        uint32_t nl_run = 0, nr_run = 0;
        for (uint32_t base = start; base < end; base += 32u) {
            uint32_t j = base + lane;
            bool valid = j < end, left = false;
            uint32_t k = valid ? order[j] : 0u;
            if (valid) {
                if (binned) {
                    left = bin_of(comp(T.centre[k], best_axis), comp3(clo, best_axis), scale[best_axis]) < best_split;
                } else {
                    left = median_left(T, order, start, end, k, med_axis);
                }
            }
            unsigned lm = __ballot_sync(~0u, valid && left), rm = __ballot_sync(~0u, valid && !left);
            unsigned below = (1u << lane) - 1u;
            if (valid) {
                if (left) out[start + nl_run + __popc(lm & below)] = k;
                else out[start + mid + nr_run + __popc(rm & below)] = k;
            }
            nl_run += __popc(lm);
            nr_run += __popc(rm);
        }
        if (lane == 0) {
            if (nl_run != mid) atomicOr(T.err, E_TREE);
            store_box(T.nodes, node, lo, hi, 1u + 2u * pre, 0u);
            push_children(T, level, start, mid, end, pre);
        }
    }
}


// The same step for nodes of more than TOP_SMALL units, a CTA a node: each warp bins its share of the units into its
// own set of bins, the sets are joined, one thread sweeps them, and the partition is a CTA-wide stable scan.
__global__ void __launch_bounds__(BIG_WARPS * 32) k_top_big(TopBuild T, uint32_t level) {
    __shared__ float s_lo[BIG_WARPS][3][3][TOP_BINS], s_hi[BIG_WARPS][3][3][TOP_BINS];
    __shared__ uint32_t s_n[BIG_WARPS][3][TOP_BINS];
    __shared__ float s_red[BIG_WARPS][12];
    __shared__ uint32_t s_side[BIG_WARPS][2];
    __shared__ float s_cost;
    __shared__ uint32_t s_best[3];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5, nt = BIG_WARPS * 32u;
    const float pinf = __uint_as_float(0x7f800000u), ninf = __uint_as_float(0xff800000u);
    uint32_t n_tasks = T.cnt[2 * level + 1];
    const uint32_t* order = T.order[level & 1u];
    uint32_t* out = T.order[(level + 1u) & 1u];
    const uint4* tasks = T.big[level & 1u];
    for (uint32_t ti = blockIdx.x; ti < n_tasks; ti += gridDim.x) {
        uint4 task = tasks[ti];
        uint32_t start = task.x, end = task.y, fin = task.z, pre = task.w, count = end - start;
        if (fin >= 2u * T.n_units - 1u || end > T.n_units || level >= TOP_MAX_DEPTH) {
            if (tid == 0) atomicOr(T.err, level >= TOP_MAX_DEPTH ? E_DEPTH : E_TREE);
            continue;
        }
        // The node's box and its units' centres' box.
        float r[12] = {pinf, pinf, pinf, ninf, ninf, ninf, pinf, pinf, pinf, ninf, ninf, ninf};
        for (uint32_t j = start + tid; j < end; j += nt) {
            uint32_t k = order[j];
            float4 bl = T.box[2ull * k], bh = T.box[2ull * k + 1], c = T.centre[k];
            r[0] = gmin(r[0], bl.x); r[1] = gmin(r[1], bl.y); r[2] = gmin(r[2], bl.z);
            r[3] = gmax(r[3], bh.x); r[4] = gmax(r[4], bh.y); r[5] = gmax(r[5], bh.z);
            r[6] = gmin(r[6], c.x); r[7] = gmin(r[7], c.y); r[8] = gmin(r[8], c.z);
            r[9] = gmax(r[9], c.x); r[10] = gmax(r[10], c.y); r[11] = gmax(r[11], c.z);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                float v = __shfl_xor_sync(~0u, r[q], o);
                r[q] = (q % 6) < 3 ? gmin(r[q], v) : gmax(r[q], v);
            }
        if (lane == 0)
            for (int q = 0; q < 12; ++q) s_red[w][q] = r[q];
        for (uint32_t i = tid; i < BIG_WARPS * 3u * TOP_BINS; i += nt)
            bins_clear(s_lo[i / (3u * TOP_BINS)], s_hi[i / (3u * TOP_BINS)], s_n[i / (3u * TOP_BINS)],
                       i % (3u * TOP_BINS), 3u * TOP_BINS);
        __syncthreads();
        for (int q = 0; q < 12; ++q) {
            float v = s_red[0][q];
            for (uint32_t ww = 1; ww < BIG_WARPS; ++ww) v = (q % 6) < 3 ? gmin(v, s_red[ww][q]) : gmax(v, s_red[ww][q]);
            r[q] = v;
        }
        V3 lo{r[0], r[1], r[2]}, hi{r[3], r[4], r[5]}, clo{r[6], r[7], r[8]}, chi{r[9], r[10], r[11]};
        uint32_t room = 1u << (TOP_MAX_DEPTH - level - 1u);
        V3 ext = chi - clo;
        float scale[3] = {(float)TOP_BINS / ext.x, (float)TOP_BINS / ext.y, (float)TOP_BINS / ext.z};
        bool use[3] = {ext.x > 0.0f, ext.y > 0.0f, ext.z > 0.0f};
        for (uint32_t base = start + 32u * w; base < end; base += nt) {
            uint32_t j = base + lane;
            bool valid = j < end;
            uint32_t k = valid ? order[j] : order[start];
            float4 bl = T.box[2ull * k], bh = T.box[2ull * k + 1], c = T.centre[k];
            bins_add(s_lo[w], s_hi[w], s_n[w], pack_bins(valid, c, clo, scale, use), bl, bh);
        }
        __syncthreads();
        // The warps' bins joined into warp 0's, on their keys (min / max and sums do not depend on the order).
        for (uint32_t i = tid; i < 3u * TOP_BINS; i += nt) {
            uint32_t ax = i / TOP_BINS, bn = i % TOP_BINS;
            for (uint32_t ww = 1; ww < BIG_WARPS; ++ww) {
                for (int q = 0; q < 3; ++q) {
                    s_lo[0][ax][q][bn] = __int_as_float(
                        min(__float_as_int(s_lo[0][ax][q][bn]), __float_as_int(s_lo[ww][ax][q][bn])));
                    s_hi[0][ax][q][bn] = __int_as_float(
                        max(__float_as_int(s_hi[0][ax][q][bn]), __float_as_int(s_hi[ww][ax][q][bn])));
                }
                s_n[0][ax][bn] += s_n[ww][ax][bn];
            }
        }
        __syncthreads();
        bins_to_floats(s_lo[0], s_hi[0], tid, nt);
        __syncthreads();
        if (w == 0) {
            float c;
            uint32_t a, sp, l;
            sah_sweep(s_lo[0], s_hi[0], s_n[0], use, count, room, c, a, sp, l);
            if (lane == 0) {
                s_cost = c;
                s_best[0] = a; s_best[1] = sp; s_best[2] = l;
            }
        }
        __syncthreads();
        bool binned = finite1(s_cost);
        uint32_t best_axis = s_best[0], best_split = s_best[1];
        uint32_t med_axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0u : (ext.y >= ext.z ? 1u : 2u);
        uint32_t mid = binned ? s_best[2] : count / 2u;
        // Stable partition, a CTA-wide chunk at a time.
        uint32_t nl_run = 0, nr_run = 0;
        for (uint32_t base = start; base < end; base += nt) {
            uint32_t j = base + tid;
            bool valid = j < end, left = false;
            uint32_t k = valid ? order[j] : 0u;
            if (valid)
                left = binned ? bin_of(comp(T.centre[k], best_axis), comp3(clo, best_axis), scale[best_axis]) < best_split
                              : median_left(T, order, start, end, k, med_axis);
            unsigned lm = __ballot_sync(~0u, valid && left), rm = __ballot_sync(~0u, valid && !left);
            if (lane == 0) { s_side[w][0] = __popc(lm); s_side[w][1] = __popc(rm); }
            __syncthreads();
            uint32_t lb = 0, rb = 0, lt = 0, rt = 0;
            for (uint32_t ww = 0; ww < BIG_WARPS; ++ww) {
                if (ww < w) { lb += s_side[ww][0]; rb += s_side[ww][1]; }
                lt += s_side[ww][0];
                rt += s_side[ww][1];
            }
            unsigned below = (1u << lane) - 1u;
            if (valid) {
                if (left) out[start + nl_run + lb + __popc(lm & below)] = k;
                else out[start + mid + nr_run + rb + __popc(rm & below)] = k;
            }
            nl_run += lt;
            nr_run += rt;
            __syncthreads();
        }
        if (tid == 0) {
            if (nl_run != mid) atomicOr(T.err, E_TREE);
            store_box(T.nodes, T.top_first + fin, lo, hi, 1u + 2u * pre, 0u);
            push_children(T, level, start, mid, end, pre);
        }
        __syncthreads();
    }
}

}  // namespace trt

// ---- host ----------------------------------------------------------------------------------------------------------

namespace trt {

struct DeformState {
    DMesh* meshes = nullptr;
    float4* corners = nullptr;
    // The refit's level order: each mesh's shape, each distinct shape's levels (deepest first) and their nodes.
    uint32_t* shape_of = nullptr;
    Shape* shapes = nullptr;
    uint32_t* level_start = nullptr;
    uint32_t* level_nodes = nullptr;
    uint32_t* err = nullptr;
    float4* palette = nullptr;
    uint32_t palette_cap = 0;
    void* top = nullptr;           // the top build's scratch
    uint32_t top_units = 0;
    TopBuild T{};
    std::vector<DMesh> host_meshes;
    std::vector<uint32_t> max_bone;  // per mesh: the largest palette index its corners name
    uint32_t max_vertices = 0, max_tris = 0, max_nodes = 0, max_leaves = 0;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

namespace {

int cuda_err(std::string& err, cudaError_t e, const char* what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return TRT_ECUDA;
}
#define DF_CUDA(call)                                              \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_err(err, e_, #call);    \
    } while (0)

// Reads node i of the host copy.
void host_node(const std::vector<uint8_t>& nodes, uint64_t i, uint32_t w[8]) { std::memcpy(w, nodes.data() + 32 * i, 32); }

int ensure_top(DeformState* st, uint32_t n_units, std::string& err) {
    if (st->top && st->top_units >= n_units) return TRT_OK;
    if (st->top) cudaFree(st->top);
    st->top = nullptr;
    uint64_t need = 0;
    auto add = [&](uint64_t b) { uint64_t at = need; need += (b + 255) / 256 * 256; return at; };
    uint64_t n_big = n_units / (TOP_SMALL + 1u) + 1u;  // nodes of a level are disjoint: at most this many large
    uint64_t o_box = add(32ull * n_units), o_c = add(16ull * n_units), o_o0 = add(4ull * n_units),
             o_o1 = add(4ull * n_units), o_t0 = add(16ull * n_units), o_t1 = add(16ull * n_units),
             o_b0 = add(16ull * n_big), o_b1 = add(16ull * n_big), o_cnt = add(8ull * (TOP_LEVELS + 1));
    DF_CUDA(cudaMalloc(&st->top, need));
    char* b = (char*)st->top;
    st->T.box = (float4*)(b + o_box);
    st->T.centre = (float4*)(b + o_c);
    st->T.order[0] = (uint32_t*)(b + o_o0);
    st->T.order[1] = (uint32_t*)(b + o_o1);
    st->T.tasks[0] = (uint4*)(b + o_t0);
    st->T.tasks[1] = (uint4*)(b + o_t1);
    st->T.big[0] = (uint4*)(b + o_b0);
    st->T.big[1] = (uint4*)(b + o_b1);
    st->T.cnt = (uint32_t*)(b + o_cnt);
    st->top_units = n_units;
    return TRT_OK;
}

dim3 mesh_grid(uint32_t per_mesh, uint32_t n_meshes) {
    uint32_t x = std::max(1u, std::min((per_mesh + 255u) / 256u, 1024u));
    uint32_t y = std::max(1u, std::min(n_meshes, 65535u));
    return dim3(x, y);
}

}  // namespace

void deform_free(DeformState* st) {
    if (!st) return;
    for (void* p : {(void*)st->meshes, (void*)st->corners, (void*)st->shape_of, (void*)st->shapes,
                    (void*)st->level_start, (void*)st->level_nodes, (void*)st->err, (void*)st->palette, st->top})
        if (p) cudaFree(p);
    for (auto& e : st->ev)
        if (e) cudaEventDestroy(e);
    delete st;
}

int deform_setup(DeformState** out, const SceneBuffers& sb, const trt_deform_desc* d, std::string& err) {
    if (!d || (d->n_meshes && !d->meshes) || (d->n_corners && !d->corners)) { err = "trt_deform_setup: a null array"; return TRT_EINVAL; }
    const uint64_t n_vertices = sb.bytes[0] / 48, n_tris = sb.bytes[1] / 48, n_nodes = sb.bytes[2] / 32;
    const std::vector<uint8_t>& hn = sb.host[2];
    if (hn.size() != sb.bytes[2]) { err = "trt_deform_setup: the scene's node copy is missing"; return TRT_EINVAL; }
    std::vector<uint32_t> refs(n_nodes, 0);
    auto* st = new DeformState();
    auto fail = [&](const std::string& m) { deform_free(st); err = "trt_deform_setup: " + m; return TRT_EINVAL; };
    st->host_meshes.assign((const DMesh*)d->meshes, (const DMesh*)d->meshes + d->n_meshes);
    st->max_bone.assign(d->n_meshes, 0);
    // Distinct tree shapes (the links and counts of a tree's nodes), each with its nodes by level, deepest first.
    std::unordered_map<std::string, uint32_t> shape_ids;
    std::vector<Shape> shapes;
    std::vector<uint32_t> shape_of(d->n_meshes), level_start, level_nodes;
    for (uint32_t m = 0; m < d->n_meshes; ++m) {
        const DMesh& M = st->host_meshes[m];
        std::string at = "mesh " + std::to_string(m) + ": ";
        if ((uint64_t)M.first_vertex + M.n_vertices > n_vertices) return fail(at + "vertices past the scene's");
        if ((uint64_t)M.first_corner + M.n_vertices > d->n_corners) return fail(at + "corners past the corners given");
        if ((uint64_t)M.first_tri + M.n_tris > n_tris) return fail(at + "triangles past the scene's");
        if (M.n_nodes == 0 || (uint64_t)M.root + M.n_nodes > n_nodes) return fail(at + "nodes past the scene's");
        // The tree: children after their parent and inside the tree, each node a child once, each of the mesh's
        // triangles in one leaf.
        std::string key(8ull * M.n_nodes, '\0');
        std::vector<uint8_t> covered(M.n_tris, 0);
        for (uint32_t k = 0; k < M.n_nodes; ++k) {
            uint32_t w[8];
            host_node(hn, M.root + k, w);
            std::memcpy(&key[8ull * k], &w[3], 4);
            std::memcpy(&key[8ull * k + 4], &w[7], 4);
            if (w[7] == 0) {
                if (w[3] <= k || (uint64_t)w[3] + 1 >= M.n_nodes) return fail(at + "a node's children are not after it in its tree");
                refs[M.root + w[3]]++;
                refs[M.root + w[3] + 1]++;
            } else {
                if ((uint64_t)w[3] + w[7] > M.n_tris) return fail(at + "a leaf's triangles are past the mesh's");
                for (uint32_t t = w[3]; t < w[3] + w[7]; ++t)
                    if (covered[t]++) return fail(at + "a triangle is in two leaves");
            }
        }
        for (uint32_t k = 0; k < M.n_nodes; ++k)
            if (refs[M.root + k] != (k == 0 ? 0u : 1u)) return fail(at + "a node is not the child of one node");
        for (uint32_t t = 0; t < M.n_tris; ++t)
            if (!covered[t]) return fail(at + "a triangle is in no leaf");
        auto found = shape_ids.find(key);
        if (found != shape_ids.end()) {
            shape_of[m] = found->second;
        } else {
            std::vector<uint32_t> depth(M.n_nodes, 0);
            uint32_t deepest = 0;
            for (uint32_t k = 0; k < M.n_nodes; ++k) {  // children after parents: a parent's depth is known first
                uint32_t w[8];
                host_node(hn, M.root + k, w);
                if (w[7] == 0) depth[w[3]] = depth[w[3] + 1] = depth[k] + 1;
                deepest = std::max(deepest, depth[k]);
            }
            if (deepest >= 64) return fail(at + "a tree deeper than 64 levels");
            // The shape: its leaves by first triangle, then its interior nodes by level, deepest first
            // (n_levels + 1 offsets into them from level_start[levels_first]).
            Shape sh{(uint32_t)level_nodes.size(), 0, 0, (uint32_t)level_start.size(), deepest + 1};
            std::vector<std::pair<uint32_t, uint32_t>> by_tri;
            for (uint32_t k = 0; k < M.n_nodes; ++k) {
                uint32_t w[8];
                host_node(hn, M.root + k, w);
                if (w[7] > 0) by_tri.push_back({w[3], k});
            }
            std::sort(by_tri.begin(), by_tri.end());
            for (auto& pr : by_tri) level_nodes.push_back(pr.second);
            sh.n_leaves = (uint32_t)by_tri.size();
            sh.interior_first = (uint32_t)level_nodes.size();
            level_start.push_back(0);
            for (uint32_t l = deepest + 1; l-- > 0;) {
                for (uint32_t k = 0; k < M.n_nodes; ++k) {
                    uint32_t w[8];
                    host_node(hn, M.root + k, w);
                    if (depth[k] == l && w[7] == 0) level_nodes.push_back(k);
                }
                level_start.push_back((uint32_t)level_nodes.size() - sh.interior_first);
            }
            shape_of[m] = (uint32_t)shapes.size();
            shape_ids.emplace(std::move(key), shape_of[m]);
            shapes.push_back(sh);
        }
        for (uint32_t v = 0; v < M.n_vertices; ++v) {
            const trt_corner& c = d->corners[M.first_corner + v];
            uint32_t a, b;
            std::memcpy(&a, &c.p[3], 4);
            std::memcpy(&b, &c.n[3], 4);
            st->max_bone[m] = std::max({st->max_bone[m], a & 0xffffu, a >> 16, b & 0xffffu, b >> 16});
        }
        st->max_vertices = std::max(st->max_vertices, M.n_vertices);
        st->max_tris = std::max(st->max_tris, M.n_tris);
        st->max_nodes = std::max(st->max_nodes, M.n_nodes);
        st->max_leaves = std::max(st->max_leaves, shapes[shape_of[m]].n_leaves);
    }
    cudaError_t e = cudaSuccess;
    auto upload = [&](auto** dst, const void* src, uint64_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMalloc((void**)dst, bytes);
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, sb.stream);
    };
    upload(&st->meshes, d->meshes, sizeof(DMesh) * d->n_meshes);
    upload(&st->corners, d->corners, sizeof(trt_corner) * d->n_corners);
    upload(&st->shape_of, shape_of.data(), 4ull * shape_of.size());
    upload(&st->shapes, shapes.data(), sizeof(Shape) * shapes.size());
    upload(&st->level_start, level_start.data(), 4ull * level_start.size());
    upload(&st->level_nodes, level_nodes.data(), 4ull * level_nodes.size());
    if (e == cudaSuccess) e = cudaMalloc(&st->err, 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->err, 0, 4, sb.stream);
    for (auto& ev : st->ev)
        if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sb.stream);
    if (e != cudaSuccess) {
        deform_free(st);
        return cuda_err(err, e, "trt_deform_setup");
    }
    *out = st;
    return TRT_OK;
}

int deform_run(DeformState* st, const SceneBuffers& sb, const uint32_t* P, const float* palette_rows,
               uint32_t n_matrices, uint32_t flags, trt_deform_stats* stats, std::string& err) {
    if (flags != 0) { err = "trt_deform: flags must be 0"; return TRT_EINVAL; }
    uint32_t n_meshes = (uint32_t)st->host_meshes.size();
    for (uint32_t m = 0; m < n_meshes; ++m)
        if ((uint64_t)st->host_meshes[m].palette + st->max_bone[m] >= n_matrices) {
            err = "trt_deform: mesh " + std::to_string(m) + "'s palette indices reach past the matrices given";
            return TRT_EINVAL;
        }
    if (n_meshes && !palette_rows) { err = "trt_deform: no palette"; return TRT_EINVAL; }
    const uint64_t n_nodes = sb.bytes[2] / 32;
    uint32_t t_instances = P[P_TABLE_FIRST + 7], w_indices = P[P_WORD_FIRST + 4];
    uint32_t top = P[P_MOTION + 2], n_units = P[P_MOTION + 3];
    if (n_units == 0 || n_units > MAX_UNITS) { err = "trt_deform: Params.motion.w (units) must be 1 to 2^18"; return TRT_EINVAL; }
    if ((uint64_t)top + 2ull * n_units - 1 > n_nodes) { err = "trt_deform: the top tree's nodes reach past the node buffer"; return TRT_EINVAL; }
    if ((uint64_t)t_instances + 10ull * n_units > sb.bytes[3] / 16) { err = "trt_deform: the units' records reach past the tables"; return TRT_EINVAL; }
    for (uint32_t m = 0; m < n_meshes; ++m)
        if ((uint64_t)w_indices + 3ull * (st->host_meshes[m].first_tri + st->host_meshes[m].n_tris) > sb.bytes[4] / 4) {
            err = "trt_deform: a mesh's indices reach past the words";
            return TRT_EINVAL;
        }
    cudaStream_t s = sb.stream;
    if (n_meshes) {
        if (n_matrices > st->palette_cap) {
            if (st->palette) cudaFree(st->palette);
            st->palette = nullptr;
            DF_CUDA(cudaMalloc(&st->palette, 48ull * n_matrices));
            st->palette_cap = n_matrices;
        }
        DF_CUDA(cudaMemcpyAsync(st->palette, palette_rows, 48ull * n_matrices, cudaMemcpyHostToDevice, s));
    }
    int rc = ensure_top(st, n_units, err);
    if (rc) return rc;
    if (stats) DF_CUDA(cudaEventRecord(st->ev[0], s));
    float4* vertices = (float4*)sb.buf[0];
    float4* leaves = (float4*)sb.buf[1];
    uint4* nodes = (uint4*)sb.buf[2];
    const uint32_t* words = (const uint32_t*)sb.buf[4];
    if (n_meshes) k_skin<<<mesh_grid(st->max_vertices, n_meshes), 256, 0, s>>>(st->meshes, n_meshes, st->corners, st->palette, vertices);
    if (stats) DF_CUDA(cudaEventRecord(st->ev[1], s));
    // (The leaf gather is the refit's leaf level: gather_ms stays 0 and refit_ms holds both.)
    if (stats) DF_CUDA(cudaEventRecord(st->ev[2], s));
    if (n_meshes) {
        // A CTA a mesh; few meshes get wide CTAs so that a single tree's levels still fill many warps.
        uint32_t threads = n_meshes < 296u ? 1024u : 256u;
        uint32_t blocks = std::min(n_meshes, 148u * (2048u / threads) * 4u);
        k_refit_leaves<<<mesh_grid(st->max_leaves, n_meshes), 256, 0, s>>>(st->meshes, st->shape_of, n_meshes, st->shapes,
                                                                            st->level_nodes, vertices, words, w_indices,
                                                                            leaves, nodes, st->err);
        k_refit<<<blocks, threads, 0, s>>>(st->meshes, st->shape_of, n_meshes, st->shapes, st->level_start,
                                           st->level_nodes, nodes);
    }
    if (stats) DF_CUDA(cudaEventRecord(st->ev[3], s));
    TopBuild T = st->T;
    T.err = st->err;
    T.nodes = nodes;
    T.top_first = top;
    T.n_units = n_units;
    k_unit_boxes<<<(n_units + 255) / 256, 256, 0, s>>>((const uint4*)sb.buf[3], t_instances, n_nodes, T);
    for (uint32_t level = 0; level < TOP_LEVELS; ++level) {
        uint32_t most = std::min<uint32_t>(1u << level, n_units);  // a level holds at most 2^level nodes
        uint32_t big = std::min(most, n_units / (TOP_SMALL + 1u));  // ... and at most this many of over TOP_SMALL
        if (big) k_top_big<<<std::min(big, 148u * 2u), BIG_WARPS * 32, 0, s>>>(T, level);
        uint32_t blocks = std::max(1u, std::min((most + TOP_WARPS - 1) / TOP_WARPS, 148u * 8u));
        k_top_level<<<blocks, TOP_WARPS * 32, 0, s>>>(T, level);
    }
    if (stats) DF_CUDA(cudaEventRecord(st->ev[4], s));
    DF_CUDA(cudaGetLastError());
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        DF_CUDA(cudaEventSynchronize(st->ev[4]));
        cudaEventElapsedTime(&stats->device_ms, st->ev[0], st->ev[4]);
        cudaEventElapsedTime(&stats->skin_ms, st->ev[0], st->ev[1]);
        cudaEventElapsedTime(&stats->gather_ms, st->ev[1], st->ev[2]);
        cudaEventElapsedTime(&stats->refit_ms, st->ev[2], st->ev[3]);
        cudaEventElapsedTime(&stats->top_ms, st->ev[3], st->ev[4]);
        rc = deform_errors(st, s, &stats->errors);
        if (rc) return rc;
        if (stats->errors) {
            err = "trt_deform: the device found a bad tree (error bits " + std::to_string(stats->errors) + ")";
            return TRT_EGUARD;
        }
    }
    return TRT_OK;
}

uint32_t* deform_error_word(DeformState* st) { return st->err; }

int deform_errors(DeformState* st, cudaStream_t stream, uint32_t* errors) {
    uint32_t e = 0;
    if (cudaMemcpyAsync(&e, st->err, 4, cudaMemcpyDeviceToHost, stream) != cudaSuccess) return TRT_ECUDA;
    if (cudaMemsetAsync(st->err, 0, 4, stream) != cudaSuccess) return TRT_ECUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return TRT_ECUDA;
    *errors = e;
    return TRT_OK;
}

}  // namespace trt
