// The wide BVH: the reference's binary trees (the units' top tree and every mesh tree) collapsed into 8-wide nodes
// whose child boxes are quantised to 8 bits against the node's origin, each node five 16-byte loads. It is built from
// the uploaded buffers (wide_bvh.cu) and walked by `trace_wide`; the triangle test is the reference's own
// Moller-Trumbore on the same unit-space ray (pathtrace.wgsl:742-761), so every hit and its t are the reference's.
//
// Node (80 bytes):
//   [0, 12)  origin xyz (f32)                     [12, 15) exponent byte a axis (the scale 2^(e - 127))
//   [15]     interior mask: bit i, slot i is a wide node
//   [16, 20) first interior child's node index   [20, 24) first leaf item of the node
//   [24, 32) items of each leaf slot (0: interior or empty): a leaf slot's items follow the lower slots' in order
//   [32, 80) q_lo x[8], q_lo y[8], q_lo z[8], q_hi x[8], q_hi y[8], q_hi z[8]: slot i's box is
//            origin + q * scale, widened by a step on every side; an empty slot has q_lo > q_hi.
// Leaf items: in a mesh tree, triangles (a copy of the reference's leaf record, three vec4s, with the reference's
// triangle index in the third's w); in the top tree, unit records (bit 31: the unit casts shadows).
#pragma once
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "traverse.cuh"

namespace trt {

struct WideView {
    const uint4* nodes;        // 5 uint4 a node
    const float4* tris;        // 3 float4 a triangle: (v0, section), (e1, rank), (e2, reference index)
    const uint32_t* units;     // the top tree's leaf items: unit record | shadow bit << 31
    const uint32_t* unit_root; // a unit record's mesh tree root (wide node index)
    uint32_t top_root;         // the top tree's root (wide node index)
    uint32_t n_nodes, n_tris, n_units, n_records;
};

constexpr uint32_t WIDE_UNIT_BIT = 0x80000000u;
// The walk's stack: entries of 8 bytes, the first WIDE_SHORT of each thread's in shared memory (a column a thread),
// the rest in local memory. A kernel that walks the wide BVH runs blocks of at most WIDE_BLOCK threads.
constexpr int WIDE_SHORT = 8;
constexpr int WIDE_STACK = 64;
constexpr uint32_t WIDE_BLOCK = 128;

// std::min / std::max on floats as the host build calls them (the second operand when it compares smaller / larger,
// else the first), so that the device refit rounds and picks as the host build does.
__host__ __device__ __forceinline__ float wmin(float a, float b) { return b < a ? b : a; }
__host__ __device__ __forceinline__ float wmax(float a, float b) { return a < b ? b : a; }

// Writes wide node W (the layout above) over child boxes bmin / bmax by slot: `present` the occupied slots, `imask`
// the interior ones, counts[i] a leaf slot's items (0 otherwise). The node's own box is the children's, widened by a
// pad (a 253rd of its extent, 2^-16 of its coordinates' magnitude and the tree's pad) so that the widened boxes stay
// within 0..255 steps; each axis's step is the power of two that covers the padded extent in 255 steps, and each child
// box is rounded outwards and widened by a step on every side. Shared by the host build and the device refit.
__host__ __device__ inline void wide_encode(uint32_t W[20], const float bmin[8][3], const float bmax[8][3],
                                            uint32_t present, uint32_t imask, uint32_t child_base, uint32_t leaf_base,
                                            const uint32_t counts[8], float tree_pad) {
    for (int i = 0; i < 20; ++i) W[i] = 0u;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < 8; ++i)
        if (present >> i & 1u)
            for (int k = 0; k < 3; ++k) { lo[k] = wmin(lo[k], bmin[i][k]); hi[k] = wmax(hi[k], bmax[i][k]); }
    float origin[3];
    int ex[3];
    for (int k = 0; k < 3; ++k) {
        const float ext = hi[k] - lo[k];
        const float mag = wmax(fabsf(lo[k]), fabsf(hi[k]));
        const float pad = ext * (1.0f / 253.0f) + mag * (1.0f / 65536.0f) + tree_pad + 1e-20f;
        origin[k] = lo[k] - pad;
        const float range = (hi[k] + pad) - origin[k];
        int e;
        frexpf(range / 255.0f, &e);  // range / 255 < 2^e
        for (int guard = 0; guard < 512 && ldexpf(255.0f, e) < range; ++guard) ++e;
        ex[k] = e < -126 ? -126 : (e > 127 ? 127 : e);
    }
    uint32_t q[12] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};  // q_lo x, y, z then q_hi x, y, z: 8 bytes each
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) {
            uint32_t a = 255u, b = 0u;  // an empty slot: q_lo > q_hi
            if (present >> i & 1u) {
                const double s = (double)ldexpf(1.0f, ex[k]);
                const double fa = floor((double)(bmin[i][k] - origin[k]) / s) - 1.0;
                const double fb = ceil((double)(bmax[i][k] - origin[k]) / s) + 1.0;
                const double ca = fa < 255.0 ? fa : 255.0, cb = fb < 255.0 ? fb : 255.0;
                a = (uint32_t)(0.0 < ca ? ca : 0.0);
                b = (uint32_t)(0.0 < cb ? cb : 0.0);
            }
            q[2 * k + (i >> 2)] |= a << (8 * (i & 3));
            q[6 + 2 * k + (i >> 2)] |= b << (8 * (i & 3));
        }
    for (int k = 0; k < 3; ++k) {
        float o = origin[k];
        uint32_t u;
        memcpy(&u, &o, 4);
        W[k] = u;
    }
    W[3] = (uint32_t)(ex[0] + 127) | ((uint32_t)(ex[1] + 127) << 8) | ((uint32_t)(ex[2] + 127) << 16) | (imask << 24);
    W[4] = child_base;
    W[5] = leaf_base;
    for (int i = 0; i < 8; ++i) W[6 + (i >> 2)] |= (counts[i] & 0xffu) << (8 * (i & 3));
    for (int j = 0; j < 12; ++j) W[8 + j] = q[j];
}

// A slot of the build's record: no child, or (for every slot of a node of the units' top tree) not refit in place:
// the top tree is built again by each deformation, so its wide nodes are collapsed again instead.
constexpr uint32_t WIDE_SLOT_EMPTY = 0xFFFFFFFFu, WIDE_SLOT_TOP = 0xFFFFFFFEu;

struct WideBvh {
    uint4* nodes = nullptr;  // the built nodes, then room for a collapsed-again top tree
    float4* tris = nullptr;
    uint32_t* units = nullptr;
    uint32_t* unit_root = nullptr;
    WideView v{};
    bool built = false;
    uint32_t key[6] = {0, 0, 0, 0, 0, 0};  // the Params words the build read (it is redone when they change)
    double build_ms = 0.0;
    // What a refit needs: for each built node the binary node each slot was collapsed from (8 a node) and its tree's
    // pad, on the host from the build, on the device from the first refit on.
    std::vector<uint32_t> slot_host;
    std::vector<float> pad_host;
    uint32_t* slot_dev = nullptr;
    float* pad_dev = nullptr;
    uint2* frontier = nullptr;   // the top collapse's two frontiers of (binary node, wide node), top_cap each
    uint32_t n_built = 0;        // nodes of the build; the top region starts here
    uint32_t top_cap = 0;        // the top region's nodes: a collapsed top tree has at most one a unit
    uint64_t refit_gen = 0;      // the deformation the wide trees were last brought to (0: the scene as uploaded)
    bool ready() const { return built; }
    WideView view() const { return v; }
    std::string error;
    // Builds (or keeps) the wide trees for the scene as `params` lays it out, from host copies of the scene's nodes,
    // leaves and tables (host[2], host[1], host[3]). 0, or 1 with `error` set.
    int ensure(const uint32_t* params, const std::vector<uint8_t>* host, cudaStream_t st);
    // Brings built wide trees to the scene's device buffers after a deformation (units.rs:251-275 refit, then the top
    // tree's collapse): every mesh tree's node quantised again over its binary children's refit boxes, the triangle
    // copies gathered again from the leaves, the rebuilt top tree collapsed again into the top region. Asynchronous on
    // `st`; an index out of its buffer sets err_bit in *err (the kernels skip the access). 0, or 1 with `error` set.
    int refit(const uint32_t* params, const void* bin_nodes, uint64_t n_bin, const void* leaves, uint64_t n_leaf_tris,
              const void* tables, uint64_t n_table_vec4, uint32_t* err, uint32_t err_bit, cudaStream_t st);
    // Whether `params` lays the scene out as the build read it.
    bool key_matches(const uint32_t* params) const;
    // Whether writing src[0, bytes) at byte `offset` of the tables (old: the host copy before it) changes a word the
    // build read: a unit record's mesh root, first triangle or bits.
    bool reads_edit(const uint8_t* old_tables, uint64_t tables_bytes, uint64_t offset, const uint8_t* src,
                    uint64_t bytes) const;
    void release();
    void invalidate() { built = false; }
};

struct WideRay {
    V3 o, d, inv;
    uint32_t neg;  // bit k: the direction's axis k is negative (its near planes are the boxes' high sides)
};
__device__ __forceinline__ WideRay wide_ray(V3 o, V3 d, V3 inv) {
    return WideRay{o, d, inv, (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u)};
}

// Byte k of w as an exact float: one byte permute builds 2^23 + byte (the float 0x4B0000bb), one add removes 2^23.
// (It keeps the conversion off the XU pipe, whose quarter rate bounded the walk when it used integer-to-float
// conversions: 48 a node.)
__device__ __forceinline__ float q_byte(uint32_t w, int k) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | (uint32_t)k)) - 8388608.0f;
}

// The eight child boxes of node `nd` against the ray: bit i of the result is set when slot i's box is entered before
// tmax; *tmin is the nearest hit slot's entry t (INF: none). A slot's plane at q steps is origin + q 2^e:
// t = q (2^e / d) + (origin - o) / d, one FMA. The near and far planes of each axis are picked once by the ray's signs;
// an empty slot (q_lo > q_hi) has its near plane past its far one on every axis, so it misses whatever the signs.
__device__ __forceinline__ uint32_t wide_hits(const uint4 nd[5], const WideRay& r, float tmax, float* tmin) {
    const uint32_t eb = nd[0].w;
    const float Sx = __uint_as_float((eb & 0xffu) << 23) * r.inv.x;
    const float Sy = __uint_as_float(((eb >> 8) & 0xffu) << 23) * r.inv.y;
    const float Sz = __uint_as_float(((eb >> 16) & 0xffu) << 23) * r.inv.z;
    const float Bx = (bf(nd[0].x) - r.o.x) * r.inv.x, By = (bf(nd[0].y) - r.o.y) * r.inv.y,
                Bz = (bf(nd[0].z) - r.o.z) * r.inv.z;
    // q_lo x: nd[2].x,y; y: nd[2].z,w; z: nd[3].x,y. q_hi x: nd[3].z,w; y: nd[4].x,y; z: nd[4].z,w.
    const bool nx = r.neg & 1u, ny = r.neg & 2u, nz = r.neg & 4u;
    const uint32_t nearx[2] = {nx ? nd[3].z : nd[2].x, nx ? nd[3].w : nd[2].y};
    const uint32_t farx[2] = {nx ? nd[2].x : nd[3].z, nx ? nd[2].y : nd[3].w};
    const uint32_t neary[2] = {ny ? nd[4].x : nd[2].z, ny ? nd[4].y : nd[2].w};
    const uint32_t fary[2] = {ny ? nd[2].z : nd[4].x, ny ? nd[2].w : nd[4].y};
    const uint32_t nearz[2] = {nz ? nd[4].z : nd[3].x, nz ? nd[4].w : nd[3].y};
    const uint32_t farz[2] = {nz ? nd[3].x : nd[4].z, nz ? nd[3].y : nd[4].w};
    uint32_t hits = 0;
    float tm = INF;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int h = i >> 2, k = i & 3;
        const float x0 = fmaf(q_byte(nearx[h], k), Sx, Bx), x1 = fmaf(q_byte(farx[h], k), Sx, Bx);
        const float y0 = fmaf(q_byte(neary[h], k), Sy, By), y1 = fmaf(q_byte(fary[h], k), Sy, By);
        const float z0 = fmaf(q_byte(nearz[h], k), Sz, Bz), z1 = fmaf(q_byte(farz[h], k), Sz, Bz);
        const float tnear = max3f(x0, y0, fmaxf(z0, 0.0f));
        const float tfar = min3f(x1, y1, fminf(z1, tmax));
        const bool hit = tnear <= tfar;
        hits |= (hit ? 1u : 0u) << i;
        tm = fminf(tm, hit ? tnear : INF);
    }
    *tmin = tm;
    return hits;
}

// An 8-bit slot mask in visit order: bit k is slot k ^ oct's. The builder places children in slots by octant (slot
// bit a: the upper half along axis a), so the ray's sign bits as oct make the lowest visit bit the nearest octant.
__device__ __forceinline__ uint32_t visit_mask(uint32_t m, uint32_t oct) {
    m = (oct & 1u) ? (((m & 0x55u) << 1) | ((m >> 1) & 0x55u)) : m;
    m = (oct & 2u) ? (((m & 0x33u) << 2) | ((m >> 2) & 0x33u)) : m;
    m = (oct & 4u) ? (((m & 0x0fu) << 4) | ((m >> 4) & 0x0fu)) : m;
    return m;
}

// Slot i's items in a node's leaf list: (first item, count). (A node's items number at most 8 x 16: the byte-wise
// running sum does not carry.)
__device__ __forceinline__ uint2 slot_items(uint32_t leaf_base, uint32_t c_lo, uint32_t c_hi, uint32_t slot) {
    const uint64_t counts = ((uint64_t)c_hi << 32) | c_lo;
    const uint32_t cnt = (uint32_t)(counts >> (8 * slot)) & 0xffu;
    const uint32_t upto = (uint32_t)((counts * 0x0101010101010101ull) >> (8 * slot)) & 0xffu;  // slots 0..slot
    return make_uint2(leaf_base + upto - cnt, cnt);
}

// The walk over both levels by node groups (Ylitie, Karras and Laine, "Efficient incoherent ray traversal on GPUs
// through compressed wide BVHs", HPG 2017): opening a node tests its eight children at once and leaves its hit
// interior children as one group, (first child's index, hit mask in visit order | interior mask), from which the walk
// takes the nearest child next; what is left of a group goes onto the stack as one 8-byte entry when the walk
// descends. No child is sorted or pushed on its own. A node's hit leaf slots are done before its children, in visit
// order: a mesh's triangles are tested on the spot (the reference's Moller-Trumbore on the unit-space ray,
// pathtrace.wgsl:742-761), and a top-tree node's hit units become a unit group entry (node, slots in visit order, item
// cursor) that enters them one at a time, the ray taken into each unit's space as trace_units.wgsl:86-105 does; a
// unit's walk ends when the stack is back to where it was entered. Each entry carries a lower bound of its group's
// nearest entry distance, and a group that lies past the closest hit is dropped unopened. Shadow rays (TRACE_SHADOW)
// skip units that cast no shadow, and any-hit rays stop at the first triangle hit. The first WIDE_SHORT entries of a
// thread's stack are in shared memory (wide_smem, a column a thread); more than WIDE_STACK end the walk with the
// guard set.
//
// The walk is a state (WideWalk) advanced one node at a time (wide_step). (Measured on the city frame: giving a lane
// whose ray is done the next ray between steps, while its warp's other lanes walk on, gained 3 % at best against a
// warp that takes 32 new rays when all are done, and the state kept across steps cost more than that in spills.)
struct WideWalk {
    V3 o, d, inv_d;          // the world's ray
    WideRay r;               // the ray in the current level's space
    Hit hit;
    uint32_t node;           // the node to open next
    uint32_t g_base, g_bits; // the current node group (entry layout)
    uint32_t rec, iter, mode;
    int sp, base;            // stack depth; the depth at which the current unit was entered
};

__device__ __forceinline__ uint2* wide_smem() {
    __shared__ uint2 short_stack[WIDE_SHORT * WIDE_BLOCK];
    return short_stack;
}

// Starts a walk; false when there is nothing to walk (w.hit is then the miss).
__device__ __forceinline__ bool wide_begin(WideWalk& w, const WideView& W, V3 o, V3 d, float tmax, uint32_t mode) {
    w.hit = Hit{tmax, MISS, 0.0f, 0.0f, NO_INST, 0u};
    if (W.n_units == 0) return false;
    w.o = o;
    w.d = d;
    w.inv_d = safe_inv(d);
    w.r = wide_ray(o, d, w.inv_d);
    w.node = W.top_root;
    w.g_base = w.g_bits = 0;
    w.rec = NO_INST;
    w.iter = 0;
    w.mode = mode;
    w.sp = w.base = 0;
    return true;
}

// One node of the walk: opens w.node, tests its hit leaves, takes the next node. Returns false when the walk is over
// (w.hit is its result; *guard set when it gave up on a tree that is not one).
template <bool COUNT>
__device__ __forceinline__ bool wide_step(WideWalk& w, const DScene& S, const WideView& W, const Sections& X,
                                          uint2* short_stack, uint2* spill, WalkCount* wc, bool* guard) {
    const uint32_t tid = threadIdx.x;
#define WIDE_PUSH(X_, Y_)                                                                      \
    do {                                                                                       \
        if (w.sp >= WIDE_STACK) { *guard = true; return false; }                               \
        if (w.sp < WIDE_SHORT) short_stack[w.sp * WIDE_BLOCK + tid] = make_uint2((X_), (Y_)); \
        else spill[w.sp - WIDE_SHORT] = make_uint2((X_), (Y_));                                \
        ++w.sp;                                                                                \
    } while (0)
    // An entry: a node group, x its first child's index, y = imask | hits (visit order) << 8 | t << 16; or a unit
    // group, x its node | ENTRY_UNITS, y = item cursor | slots (visit order) << 8 | t << 16. t: the top 16 bits of
    // the group's nearest entry distance (truncated: a lower bound).
    constexpr uint32_t ENTRY_UNITS = 0x80000000u;
    const auto t_of = [](uint32_t y) { return __uint_as_float(y & 0xffff0000u); };
    if (w.iter++ >= WALK_GUARD || w.node >= W.n_nodes) { *guard = true; return false; }
    {
        const uint4* np = W.nodes + 5ull * w.node;
        uint4 nd[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) nd[k] = __ldg(np + k);
        if (COUNT) wc->nodes++;
        float tmin;
        const uint32_t hm = wide_hits(nd, w.r, w.hit.t, &tmin);
        const uint32_t imask = nd[0].w >> 24;
        const uint32_t t16 = __float_as_uint(tmin) & 0xffff0000u;
        w.g_base = nd[1].x;
        w.g_bits = (visit_mask(hm & imask, w.r.neg) << 8) | imask | t16;
        uint32_t leaf = visit_mask(hm & ~imask, w.r.neg);
        if (leaf != 0u) {
            if (w.rec == NO_INST) {
                // Units: the group of this node's hit unit slots goes on top of what is left of its children.
                if (w.g_bits & 0xff00u) WIDE_PUSH(w.g_base, w.g_bits);
                w.g_bits = 0;
                WIDE_PUSH(w.node | ENTRY_UNITS, (leaf << 8) | t16);
            } else {
                do {
                    const uint32_t slot = ((uint32_t)__ffs(leaf) - 1u) ^ w.r.neg;
                    leaf &= leaf - 1u;
                    const uint2 it = slot_items(nd[1].y, nd[1].z, nd[1].w, slot);
                    for (uint32_t q = 0; q < it.y; ++q) {
                        const uint32_t ti = it.x + q;
                        if (ti >= W.n_tris) { *guard = true; return false; }
                        const float4* tp = W.tris + 3ull * ti;
                        const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
                        if (COUNT) wc->tris++;
                        // pathtrace.wgsl:742-761 intersect_tri, on the copy of the reference's leaf record.
                        const V3 v0 = xyz(a), e1 = xyz(b), e2 = xyz(c);
                        const V3 pv = cross(w.r.d, e2);
                        const float det = dot(e1, pv);
                        if (fabsf(det) < 1e-12f) continue;
                        const float inv = 1.0f / det;
                        const V3 tv = w.r.o - v0;
                        const float u = dot(tv, pv) * inv;
                        if (u < 0.0f || u > 1.0f) continue;
                        const V3 qv = cross(tv, e1);
                        const float v = dot(w.r.d, qv) * inv;
                        if (v < 0.0f || u + v > 1.0f) continue;
                        const float t = dot(e2, qv) * inv;
                        if (t <= 0.0f || t >= w.hit.t) continue;
                        w.hit = Hit{t, bu(c.w), u, v, w.rec, bu(a.w)};
                        if (w.mode != TRACE_CLOSEST) return false;
                    }
                } while (leaf != 0u);
            }
        }
    }
    // The next node: the nearest child left in the group, else the stack's top (a group, or the next unit of a unit
    // group, entered); groups whose nearest entry lies past the closest hit are dropped.
    for (;;) {
        if ((w.g_bits & 0xff00u) && t_of(w.g_bits) < w.hit.t) {
            const uint32_t k = (uint32_t)__ffs(w.g_bits >> 8) - 1u;
            w.g_bits &= ~(1u << (k + 8u));
            const uint32_t slot = k ^ w.r.neg;
            w.node = w.g_base + (uint32_t)__popc(w.g_bits & ((1u << slot) - 1u) & 0xffu);
            if (w.g_bits & 0xff00u) WIDE_PUSH(w.g_base, w.g_bits);
            return true;
        }
        if (w.rec != NO_INST && w.sp == w.base) {  // the unit's walk is over: back to the world's ray
            w.rec = NO_INST;
            w.r = wide_ray(w.o, w.d, w.inv_d);
        }
        if (w.sp == 0) return false;
        --w.sp;
        const uint2 e = w.sp < WIDE_SHORT ? short_stack[w.sp * WIDE_BLOCK + tid] : spill[w.sp - WIDE_SHORT];
        w.g_bits = 0;
        if (t_of(e.y) >= w.hit.t) continue;
        if (!(e.x & ENTRY_UNITS)) {
            w.g_base = e.x;
            w.g_bits = e.y;
            continue;
        }
        // The next unit of a unit group (its slots in the world ray's visit order, a cursor in the first).
        const uint32_t un = e.x & ~ENTRY_UNITS;
        if (un >= W.n_nodes) { *guard = true; return false; }
        const uint4 n1 = __ldg(W.nodes + 5ull * un + 1);
        uint32_t um = (e.y >> 8) & 0xffu;
        const uint32_t cursor = e.y & 0xffu;
        const uint32_t slot = ((uint32_t)__ffs(um) - 1u) ^ w.r.neg;
        const uint2 it = slot_items(n1.y, n1.z, n1.w, slot);
        const uint32_t item = it.x + cursor;
        if (cursor + 1u < it.y) {
            WIDE_PUSH(e.x, (e.y & 0xffff0000u) | (um << 8) | (cursor + 1u));
        } else {
            um &= um - 1u;
            if (um) WIDE_PUSH(e.x, (e.y & 0xffff0000u) | (um << 8));
        }
        if (cursor >= it.y || item >= W.n_units) { *guard = true; return false; }
        const uint32_t uu = __ldg(W.units + item);
        if (w.mode == TRACE_SHADOW && !(uu & WIDE_UNIT_BIT)) continue;
        const uint32_t u = uu & ~WIDE_UNIT_BIT;
        const uint32_t b = X.t_instances + u * 10u;
        if (u >= W.n_records || (uint64_t)b + 10u > S.n_table_vec4) { *guard = true; return false; }
        if (COUNT) wc->units++;
        const float4 m0 = tab(S, b), m1 = tab(S, b + 1), m2 = tab(S, b + 2);
        const float4 n0 = tab(S, b + 3), nn1 = tab(S, b + 4), n2 = tab(S, b + 5);
        w.rec = u;
        V3 ro = w.o - V3{m0.w, m1.w, m2.w};
        V3 rd = w.d, rinv = w.inv_d;
        if ((bu(nn1.w) & UNIT_SHIFTED) == 0) {
            ro = proc_dir(n0, nn1, n2, ro);
            rd = proc_dir(n0, nn1, n2, w.d);
            rinv = safe_inv(rd);
        }
        w.r = wide_ray(ro, rd, rinv);
        w.base = w.sp;
        w.node = __ldg(W.unit_root + u);
        return true;
    }
#undef WIDE_PUSH
}

// The whole walk of one ray (trt_trace's queries): the steps until it is over. A block has at most WIDE_BLOCK threads.
template <bool COUNT>
__device__ Hit trace_wide(const DScene& S, const WideView& W, const Sections& X, V3 o, V3 d, float tmax, uint32_t mode,
                          WalkCount* wc, bool* guard) {
    WideWalk w;
    if (blockDim.x > WIDE_BLOCK) { *guard = true; return Hit{tmax, MISS, 0.0f, 0.0f, NO_INST, 0u}; }
    if (!wide_begin(w, W, o, d, tmax, mode)) return w.hit;
    uint2 spill[WIDE_STACK - WIDE_SHORT];
    uint2* sh = wide_smem();
    while (wide_step<COUNT>(w, S, W, X, sh, spill, wc, guard)) {
    }
    return w.hit;
}

}  // namespace trt
