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
constexpr int WIDE_STACK = 64;

struct WideBvh {
    uint4* nodes = nullptr;
    float4* tris = nullptr;
    uint32_t* units = nullptr;
    uint32_t* unit_root = nullptr;
    WideView v{};
    bool built = false;
    uint32_t key[6] = {0, 0, 0, 0, 0, 0};  // the Params words the build read (it is redone when they change)
    double build_ms = 0.0;
    bool ready() const { return built; }
    WideView view() const { return v; }
    std::string error;
    // Builds (or keeps) the wide trees for the scene as `params` lays it out, from host copies of the scene's nodes,
    // leaves and tables (host[2], host[1], host[3]). 0, or 1 with `error` set.
    int ensure(const uint32_t* params, const std::vector<uint8_t>* host, cudaStream_t st);
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

// Byte k of w as a float (the conversion runs beside the walk's integer work, which keeps the ALU pipe busy).
__device__ __forceinline__ float q_float(uint32_t w, int k) { return __uint2float_rn((w >> (8 * k)) & 0xffu); }

// Visit order: slot i is visited k-th for i = k ^ oct. A node's byte arrays (one byte a slot, slots 0-3 in the low word)
// are put in that order with one byte permute a word: oct bit 0 swaps neighbouring bytes, bit 1 byte pairs, bit 2 the
// two words.
__device__ __forceinline__ void visit_order(uint32_t oct, uint32_t a, uint32_t b, uint32_t& x, uint32_t& y) {
    const uint32_t sel = (oct & 3u) == 0u ? 0x3210u : ((oct & 3u) == 1u ? 0x2301u : ((oct & 3u) == 2u ? 0x1032u : 0x0123u));
    uint32_t pa = __byte_perm(a, 0u, sel), pb = __byte_perm(b, 0u, sel);
    x = (oct & 4u) ? pb : pa;
    y = (oct & 4u) ? pa : pb;
}

// The eight child boxes of node `nd` against the ray, in visit order: tv[k] is the entry t of slot k ^ r.neg (INF:
// missed, or past tmax). A slot's plane at q steps is origin + q 2^e: t = q (2^e / d) + (origin - o) / d, one FMA.
// The near and far planes of each axis are picked once by the ray's signs; an empty slot (q_lo > q_hi) has its near
// plane past its far one on every axis, so it misses whatever the signs.
__device__ __forceinline__ void wide_children(const uint4 nd[5], const WideRay& r, float tmax, float tv[8]) {
    uint32_t eb = nd[0].w;
    float Sx = bf((eb & 0xffu) << 23) * r.inv.x, Sy = bf(((eb >> 8) & 0xffu) << 23) * r.inv.y,
          Sz = bf(((eb >> 16) & 0xffu) << 23) * r.inv.z;
    float Bx = (bf(nd[0].x) - r.o.x) * r.inv.x, By = (bf(nd[0].y) - r.o.y) * r.inv.y, Bz = (bf(nd[0].z) - r.o.z) * r.inv.z;
    // q_lo x: nd[2].x,y; y: nd[2].z,w; z: nd[3].x,y. q_hi x: nd[3].z,w; y: nd[4].x,y; z: nd[4].z,w.
    bool nx = r.neg & 1u, ny = r.neg & 2u, nz = r.neg & 4u;
    uint32_t nearx[2], farx[2], neary[2], fary[2], nearz[2], farz[2];
    visit_order(r.neg, nx ? nd[3].z : nd[2].x, nx ? nd[3].w : nd[2].y, nearx[0], nearx[1]);
    visit_order(r.neg, nx ? nd[2].x : nd[3].z, nx ? nd[2].y : nd[3].w, farx[0], farx[1]);
    visit_order(r.neg, ny ? nd[4].x : nd[2].z, ny ? nd[4].y : nd[2].w, neary[0], neary[1]);
    visit_order(r.neg, ny ? nd[2].z : nd[4].x, ny ? nd[2].w : nd[4].y, fary[0], fary[1]);
    visit_order(r.neg, nz ? nd[4].z : nd[3].x, nz ? nd[4].w : nd[3].y, nearz[0], nearz[1]);
    visit_order(r.neg, nz ? nd[3].x : nd[4].z, nz ? nd[3].y : nd[4].w, farz[0], farz[1]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        int h = k >> 2, j = k & 3;
        float x0 = fmaf(q_float(nearx[h], j), Sx, Bx), x1 = fmaf(q_float(farx[h], j), Sx, Bx);
        float y0 = fmaf(q_float(neary[h], j), Sy, By), y1 = fmaf(q_float(fary[h], j), Sy, By);
        float z0 = fmaf(q_float(nearz[h], j), Sz, Bz), z1 = fmaf(q_float(farz[h], j), Sz, Bz);
        float tnear = fmaxf(fmaxf(x0, y0), fmaxf(z0, 0.0f));
        float tfar = fminf(fminf(x1, y1), fminf(z1, tmax));
        tv[k] = tnear <= tfar ? tnear : INF;
    }
}

// Ascending sort of eight keys (a sorting network of 19 compare-exchanges).
__device__ __forceinline__ void cas(uint32_t& a, uint32_t& b) {
    uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}
__device__ __forceinline__ void sort8(uint32_t k[8]) {
    cas(k[0], k[2]); cas(k[1], k[3]); cas(k[4], k[6]); cas(k[5], k[7]);
    cas(k[0], k[4]); cas(k[1], k[5]); cas(k[2], k[6]); cas(k[3], k[7]);
    cas(k[0], k[1]); cas(k[2], k[3]); cas(k[4], k[5]); cas(k[6], k[7]);
    cas(k[2], k[4]); cas(k[3], k[5]);
    cas(k[1], k[4]); cas(k[3], k[6]);
    cas(k[1], k[2]); cas(k[3], k[4]); cas(k[5], k[6]);
}

// The walk over both levels: the top tree's hit leaves are units, entered (the ray in the unit's space, as
// trace_units.wgsl:86-105) when popped; a unit's walk ends when the stack is back to where it was entered. Entries
// carry the t they were hit at and are skipped once a closer hit is known.
template <bool COUNT>
__device__ Hit trace_wide(const DScene& S, const WideView& W, const Sections& X, V3 o, V3 d, float tmax, uint32_t mode,
                          WalkCount* wc, bool* guard) {
    Hit hit{tmax, MISS, 0.0f, 0.0f, NO_INST, 0u};
    if (W.n_units == 0) return hit;
    V3 inv_d = safe_inv(d);
    WideRay r = wide_ray(o, d, inv_d);
    uint32_t stack_ref[WIDE_STACK];
    float stack_t[WIDE_STACK];
    int sp = 0;
#define STACK_PUSH(ref, tt)                                   \
    do {                                                      \
        if (sp < WIDE_STACK) {                                \
            stack_ref[sp] = (ref);                            \
            stack_t[sp] = (tt);                               \
            sp++;                                             \
        }                                                     \
    } while (0)
    uint32_t cur = W.top_root;  // the node to open next (NO_INST: pop)
    uint32_t rec = NO_INST;
    int base = 0;
    for (uint32_t iter = 0;; ++iter) {
        if (iter >= WALK_GUARD) { *guard = true; break; }
        if (cur != NO_INST) {
            if (cur >= W.n_nodes) { *guard = true; break; }
            const uint4* np = W.nodes + 5ull * cur;
            uint4 nd[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) nd[k] = __ldg(np + k);
            if (COUNT) wc->nodes++;
            float tn[8];
            wide_children(nd, r, hit.t, tn);
            uint32_t imask = nd[0].w >> 24;
            uint32_t child_base = nd[1].x, leaf_base = nd[1].y;
            uint64_t counts = ((uint64_t)nd[1].w << 32) | nd[1].z;
            uint64_t prefix = counts * 0x0101010101010101ull;  // byte i: the items of slots 0..i
            // The visit order: for closest hits the hit slots sorted by their entry t; for any-hit rays (shadow
            // rays stop at the first hit, whichever) the octant order k ^ (the ray's signs), nearly front to back
            // as the builder put children by octant. order[j]: visit index of the j-th slot to visit (9: none).
            uint32_t oct = r.neg;
            uint32_t key[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) key[k] = tn[k] >= hit.t ? 0xffffffffu : ((bu(tn[k]) & ~7u) | (uint32_t)k);
            if (mode == TRACE_CLOSEST) {
                uint32_t hits = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k) hits += key[k] != 0xffffffffu;
                if (hits > 1) sort8(key);
                else if (hits == 1) {
                    // (One hit: move it first.)
                    uint32_t m = key[0];
#pragma unroll
                    for (int k = 1; k < 8; ++k) m = min(m, key[k]);
                    key[0] = m;
#pragma unroll
                    for (int k = 1; k < 8; ++k) key[k] = 0xffffffffu;
                }
            }
            // Leaves first (their hits cull the farther entries), then the other entries pushed farthest first,
            // so the nearest is on top.
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (key[j] == 0xffffffffu) continue;
                uint32_t i = (key[j] & 7u) ^ oct;
                if (imask & (1u << i)) continue;
                if (bf(key[j] & ~7u) >= hit.t) continue;
                uint32_t cnt = (uint32_t)(counts >> (8 * i)) & 0xffu;
                if (cnt == 0 || rec == NO_INST) continue;  // (top-tree leaves are units: entries, below)
                uint32_t item = leaf_base + ((uint32_t)(prefix >> (8 * i)) & 0xffu) - cnt;
                for (uint32_t q = 0; q < cnt; ++q) {
                    uint32_t ti = item + q;
                    if (ti >= W.n_tris) { *guard = true; return hit; }
                    const float4* tp = W.tris + 3ull * ti;
                    float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
                    if (COUNT) wc->tris++;
                    // pathtrace.wgsl:742-761 intersect_tri, on the copy of the reference's leaf record.
                    V3 v0 = xyz(a), e1 = xyz(b), e2 = xyz(c);
                    V3 pv = cross(r.d, e2);
                    float det = dot(e1, pv);
                    if (fabsf(det) < 1e-12f) continue;
                    float inv = 1.0f / det;
                    V3 tv = r.o - v0;
                    float u = dot(tv, pv) * inv;
                    if (u < 0.0f || u > 1.0f) continue;
                    V3 qv = cross(tv, e1);
                    float v = dot(r.d, qv) * inv;
                    if (v < 0.0f || u + v > 1.0f) continue;
                    float t = dot(e2, qv) * inv;
                    if (t <= 0.0f || t >= hit.t) continue;
                    hit = Hit{t, bu(c.w), u, v, rec, bu(a.w)};
                    if (mode != TRACE_CLOSEST) return hit;
                }
            }
#pragma unroll
            for (int j = 7; j >= 0; --j) {
                if (key[j] == 0xffffffffu) continue;
                float t = bf(key[j] & ~7u);
                if (t >= hit.t) continue;
                uint32_t i = (key[j] & 7u) ^ oct;
                if (imask & (1u << i)) {
                    STACK_PUSH(child_base + (uint32_t)__popc(imask & ((1u << i) - 1u)), t);
                } else if (rec == NO_INST) {
                    uint32_t cnt = (uint32_t)(counts >> (8 * i)) & 0xffu;
                    uint32_t item = leaf_base + ((uint32_t)(prefix >> (8 * i)) & 0xffu) - cnt;
                    if (COUNT) wc->units += cnt;
                    for (uint32_t q = 0; q < cnt; ++q) {
                        if (item + q >= W.n_units) { *guard = true; return hit; }
                        uint32_t u = __ldg(W.units + item + q);
                        if (mode == TRACE_SHADOW && !(u & WIDE_UNIT_BIT)) continue;
                        STACK_PUSH(u | WIDE_UNIT_BIT, t);
                    }
                }
            }
        }
        // Pop: the nearest pending entry still in front of the closest hit.
        for (;;) {
            if (rec != NO_INST && sp == base) {
                rec = NO_INST;
                r = wide_ray(o, d, inv_d);
            }
            if (sp == 0) return hit;
            --sp;
            if (stack_t[sp] < hit.t) break;
        }
        uint32_t e = stack_ref[sp];
        if (e & WIDE_UNIT_BIT) {
            uint32_t u = e & ~WIDE_UNIT_BIT;
            uint32_t b = X.t_instances + u * 10u;
            if (u >= W.n_records || (uint64_t)b + 10u > S.n_table_vec4) { *guard = true; break; }
            float4 m0 = tab(S, b), m1 = tab(S, b + 1), m2 = tab(S, b + 2);
            float4 n0 = tab(S, b + 3), n1 = tab(S, b + 4), n2 = tab(S, b + 5);
            rec = u;
            V3 ro = o - V3{m0.w, m1.w, m2.w};
            V3 rd = d;
            V3 rinv = inv_d;
            if ((bu(n1.w) & UNIT_SHIFTED) == 0) {
                ro = proc_dir(n0, n1, n2, ro);
                rd = proc_dir(n0, n1, n2, d);
                rinv = safe_inv(rd);
            }
            r = wide_ray(ro, rd, rinv);
            base = sp;
            cur = __ldg(W.unit_root + u);
        } else {
            cur = e;
        }
    }
    return hit;
#undef STACK_PUSH
}

}  // namespace trt
