// Software traversal over the reference's own two-level binary trees (renderer/shaders/trace_units.wgsl:44-135):
// the top tree over the units' world boxes, each unit's mesh tree in its model space, one loop over both levels.
// It is the pass's walk (faster on B200 than the wide-BVH walk of wide_bvh.cuh, which TRT_RENDER_WIDE selects), in
// two forms with the same nodes, tests and results a ray: trace_binary's single loop, and trace_binary_split's loop
// split into interior nodes and leaves.
#pragma once
#include "device_common.cuh"

namespace trt {

struct Hit { float t; uint32_t tri; float u, v; uint32_t inst, part; };

struct Node { V3 bmin; uint32_t left_or_first; V3 bmax; uint32_t count; };
__device__ __forceinline__ Node node_at(const DScene& S, uint32_t i) {
    uint4 a = __ldg(S.nodes + 2ull * i), b = __ldg(S.nodes + 2ull * i + 1);
    return {{bf(a.x), bf(a.y), bf(a.z)}, a.w, {bf(b.x), bf(b.y), bf(b.z)}, b.w};
}

// Three-input minimum and maximum (one instruction each on sm_100; exact, like two fminf / fmaxf).
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// pathtrace.wgsl:732-739 ray_aabb (min and max are exact, so grouping them three at a time rounds nothing)
__device__ __forceinline__ float ray_aabb(V3 o, V3 inv_d, V3 bmin, V3 bmax, float tmax) {
    V3 t0 = (bmin - o) * inv_d;
    V3 t1 = (bmax - o) * inv_d;
    V3 tmin_v = vmin(t0, t1);
    V3 tmax_v = vmax(t0, t1);
    float tn = max3f(tmin_v.x, tmin_v.y, fmaxf(tmin_v.z, 0.0f));
    float tf = min3f(tmax_v.x, tmax_v.y, fminf(tmax_v.z, tmax));
    return tn <= tf ? tn : INF;
}

// pathtrace.wgsl:742-761 intersect_tri (Moller-Trumbore on the leaf's v0, e1, e2), t = INF for none.
__device__ __forceinline__ float3 intersect_tri(const DScene& S, V3 o, V3 d, uint32_t i, float tmax) {
    float4 a = __ldg(S.leaves + 3ull * i), b = __ldg(S.leaves + 3ull * i + 1), c = __ldg(S.leaves + 3ull * i + 2);
    V3 v0 = xyz(a), e1 = xyz(b), e2 = xyz(c);
    V3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (fabsf(det) < 1e-12f) return make_float3(INF, 0.0f, 0.0f);
    float inv = 1.0f / det;
    V3 tv = o - v0;
    float u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return make_float3(INF, 0.0f, 0.0f);
    V3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return make_float3(INF, 0.0f, 0.0f);
    float t = dot(e2, qv) * inv;
    if (t <= 0.0f || t >= tmax) return make_float3(INF, 0.0f, 0.0f);
    return make_float3(t, u, v);
}

// pathtrace.wgsl:661 proc_dir: world -> a record's model space by its normal rows.
__device__ __forceinline__ V3 proc_dir(const float4& n0, const float4& n1, const float4& n2, V3 d) {
    return xyz(n0) * d.x + xyz(n1) * d.y + xyz(n2) * d.z;
}
__device__ __forceinline__ V3 safe_inv(V3 d) {
    V3 s = {fabsf(d.x) < 1e-20f ? 1e-20f : d.x, fabsf(d.y) < 1e-20f ? 1e-20f : d.y, fabsf(d.z) < 1e-20f ? 1e-20f : d.z};
    return V3{1.0f / s.x, 1.0f / s.y, 1.0f / s.z};
}

struct WalkCount { uint32_t nodes, tris, units; };

// The loop guard (renderer/src/gpu.rs:1214-1285 guard_loops): a walk that has not ended after this many nodes stops,
// sets *guard and returns what it has; the render then reports an error instead of hanging on trees that are not
// trees.
constexpr uint32_t WALK_GUARD = 1u << 20;

// trace_units.wgsl:44-135, with a 64-entry stack of its own. Returns the hit (tri MISS for none).
template <bool COUNT>
__device__ Hit trace_binary(const DScene& S, const Sections& X, uint32_t top, uint32_t n_units, V3 o, V3 d, float tmax,
                            uint32_t mode, WalkCount* wc, bool* guard) {
    Hit hit{tmax, MISS, 0.0f, 0.0f, NO_INST, 0u};
    if (n_units == 0) return hit;
    if (top >= S.n_nodes) { *guard = true; return hit; }
    V3 inv_d = safe_inv(d);
    Node whole = node_at(S, top);
    if (COUNT) wc->nodes++;
    if (ray_aabb(o, inv_d, whole.bmin, whole.bmax, hit.t) == INF) return hit;
    uint32_t stack[64];
    uint32_t sp = 0, node = top, rec = NO_INST;
    V3 ro = o, rd = d, rinv = inv_d;
    uint32_t off = top, first = 0, base = 0;
    for (uint32_t iter = 0;; ++iter) {
        // (Every index a walk follows is checked: a bad tree ends the walk with the guard set, never a fault.)
        if (iter >= WALK_GUARD || node >= S.n_nodes) { *guard = true; break; }
        Node n = node_at(S, node);
        if (COUNT) wc->nodes++;
        if (n.count == 0) {
            uint32_t l = off + n.left_or_first, r = l + 1;
            if (r >= S.n_nodes) { *guard = true; break; }
            Node nl = node_at(S, l), nr = node_at(S, r);
            if (COUNT) wc->nodes += 2;
            float tl = ray_aabb(ro, rinv, nl.bmin, nl.bmax, hit.t);
            float tr = ray_aabb(ro, rinv, nr.bmin, nr.bmax, hit.t);
            if (tl != INF || tr != INF) {
                uint32_t nearn = l, farn = r;
                if (tr < tl) { nearn = r; farn = l; float tmp = tl; tl = tr; tr = tmp; }
                node = nearn;
                if (tr != INF && sp < 64) stack[sp++] = farn;
                continue;
            }
        } else if (rec == NO_INST) {
            uint32_t b = X.t_instances + n.left_or_first * 10u;
            if ((uint64_t)b + 10u > S.n_table_vec4) { *guard = true; break; }
            float4 n1 = tab(S, b + 4);
            uint32_t ubits = bu(n1.w);
            if (COUNT) wc->units++;
            if (mode != TRACE_SHADOW || (ubits & UNIT_SHADOW) != 0) {
                float4 m0 = tab(S, b), m1 = tab(S, b + 1), m2 = tab(S, b + 2), n0 = tab(S, b + 3), n2 = tab(S, b + 5);
                uint4 info = tabu(S, b + 6);
                rec = n.left_or_first;
                ro = o - V3{m0.w, m1.w, m2.w};
                if ((ubits & UNIT_SHIFTED) == 0) {
                    ro = proc_dir(n0, n1, n2, ro);
                    rd = proc_dir(n0, n1, n2, d);
                    rinv = safe_inv(rd);
                }
                off = bu(n0.w);
                first = info.x;
                base = sp;
                node = off;
                continue;
            }
        } else {
            for (uint32_t k = 0; k < n.count; ++k) {
                uint32_t ti = first + n.left_or_first + k;
                if (ti >= S.n_tris) { *guard = true; return hit; }
                if (COUNT) wc->tris++;
                float3 x = intersect_tri(S, ro, rd, ti, hit.t);
                if (x.x < hit.t) {
                    uint32_t part = bu(__ldg(S.leaves + 3ull * ti).w);
                    hit = Hit{x.x, ti, x.y, x.z, rec, part};
                    if (mode != TRACE_CLOSEST) return hit;
                }
            }
        }
        if (rec != NO_INST && sp == base) {
            rec = NO_INST;
            ro = o; rd = d; rinv = inv_d;
            off = top;
        }
        if (sp == 0) break;
        sp--;
        node = stack[sp];
    }
    return hit;
}

// The same walk with its loop split in two (Aila and Laine's "while-while"): interior nodes in an inner loop until a
// leaf, then the leaf. A ray's nodes, tests, pops and result are trace_binary's; only the lanes of a warp fall into
// step differently. Measured on B200 (the city frame): the shadow walks 6 % faster with it (2.49 -> 2.33 ms a
// frame, compiled for 8 blocks an SM); the closest-hit walk 4.6 % slower with it on every depth but 2 % faster on
// the depths past the camera's rays, so the shadow walks and the closest-hit walks past depth 0 use this one.
template <bool COUNT>
__device__ Hit trace_binary_split(const DScene& S, const Sections& X, uint32_t top, uint32_t n_units, V3 o, V3 d, float tmax,
                            uint32_t mode, WalkCount* wc, bool* guard) {
    Hit hit{tmax, MISS, 0.0f, 0.0f, NO_INST, 0u};
    if (n_units == 0) return hit;
    if (top >= S.n_nodes) { *guard = true; return hit; }
    V3 inv_d = safe_inv(d);
    Node whole = node_at(S, top);
    if (COUNT) wc->nodes++;
    if (ray_aabb(o, inv_d, whole.bmin, whole.bmax, hit.t) == INF) return hit;
    uint32_t stack[64];
    uint32_t sp = 0, node = top, rec = NO_INST;
    V3 ro = o, rd = d, rinv = inv_d;
    uint32_t off = top, first = 0, base = 0;
    uint32_t iter = 0;
    // The pop after a node that leads nowhere: out of a unit whose subtree is done, then the next node (false: the walk
    // is over).
#define TRT_WALK_POP()                        \
    (((rec != NO_INST && sp == base)          \
          ? (rec = NO_INST, ro = o, rd = d, rinv = inv_d, off = top, 0) \
          : 0),                               \
     sp == 0 ? false : (node = stack[--sp], true))
    for (;;) {
        // Interior nodes first, until a leaf (a unit's record or a mesh's triangles); the nodes, tests and pops are
        // the single loop's, in the same order.
        Node n;
        for (;; ++iter) {
            // (Every index a walk follows is checked: a bad tree ends the walk with the guard set, never a fault.)
            if (iter >= WALK_GUARD || node >= S.n_nodes) { *guard = true; return hit; }
            n = node_at(S, node);
            if (COUNT) wc->nodes++;
            if (n.count != 0) break;
            uint32_t l = off + n.left_or_first, r = l + 1;
            if (r >= S.n_nodes) { *guard = true; return hit; }
            Node nl = node_at(S, l), nr = node_at(S, r);
            if (COUNT) wc->nodes += 2;
            float tl = ray_aabb(ro, rinv, nl.bmin, nl.bmax, hit.t);
            float tr = ray_aabb(ro, rinv, nr.bmin, nr.bmax, hit.t);
            if (tl != INF || tr != INF) {
                uint32_t nearn = l, farn = r;
                if (tr < tl) { nearn = r; farn = l; float tmp = tl; tl = tr; tr = tmp; }
                node = nearn;
                if (tr != INF && sp < 64) stack[sp++] = farn;
                continue;
            }
            if (!TRT_WALK_POP()) return hit;
        }
        ++iter;
        if (rec == NO_INST) {
            uint32_t b = X.t_instances + n.left_or_first * 10u;
            if ((uint64_t)b + 10u > S.n_table_vec4) { *guard = true; return hit; }
            float4 n1 = tab(S, b + 4);
            uint32_t ubits = bu(n1.w);
            if (COUNT) wc->units++;
            if (mode != TRACE_SHADOW || (ubits & UNIT_SHADOW) != 0) {
                float4 m0 = tab(S, b), m1 = tab(S, b + 1), m2 = tab(S, b + 2), n0 = tab(S, b + 3), n2 = tab(S, b + 5);
                uint4 info = tabu(S, b + 6);
                rec = n.left_or_first;
                ro = o - V3{m0.w, m1.w, m2.w};
                if ((ubits & UNIT_SHIFTED) == 0) {
                    ro = proc_dir(n0, n1, n2, ro);
                    rd = proc_dir(n0, n1, n2, d);
                    rinv = safe_inv(rd);
                }
                off = bu(n0.w);
                first = info.x;
                base = sp;
                node = off;
                continue;
            }
        } else {
            for (uint32_t k = 0; k < n.count; ++k) {
                uint32_t ti = first + n.left_or_first + k;
                if (ti >= S.n_tris) { *guard = true; return hit; }
                if (COUNT) wc->tris++;
                float3 x = intersect_tri(S, ro, rd, ti, hit.t);
                if (x.x < hit.t) {
                    uint32_t part = bu(__ldg(S.leaves + 3ull * ti).w);
                    hit = Hit{x.x, ti, x.y, x.z, rec, part};
                    if (mode != TRACE_CLOSEST) return hit;
                }
            }
        }
        if (!TRT_WALK_POP()) break;
    }
#undef TRT_WALK_POP
    return hit;
}

}  // namespace trt
