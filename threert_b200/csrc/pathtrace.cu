// The path-trace pass as a wavefront of sm_100a kernels, and the C ABI around it (include/threert_cuda.h).
//
// The reference runs one megakernel invocation per pixel per sample (renderer/shaders/pathtrace.wgsl:4105-4558,
// dispatched per sample by renderer/src/gpu.rs:4174-4196). Here a wave is every pixel for K samples at once, and each
// path vertex is four kernels over compacted queues:
//   extend  - closest hit of every live path's ray (persistent threads fetching warps of rays);
//   shade   - surface, emission with its MIS weight, the vertex's light samples (sun, emitter, sky) as shadow rays
//             with their unoccluded contributions, the BSDF sample and Russian roulette; live paths go to the next
//             queue (warp-aggregated appends);
//   shadow  - any-hit of every shadow ray, a visibility bit per light slot;
//   resolve - the vertex's direct light from the visible slots, in the reference's order and with its clamp, then
//             the finished paths' last fixes.
// Every random number is keyed by (pixel, sample, vertex, decision) (sample.wgsl), so nothing a path draws depends on
// how the wave is scheduled, and a path's floating-point sums are taken in the megakernel's order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "deform.h"

// Resident blocks of 128 an SM the walks and the shading are compiled for (their register budgets: 64 a thread each).
// Measured on the city frame: the extend walk 3 % faster than at 6 blocks (72 registers, no spills), 2.6 % faster
// than at 7 (70, no spills; both of its loops compiled in) and 6 % faster than at 9 (56); the split shadow walk (trace_binary_split) 5 % faster at 8 than at 7 (67 registers), 3 % faster
// than at 9 and 9 % faster than at 10; the shading, latency-bound, 2.5 % faster at 8 blocks than at 6 (80
// registers), its spills notwithstanding, and no faster at 10 (48).
#ifndef TRT_BLOCKS_EXTEND
#define TRT_BLOCKS_EXTEND 8
#endif
#ifndef TRT_BLOCKS_SHADOW
#define TRT_BLOCKS_SHADOW 8
#endif
#ifndef TRT_BLOCKS_SHADE
#define TRT_BLOCKS_SHADE 8
#endif
// The closest-hit walk's loop (see trace_binary_split): 0 single, 1 split, 2 split past the camera's rays (the
// default: measured on the city, split everywhere the extend walk is 4.6 % slower, split past depth 0 2 % faster; the
// camera's coherent rays keep the single loop).
#ifndef TRT_SPLIT_CLOSEST
#define TRT_SPLIT_CLOSEST 2
#endif
#include "sky.h"
#include "unet.h"
#include "shade.cuh"
#include "denoise.cuh"
#include "threert_cuda.h"
#include "wide_bvh.cuh"

namespace trt {

// ---- path state -----------------------------------------------------------------------------------------------------

constexpr uint32_t F_SPECULAR_BOUNCE = 1u, F_STRAIGHT = 2u, F_MIRROR = 4u, F_DONE = 8u;
constexpr uint32_t MAX_DIR_LIGHTS = 4u;
constexpr uint32_t SLOT_EMIT = MAX_DIR_LIGHTS, SLOT_ENV = MAX_DIR_LIGHTS + 1, N_SLOTS = MAX_DIR_LIGHTS + 2;
constexpr uint32_t MAX_DEPTH = 64u;            // counters are kept for this many vertices

struct PathBufs {
    float4* o;        // origin, w: last_pdf
    float4* d;        // direction, w: flags (bits)
    float4* thr;      // throughput, w: pixel (bits)
    float4* rad;      // radiance, w: sample (bits)
    float4* alb;      // first-hit albedo
    float4* nrm;      // first-hit normal
    float4* mis_x;    // the last light-sampling vertex's point
    float4* mis_n;    // and normal
    float4* nee;      // N_SLOTS contributions a path (slot-major: nee[slot * n + p])
    float4* nee_thr;  // throughput at the light samples, w: slot mask | clamp << 8 (bits)
    uint32_t* vis;    // visible slots (bits)
    uint32_t* job;    // the job (index into the wave's job table) whose path a slot holds
    uint32_t n;       // slots
};
struct Queues {
    uint32_t* q[2];       // path queues (extend inputs), alternating by depth
    uint32_t* qx;         // a depth's queue sorted (a third buffer, so the two above stay the raw queues)
    float4* hit_a;        // t, u, v, tri (bits) per path
    uint2* hit_b;         // inst, part
    float4* so;           // shadow rays: origin, tmax
    float4* sd;           // direction, mode (bits)
    uint32_t* sp;         // path << 3 | slot
    uint32_t* cnt;        // per depth, CNT_STRIDE words: queue size, -, extend fetch, shadow fetch, then the shadow
                          // rays of each light class (sun, emitter, sky)
    unsigned long long* totals;
    uint2* sort_kr;       // the coherence sort: each item's key and its rank among the key's items
    uint32_t* sort_hist;  // SORT_BINS counts (zero between sorts)
    uint32_t* sort_start; // SORT_BINS starts
    uint32_t* sort_done;  // blocks of the count kernel that have finished (zero between sorts)
    uint32_t* perm;       // the shadow rays' order after their sort: perm[j] is the j-th ray's slot in so / sd / sp
    uint32_t shadow_cap;  // the three classes' regions together
    uint32_t class_base[3], class_cap[3];  // each class's region of so / sd / sp
};
// Counter words a depth: [0] paths in the extend queue, [2] extend fetch, [3] shadow fetch, [4 + c] shadow rays of
// light class c. Shadow rays are queued by class, so a warp of the shadow walk holds rays toward one kind of light
// (the sun's are nearly parallel).
constexpr uint32_t CNT_STRIDE = 8u;
constexpr uint32_t CLASS_SUN = 0u, CLASS_EMIT = 1u, CLASS_ENV = 2u;
// Cumulative counters: rays, paths, guard trips, and (TRT_RENDER_COUNT) the walks' reads by stage: node records
// read, triangles tested, unit records entered, for the extend (closest) and the shadow walks.
enum { T_CLOSEST = 0, T_SHADOW, T_PATHS, T_GUARD, T_E_NODES, T_E_TRIS, T_E_UNITS, T_S_NODES, T_S_TRIS, T_S_UNITS, T_COUNT };

// Warp-aggregated append: one atomic per warp for the lanes whose `want` is set; returns each lane's slot.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
    unsigned mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return 0;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}
// The same for lanes in divergent code: the lanes that are here together take consecutive slots.
__device__ __forceinline__ uint32_t warp_append_active(uint32_t* counter) {
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}
// Persistent-thread work fetch: a warp takes 32 consecutive items.
__device__ __forceinline__ uint32_t warp_fetch(uint32_t* counter) {
    uint32_t base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(counter, 32u);
    return __shfl_sync(0xffffffffu, base, 0) + (threadIdx.x & 31);
}
__device__ __forceinline__ void warp_add64(unsigned long long* p, unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(p, v);
}

// The slot -> pixel map: 8 x 4 tiles in rows, so a warp's paths start from one tile.
__device__ __forceinline__ bool slot_pixel(uint32_t idx, uint32_t w, uint32_t h, uint32_t& gx, uint32_t& gy) {
    uint32_t tiles_x = (w + 7u) / 8u;
    uint32_t t = idx / 32u, within = idx % 32u;
    gx = (t % tiles_x) * 8u + (within % 8u);
    gy = (t / tiles_x) * 4u + (within / 8u);
    return gx < w && gy < h;
}

struct Walk {
    DScene S;
    WideView W;
    uint32_t top, n_units;
};

// A wave's unit of work: one request's samples [first_sample, first_sample + K) of every pixel of its image, on the
// wave's slots [slot_first, slot_first + n_idx * K), with its own Params, scene and accum. trt_render's waves hold one
// job; a wave may hold several requests' (of different scenes, sizes and sample counts) in the same launches. A path
// finds its job through B.job, so nothing a path computes depends on what else the wave holds.
struct Job {
    Params P;
    Walk wk;
    float4* accum;
    uint32_t slot_first, n_idx, K, first_sample;
    uint32_t idx_first;  // the earlier jobs' n_idx summed: its pixels' place in a pass over every job's pixels
    uint32_t depth;      // 1: accumulate the first hit's distance into the Pixel's fourth vec4 (TRT_RENDER_DEPTH)
    uint32_t pix_first;  // the first of the image's pixel indices (8 x 4 tiles) the job's n_idx slots a sample take
};
// What a wave of a server step holds, in device memory ahead of its job table, so that the step's launches (and a
// graph captured from them) do not change from step to step.
struct StepHead { uint32_t n_jobs, paths, pad0, pad1; };
constexpr uint32_t MAX_JOBS = 64u;
// The hot kernels take the table and, for a wave of one job, that job as a kernel argument (MULTI = false): its reads
// then come from the kernel's constant bank, not global memory.

// Writes one entry of a wave's job table from a kernel argument (no host copy: the launch carries it).
__global__ void k_put_job(Job j, Job* table, uint32_t at) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&j);
    uint32_t* dst = reinterpret_cast<uint32_t*>(table + at);
    for (uint32_t i = threadIdx.x; i < sizeof(Job) / 4; i += blockDim.x) dst[i] = src[i];
}

// pathtrace.wgsl:4002-4026 camera_ray
__device__ void camera_ray(const Params& P, uint32_t gx, uint32_t gy, const float cam[4], V3& o, V3& d) {
    float w = (float)P.w[P_SIZE], h = (float)P.w[P_SIZE + 1];
    float ndcx = ((float)gx + cam[0]) / w * 2.0f - 1.0f;
    float ndcy = 1.0f - ((float)gy + cam[1]) / h * 2.0f;
    V3 fwd = pv(P, P_CAM_FWD), right = pv(P, P_CAM_RIGHT), up = pv(P, P_CAM_UP);
    float tanf_ = pf(P, P_CAM_POS + 3), aspect = pf(P, P_CAM_FWD + 3);
    d = normalize(fwd + right * (ndcx * tanf_ * aspect) + up * (ndcy * tanf_));
    o = pv(P, P_CAM_POS);
    if (pf(P, P_CAM_RIGHT + 3) > 0.0f) {
        V3 focus = o + d * (pf(P, P_CAM_UP + 3) / dot(d, fwd));
        float r = sqrtf(cam[2]) * pf(P, P_CAM_RIGHT + 3);
        float phi = 2.0f * PI * cam[3];
        o = o + right * (r * cosf(phi)) + up * (r * sinf(phi));
        d = normalize(focus - o);
    }
}

__global__ void k_raygen(const Job* __restrict__ jobs, uint32_t n_jobs, PathBufs B, Queues Q, uint32_t n_slots,
                         const StepHead* __restrict__ head) {
    if (head) n_jobs = head->n_jobs;
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = false;
    uint32_t gx = 0, gy = 0, j = 0;
    if (p < n_slots) {
        while (j + 1 < n_jobs && p >= jobs[j + 1].slot_first) ++j;  // jobs lie in slot order
        const Job& J = jobs[j];
        uint32_t local = p - J.slot_first;
        if (local < J.n_idx * J.K)
            valid = slot_pixel(local % J.n_idx + J.pix_first, J.P.w[P_SIZE], J.P.w[P_SIZE + 1], gx, gy);
    }
    uint32_t at = warp_append(&Q.cnt[0], valid);
    if (!valid) return;
    const Job& J = jobs[j];
    const Params& P = J.P;
    uint32_t w = P.w[P_SIZE];
    B.job[p] = j;
    uint32_t sample = J.first_sample + (p - J.slot_first) / J.n_idx;
    Rng R{sample, pixel_seed(gx, gy, P.w[P_SIZE + 3]), 0u};
    float cam[4];
    R.rng4(R.dim(D_CAMERA), cam);
    V3 o, d;
    camera_ray(P, gx, gy, cam, o, d);
    B.o[p] = f4(o, 0.0f);
    B.d[p] = f4(d, bf(F_SPECULAR_BOUNCE | F_STRAIGHT));
    B.thr[p] = f4(v3(1.0f), bf(gy * w + gx));
    B.rad[p] = f4(v3(0.0f), bf(sample));
    B.alb[p] = f4(v3(0.0f), 0.0f);
    B.nrm[p] = f4(v3(0.0f), 0.0f);
    B.mis_x[p] = f4(v3(0.0f), 0.0f);
    B.mis_n[p] = f4(v3(0.0f), 0.0f);
    B.nee_thr[p] = f4(v3(0.0f), bf(0u));
    Q.q[0][at] = p;
}

// SPLIT: the binary walk with its loop split (trace_binary_split), which the shadow walks use.
template <bool COUNT, bool WIDE, bool SPLIT = false>
__device__ __forceinline__ Hit walk(const Walk& wk, const Sections& X, V3 o, V3 d, float tmax, uint32_t mode,
                                    WalkCount* wc, bool* guard) {
    if (WIDE) return trace_wide<COUNT>(wk.S, wk.W, X, o, d, tmax, mode, wc, guard);
    if (SPLIT) return trace_binary_split<COUNT>(wk.S, X, wk.top, wk.n_units, o, d, tmax, mode, wc, guard);
    return trace_binary<COUNT>(wk.S, X, wk.top, wk.n_units, o, d, tmax, mode, wc, guard);
}

template <bool COUNT, bool WIDE, bool MULTI>
__global__ void __launch_bounds__(128, TRT_BLOCKS_EXTEND) k_extend(const Job* __restrict__ jobs, const Job one, PathBufs B, Queues Q,
                                                   uint32_t depth, const uint32_t* __restrict__ queue) {
    uint32_t* cnt = Q.cnt + depth * CNT_STRIDE;
    uint32_t n = *(volatile uint32_t*)&cnt[0];
    WalkCount wc{0, 0, 0};
    unsigned long long guard_trips = 0;
    for (;;) {
        uint32_t i = warp_fetch(&cnt[2]);
        if (__shfl_sync(0xffffffffu, i, 0) >= n) break;
        if (i < n) {
            uint32_t p = queue[i];
            const Job& J = MULTI ? jobs[B.job[p]] : one;
            Sections X(J.P);
            float4 o = B.o[p], d = B.d[p];
            bool guard = false;
            Hit h = (TRT_SPLIT_CLOSEST == 1 || (TRT_SPLIT_CLOSEST == 2 && depth > 0))
                        ? walk<COUNT, WIDE, true>(J.wk, X, xyz(o), xyz(d), INF, TRACE_CLOSEST, &wc, &guard)
                        : walk<COUNT, WIDE, false>(J.wk, X, xyz(o), xyz(d), INF, TRACE_CLOSEST, &wc, &guard);
            if (guard) guard_trips++;
            Q.hit_a[p] = make_float4(h.t, h.u, h.v, bf(h.tri));
            Q.hit_b[p] = make_uint2(h.inst, h.part);
        }
    }
    if (COUNT) {
        warp_add64(&Q.totals[T_E_NODES], wc.nodes);
        warp_add64(&Q.totals[T_E_TRIS], wc.tris);
        warp_add64(&Q.totals[T_E_UNITS], wc.units);
    }
    warp_add64(&Q.totals[T_GUARD], guard_trips);
}

// The j-th shadow ray of a depth, counting the classes' regions one after another.
__device__ __forceinline__ uint32_t shadow_slot(const Queues& Q, uint32_t j, uint32_t n0, uint32_t n1) {
    return j < n0 ? Q.class_base[0] + j : (j < n0 + n1 ? Q.class_base[1] + (j - n0) : Q.class_base[2] + (j - n0 - n1));
}

template <bool COUNT, bool WIDE, bool MULTI>
__global__ void __launch_bounds__(128, TRT_BLOCKS_SHADOW) k_shadow(const Job* __restrict__ jobs, const Job one, PathBufs B, Queues Q,
                                                   uint32_t depth, const uint32_t* __restrict__ perm) {
    uint32_t* cnt = Q.cnt + depth * CNT_STRIDE;
    uint32_t n0 = min(*(volatile uint32_t*)&cnt[4], Q.class_cap[0]);
    uint32_t n1 = min(*(volatile uint32_t*)&cnt[5], Q.class_cap[1]);
    uint32_t n2 = min(*(volatile uint32_t*)&cnt[6], Q.class_cap[2]);
    uint32_t n = n0 + n1 + n2;
    WalkCount wc{0, 0, 0};
    unsigned long long guard_trips = 0;
    for (;;) {
        uint32_t j = warp_fetch(&cnt[3]);
        if (__shfl_sync(0xffffffffu, j, 0) >= n) break;
        if (j < n) {
            // The classes' regions one after another: the j-th ray of the three (or of their sorted order).
            uint32_t i = perm ? perm[j] : shadow_slot(Q, j, n0, n1);
            uint32_t sp = Q.sp[i];
            const Job& J = MULTI ? jobs[B.job[sp >> 3]] : one;
            Sections X(J.P);
            float4 o = Q.so[i], d = Q.sd[i];
            bool guard = false;
            Hit h = walk<COUNT, WIDE, true>(J.wk, X, xyz(o), xyz(d), o.w, bu(d.w), &wc, &guard);
            if (guard) guard_trips++;
            if (h.tri == MISS) atomicOr(&B.vis[sp >> 3], 1u << (sp & 7u));
        }
    }
    if (COUNT) {
        warp_add64(&Q.totals[T_S_NODES], wc.nodes);
        warp_add64(&Q.totals[T_S_TRIS], wc.tris);
        warp_add64(&Q.totals[T_S_UNITS], wc.units);
    }
    warp_add64(&Q.totals[T_GUARD], guard_trips);
}

__device__ __forceinline__ void push_shadow(const Queues& Q, uint32_t* cnt, uint32_t cls, uint32_t p, uint32_t slot, V3 o,
                                            V3 d, float tmax, uint32_t mode) {
    uint32_t at = warp_append_active(&cnt[4 + cls]);
    if (at >= Q.class_cap[cls]) return;
    at += Q.class_base[cls];
    Q.so[at] = f4(o, tmax);
    Q.sd[at] = f4(d, bf(mode));
    Q.sp[at] = (p << 3) | slot;
}

// One path vertex: pathtrace.wgsl:4176-4477 from the hit on (the trace itself is k_extend's).
template <bool MULTI>
__global__ void __launch_bounds__(128, TRT_BLOCKS_SHADE) k_shade(const Job* __restrict__ jobs, const Job one, PathBufs B, Queues Q,
                                                  uint32_t depth, const uint32_t* __restrict__ queue,
                                                  uint32_t* __restrict__ next) {
    uint32_t* cnt = Q.cnt + depth * CNT_STRIDE;
    uint32_t n = cnt[0];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = false;
    uint32_t p = 0;
    if (i < n) {
        p = queue[i];
        const Job& J = MULTI ? jobs[B.job[p]] : one;
        const Params& P = J.P;
        const DScene& S = J.wk.S;
        Sections X(P);
        float4 o4 = B.o[p], d4 = B.d[p], thr4 = B.thr[p], rad4 = B.rad[p];
        V3 o = xyz(o4), d = xyz(d4), thr = xyz(thr4), radiance = xyz(rad4);
        float last_pdf = o4.w;
        uint32_t flags = bu(d4.w);
        uint32_t pix = bu(thr4.w), sample = bu(rad4.w);
        uint32_t w = P.w[P_SIZE];
        Rng R{sample, pixel_seed(pix % w, pix / w, P.w[P_SIZE + 3]), depth};
        float clamp_v = pf(P, P_MISC);
        uint32_t last = P.w[P_COUNTS + 2];
        bool straight = (flags & F_STRAIGHT) != 0;
        float4 ha = Q.hit_a[p];
        uint2 hb = Q.hit_b[p];
        Hit hit{ha.x, bu(ha.w), ha.y, ha.z, hb.x, hb.y};
        uint32_t nee_mask = 0, vis = 0;
        if (hit.tri == MISS) {
            V3 c = thr * sky_mis(S, X, P, d, depth > 0u ? last_pdf : 0.0f);
            if (depth > 1u && !straight) {
                float lum = luminance(c);
                if (lum > clamp_v) c = c * (clamp_v / lum);
            }
            radiance = radiance + c;
            flags |= F_DONE;
        } else {
            Surface s = surface(S, X, o, d, hit);
            if (depth == 0u) {
                V3 albedo = s.card ? s.emissive / fmaxf(fmaxf(s.emissive.x, fmaxf(s.emissive.y, s.emissive.z)), 1e-6f) : s.base;
                B.alb[p] = f4(albedo, hit.t);  // (w: the first hit's distance, for TRT_RENDER_DEPTH)
                B.nrm[p] = f4(s.n, 0.0f);
            }
            if (any_gt0(s.emissive) && (s.front || !s.card)) {
                float wgt = 1.0f;
                if (depth > 0u && (flags & F_SPECULAR_BOUNCE) == 0u)
                    wgt = emit_mis(S, X, P, hit, d, last_pdf, xyz(B.mis_x[p]), xyz(B.mis_n[p]));
                V3 c = thr * s.emissive * wgt;
                if (depth > 1u && !straight) {
                    float lum = luminance(c);
                    if (lum > clamp_v) c = c * (clamp_v / lum);
                }
                radiance = radiance + c;
            }
            if (s.card || depth == last) {
                flags |= F_DONE;
            } else {
                V3 v = -d;
                float nov = fmaxf(dot(s.n, v), 1e-4f);
                Lobes lb = lobes(S, X, P, s, nov);
                // direct_light (pathtrace.wgsl:2444-2546): each light's sample and its contribution if unoccluded.
                V3 oo = offset_origin(s.p, s.ng);
                uint32_t nd = min(P.w[P_COUNTS2], MAX_DIR_LIGHTS);
                for (uint32_t li = 0; li < nd; ++li) {
                    uint32_t b = X.t_lights + li * 5u;
                    float4 dir = tab(S, b + 1);
                    float cos_max = dir.w;
                    V3 to_light = -xyz(dir);
                    float u[2];
                    R.rng2(rng_sub(R.dim(D_SUN), li), u);
                    float cos_t = 1.0f - u[0] * (1.0f - cos_max);
                    float sin_t = sqrtf(fmaxf(0.0f, 1.0f - cos_t * cos_t));
                    float phi = 2.0f * PI * u[1];
                    Mat3 tb = basis(to_light);
                    V3 l = mul(tb, V3{sin_t * cosf(phi), sin_t * sinf(phi), cos_t});
                    V3 color = xyz(tab(S, b + 2));
                    if (all_le0(color)) continue;
                    V3 f = eval_bsdf_k(s, lb, v, l, tab(S, b + 4).y);
                    if (any_gt0(f)) {
                        float pdf_l = 1.0f / (2.0f * PI * (1.0f - cos_max));
                        float wgt = light_mis(pdf_l, s, lb, v, l);
                        B.nee[li * B.n + p] = f4(color * f * wgt * 1.0f, 0.0f);
                        nee_mask |= 1u << li;
                        if (tab(S, b + 3).w >= 0.5f) push_shadow(Q, cnt, CLASS_SUN, p, li, oo, l, INF, TRACE_SHADOW);
                        else vis |= 1u << li;
                    }
                }
                V3 ne = s.n;
                B.mis_x[p] = f4(oo, 0.0f);
                B.mis_n[p] = f4(ne, 0.0f);
                if (emitters_on(S, X, P)) {
                    // The candidates pathtrace.wgsl:2513 resamples: the tree's count at camera hits (one deeper),
                    // 6 / 3 without a tree where the camera sees the point, 2 with light LOD; else one CDF draw.
                    bool lt_on = pf(P, P_LTREE + 3) > 0.5f;
                    bool seen_directly = depth == 0u || (depth == 1u && (flags & F_MIRROR) != 0u);
                    uint32_t m = 0;
                    if (lt_on) m = depth == 0u ? (uint32_t)pf(P, P_LTREE + 3) : 1u;
                    else if (seen_directly) m = depth == 0u ? EMIT_RIS_M : EMIT_RIS_M / 2u;
                    else if (pf(P, P_LIGHT_LOD + 3) > 0.0f) m = 2u;
                    ES es = m > 0u ? sample_emitter_ris(S, X, P, R, oo, ne, m, s, lb, v, R.dim(D_EMIT))
                                   : sample_emitter(S, X, P, R, oo, ne, R.dim(D_EMIT));
                    if (es.pdf_w > 0.0f) {
                        V3 f = eval_bsdf_k(s, lb, v, es.l, 1.0f);
                        if (any_gt0(f)) {
                            float wgt = light_mis(es.pdf_w, s, lb, v, es.l) * 1.0f;
                            B.nee[SLOT_EMIT * B.n + p] = f4(es.le * f * wgt * es.w, 0.0f);
                            nee_mask |= 1u << SLOT_EMIT;
                            push_shadow(Q, cnt, CLASS_EMIT, p, SLOT_EMIT, oo, es.l, es.dist * 0.999f, TRACE_ANY);
                        }
                    }
                }
                bool env_sampled = P.w[P_COUNTS2 + 1] != 0u && (pf(P, P_ENV) > 0.5f || luminance(pv(P, P_SKY)) > 0.0f);
                if (env_sampled) {
                    V3 l = sample_env(S, P, R, R.dim(D_ENV));
                    V3 f = eval_bsdf_k(s, lb, v, l, 1.0f);
                    if (any_gt0(f)) {
                        float pdf_e = env_pdf(S, P, l);
                        if (pdf_e > 0.0f) {
                            B.nee[SLOT_ENV * B.n + p] = f4(env_radiance(S, P, l) * f * light_mis(pdf_e, s, lb, v, l) / pdf_e * 1.0f, 0.0f);
                            nee_mask |= 1u << SLOT_ENV;
                            push_shadow(Q, cnt, CLASS_ENV, p, SLOT_ENV, oo, l, INF, TRACE_SHADOW);
                        }
                    }
                }
                bool clamp_dl = depth > 0u && !straight;
                B.nee_thr[p] = f4(thr, bf(nee_mask | (clamp_dl ? 0x100u : 0u)));
                // sample_bsdf (pathtrace.wgsl:1848-1887, no coat, no glass)
                Mat3 tbn = basis(s.n);
                float r4[4];
                R.rng4(R.dim(D_BSDF), r4);
                bool sampled_spec = r4[1] < lb.p_spec;
                V3 l;
                if (sampled_spec) {
                    V3 hv = sample_vndf(v, tbn, s.roughness * s.roughness, r4[2], r4[3]);
                    l = reflect(-v, hv);
                } else {
                    float rr = sqrtf(r4[2]);
                    float phi = 2.0f * PI * r4[3];
                    l = mul(tbn, V3{rr * cosf(phi), rr * sinf(phi), sqrtf(fmaxf(0.0f, 1.0f - rr * rr))});
                }
                float pdf = pdf_bsdf(s, lb, v, l);
                V3 wgt = eval_bsdf_k(s, lb, v, l, 1.0f) / fmaxf(pdf, 1e-20f);
                if (pdf <= 0.0f || all_le0(wgt)) {
                    flags |= F_DONE;
                } else {
                    thr = thr * wgt;
                    bool mirror = (depth == 0u || (flags & F_MIRROR) != 0u) && s.roughness < MIRROR_ROUGHNESS && sampled_spec;
                    flags &= ~(F_SPECULAR_BOUNCE | F_STRAIGHT | F_MIRROR);
                    if (mirror) flags |= F_MIRROR;
                    if (depth >= P.w[P_COUNTS + 3]) {
                        float q = fminf(fmaxf(thr.x, fmaxf(thr.y, thr.z)), 0.95f);
                        if (R.rng1(R.dim(D_RR)) > q) flags |= F_DONE;
                        else thr = thr / q;
                    }
                    if ((flags & F_DONE) == 0u) {
                        o = offset_origin(s.p, dot(l, s.ng) < 0.0f ? -s.ng : s.ng);
                        d = l;
                        last_pdf = pdf;
                        live = true;
                    }
                }
            }
        }
        B.vis[p] = vis;
        if (nee_mask == 0u) B.nee_thr[p] = f4(v3(0.0f), bf(0u));
        B.o[p] = f4(o, last_pdf);
        B.d[p] = f4(d, bf(flags));
        B.thr[p] = f4(thr, bf(pix));
        B.rad[p] = f4(radiance, bf(sample));
    }
    uint32_t at = warp_append(&Q.cnt[(depth + 1u) * CNT_STRIDE], live);
    if (live && depth + 1u < MAX_DEPTH) next[at] = p;
}

// The vertex's direct light from its visible slots (pathtrace.wgsl:4398-4403), and a finished path's last fixes
// (4494-4497).
template <bool MULTI>
__global__ void k_resolve(const Job* __restrict__ jobs, const Job one, PathBufs B, Queues Q, uint32_t depth,
                          const uint32_t* __restrict__ queue) {
    uint32_t n = Q.cnt[depth * CNT_STRIDE];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t p = queue[i];
    float clamp_v = pf(MULTI ? jobs[B.job[p]].P : one.P, P_MISC);
    float4 nt = B.nee_thr[p];
    uint32_t m = bu(nt.w);
    float4 rad4 = B.rad[p];
    V3 radiance = xyz(rad4);
    if (m & 0xffu) {
        uint32_t vis = B.vis[p] & m;
        V3 sum = v3(0.0f);
        for (uint32_t k = 0; k < N_SLOTS; ++k)
            if (vis & (1u << k)) sum = sum + xyz(B.nee[k * B.n + p]);
        V3 dl = xyz(nt) * sum;
        if (m & 0x100u) {
            float lum = luminance(dl);
            if (lum > clamp_v) dl = dl * (clamp_v / lum);
        }
        radiance = radiance + dl;
    }
    uint32_t flags = bu(B.d[p].w);
    if (flags & F_DONE) {
        if (non_finite3(radiance)) radiance = v3(0.0f);
        float4 a = B.alb[p], nn = B.nrm[p];
        if (non_finite3(xyz(a))) B.alb[p] = f4(v3(0.0f), 0.0f);
        if (non_finite3(xyz(nn))) B.nrm[p] = f4(V3{0.0f, 1.0f, 0.0f}, 0.0f);
    }
    B.rad[p] = f4(radiance, rad4.w);
}

// ---- coherence sorts ----
// A counting sort of a depth's queue by a 12-bit key, on the device (no count reaches the host): each block counts
// its items' keys in shared memory and takes its range of each key with one global atomic; the last block to finish
// turns the global counts into starts (and zeroes them for the next sort); k_sort_scatter moves each item to its key's
// start plus its rank. Order within a key is the blocks' arrival order and may differ run to run: nothing depends on
// it, since a path's state, hit and random numbers belong to the path, not to its queue position.
//   SORT_RAYS: the extend queue by (queue chunk, direction octant): a warp's rays start near one another (the chunk)
//     and point the same way, so they walk the same nodes in the same order.
//   SORT_HITS (on unless TRT_RENDER_UNSORTED_HITS): the shade queue by material, misses first: a warp then reads one
//     material record and takes one set of branches, and the next depth's queue, appended in this order, starts its
//     rays from one mesh.
//   SORT_SHADOWS: the shadow rays by (position chunk, direction octant) in each light class.
constexpr uint32_t SORT_BINS = 4096u, SORT_THREADS = 256u, SORT_PER_THREAD = 8u;
constexpr uint32_t SORT_ITEMS = SORT_THREADS * SORT_PER_THREAD;
enum : uint32_t { SORT_RAYS = 0u, SORT_HITS = 1u, SORT_SHADOWS = 2u };

__device__ __forceinline__ uint32_t octant(float4 d) {
    return (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
}

// The items a sort orders: the depth's queue, or its shadow rays (n0, n1: the first two classes' counts).
template <uint32_t KIND>
__device__ __forceinline__ uint32_t sort_count(const Queues& Q, uint32_t depth, uint32_t& n0, uint32_t& n1) {
    const uint32_t* cnt = Q.cnt + depth * CNT_STRIDE;
    if (KIND != SORT_SHADOWS) return *(volatile const uint32_t*)&cnt[0];
    n0 = min(*(volatile const uint32_t*)&cnt[4], Q.class_cap[0]);
    n1 = min(*(volatile const uint32_t*)&cnt[5], Q.class_cap[1]);
    return n0 + n1 + min(*(volatile const uint32_t*)&cnt[6], Q.class_cap[2]);
}
template <uint32_t KIND>
__device__ __forceinline__ uint32_t sort_item(const Queues& Q, const uint32_t* in, uint32_t j, uint32_t n0, uint32_t n1) {
    return KIND == SORT_SHADOWS ? shadow_slot(Q, j, n0, n1) : in[j];
}
template <uint32_t KIND>
__device__ __forceinline__ uint32_t sort_key(const Job* jobs, const PathBufs& B, const Queues& Q, uint32_t j,
                                             uint32_t item, uint32_t shift) {
    if (KIND == SORT_RAYS) return ((j >> shift) << 3) | octant(B.d[item]);
    if (KIND == SORT_SHADOWS) return ((j >> shift) << 3) | octant(Q.sd[item]);
    if (bu(Q.hit_a[item].w) == MISS) return 0u;
    const Job& J = jobs[B.job[item]];
    const DScene& S = J.wk.S;
    Sections X(J.P);
    uint2 hb = Q.hit_b[item];
    uint32_t mat = 0;
    if (hb.x != NO_INST) {
        uint32_t rows = tabu(S, X.t_instances + hb.x * 10u + 6u).w;
        mat = __ldg(S.words + X.w_rows + (rows + hb.y) * 4u) & ROW_MATERIAL;
    }
    return 1u + mat % (SORT_BINS - 1u);
}

template <uint32_t KIND>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_count(const Job* __restrict__ jobs, PathBufs B, Queues Q,
                                                            const uint32_t* __restrict__ in, uint32_t depth,
                                                            uint32_t shift) {
    __shared__ uint32_t h[SORT_BINS];
    __shared__ uint32_t warp_sums[SORT_THREADS / 32u];
    __shared__ bool last;
    uint32_t n0 = 0, n1 = 0;
    uint32_t n = sort_count<KIND>(Q, depth, n0, n1);
    uint32_t base = blockIdx.x * SORT_ITEMS, tid = threadIdx.x;
    if (base < n) {
        for (uint32_t b = tid; b < SORT_BINS; b += SORT_THREADS) h[b] = 0u;
        __syncthreads();
        uint32_t key[SORT_PER_THREAD], loc[SORT_PER_THREAD];
        // The keys first, then the counts: the items' loads overlap instead of waiting behind each atomic.
#pragma unroll
        for (uint32_t k = 0; k < SORT_PER_THREAD; ++k) {
            uint32_t j = base + k * SORT_THREADS + tid;
            key[k] = j < n ? sort_key<KIND>(jobs, B, Q, j, sort_item<KIND>(Q, in, j, n0, n1), shift) & (SORT_BINS - 1u) : 0u;
        }
#pragma unroll
        for (uint32_t k = 0; k < SORT_PER_THREAD; ++k) {
            uint32_t j = base + k * SORT_THREADS + tid;
            loc[k] = j < n ? atomicAdd(&h[key[k]], 1u) : 0u;
        }
        __syncthreads();
        for (uint32_t b = tid; b < SORT_BINS; b += SORT_THREADS) {
            uint32_t c = h[b];
            if (c) h[b] = atomicAdd(&Q.sort_hist[b], c);
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 0; k < SORT_PER_THREAD; ++k) {
            uint32_t j = base + k * SORT_THREADS + tid;
            if (j < n) Q.sort_kr[j] = make_uint2(key[k], h[key[k]] + loc[k]);
        }
    }
    // The last block to finish: the counts into starts, by one exclusive scan of SORT_BINS.
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(Q.sort_done, 1u) == gridDim.x - 1u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    constexpr uint32_t PER = SORT_BINS / SORT_THREADS;
    uint32_t v[PER], sum = 0;
#pragma unroll
    for (uint32_t k = 0; k < PER; ++k) {
        v[k] = *(volatile uint32_t*)&Q.sort_hist[tid * PER + k];
        sum += v[k];
    }
    uint32_t lane = tid & 31u, warp = tid >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31u) warp_sums[warp] = incl;
    __syncthreads();
    uint32_t run = incl - sum;
    for (uint32_t w = 0; w < warp; ++w) run += warp_sums[w];
#pragma unroll
    for (uint32_t k = 0; k < PER; ++k) {
        Q.sort_start[tid * PER + k] = run;
        Q.sort_hist[tid * PER + k] = 0u;
        run += v[k];
    }
    if (tid == 0) *Q.sort_done = 0u;
}

template <uint32_t KIND>
__global__ void k_sort_scatter(Queues Q, const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t depth) {
    uint32_t n0 = 0, n1 = 0;
    uint32_t n = sort_count<KIND>(Q, depth, n0, n1);
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint2 kr = Q.sort_kr[j];
    out[Q.sort_start[kr.x] + kr.y] = sort_item<KIND>(Q, in, j, n0, n1);
}

// accum += each sample's path, in sample order (pathtrace.wgsl:4541-4557).
__device__ __forceinline__ void accumulate_one(const Job& J, const PathBufs& B, uint32_t idx) {
    uint32_t n_idx = J.n_idx, K = J.K;
    float4* accum = J.accum;
    uint32_t w = J.P.w[P_SIZE], h = J.P.w[P_SIZE + 1];
    uint32_t gx, gy;
    if (idx >= n_idx || !slot_pixel(idx + J.pix_first, w, h, gx, gy)) return;
    uint32_t pix = gy * w + gx;
    float4 c = accum[pix * 5], a = accum[pix * 5 + 1], nn = accum[pix * 5 + 2];
    float dsum = 0.0f;
    for (uint32_t k = 0; k < K; ++k) {
        uint32_t p = J.slot_first + k * n_idx + idx;
        float4 al4 = B.alb[p];
        V3 r = xyz(B.rad[p]), al = xyz(al4), nm = xyz(B.nrm[p]);
        dsum += al4.w;
        c.x += r.x; c.y += r.y; c.z += r.z; c.w += 1.0f;
        float lum = luminance(r);
        a.x += al.x; a.y += al.y; a.z += al.z; a.w += lum;
        nn.x += nm.x; nn.y += nm.y; nn.z += nm.z; nn.w += lum * lum;
    }
    accum[pix * 5] = c;
    accum[pix * 5 + 1] = a;
    accum[pix * 5 + 2] = nn;
    if (J.depth) accum[pix * 5 + 3].x += dsum;  // the sum of first-hit distances (0 where the camera ray escaped)
}
__global__ void k_accumulate(const Job* __restrict__ jobs, PathBufs B) {
    accumulate_one(jobs[blockIdx.y], B, blockIdx.x * blockDim.x + threadIdx.x);
}
// The same over every job's pixels in one flat pass (a thread a pixel index of some job).
__global__ void k_accumulate_flat(const Job* __restrict__ jobs, const StepHead* __restrict__ head, PathBufs B,
                                  uint32_t n_threads) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_threads) return;
    uint32_t n_jobs = head->n_jobs, j = 0;
    while (j + 1 < n_jobs && t >= jobs[j + 1].idx_first) ++j;
    const Job& J = jobs[j];
    if (n_jobs == 0 || t < J.idx_first || t - J.idx_first >= J.n_idx) return;
    accumulate_one(J, B, t - J.idx_first);
}

// Per-wave counts into the cumulative totals.
__global__ void k_tally(Queues Q, uint32_t depths, uint32_t paths, const StepHead* __restrict__ head) {
    if (threadIdx.x != 0) return;
    if (head) paths = head->paths;
    unsigned long long c = 0, s = 0;
    for (uint32_t d = 0; d < depths; ++d) {
        c += Q.cnt[d * CNT_STRIDE];
        for (uint32_t k = 0; k < 3; ++k) s += min(Q.cnt[d * CNT_STRIDE + 4 + k], Q.class_cap[k]);
    }
    atomicAdd(&Q.totals[T_CLOSEST], c);
    atomicAdd(&Q.totals[T_SHADOW], s);
    atomicAdd(&Q.totals[T_PATHS], (unsigned long long)paths);
}

template <bool COUNT, bool WIDE>
__global__ void k_trace(Params P, Walk wk, const trt_ray* rays, uint64_t n, trt_hit* hits, unsigned long long* totals) {
    Sections X(P);
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    WalkCount wc{0, 0, 0};
    if (i < n) {
        trt_ray r = rays[i];
        bool guard = false;
        // (closest-hit rays through the single loop, any-hit rays through the split one: the pass's own walks)
        const V3 o{r.o[0], r.o[1], r.o[2]}, d{r.d[0], r.d[1], r.d[2]};
        Hit h = r.mode == TRACE_CLOSEST ? walk<COUNT, WIDE>(wk, X, o, d, r.tmax, r.mode, &wc, &guard)
                                        : walk<COUNT, WIDE, true>(wk, X, o, d, r.tmax, r.mode, &wc, &guard);
        hits[i] = trt_hit{h.t, h.tri, h.u, h.v, h.inst, h.part};
    }
    if (COUNT) {
        warp_add64(&totals[T_E_NODES], wc.nodes);
        warp_add64(&totals[T_E_TRIS], wc.tris);
        warp_add64(&totals[T_E_UNITS], wc.units);
    }
}

// The device's single-precision transcendentals as the pass calls them (same compile flags): out[i] = f(x[i], y[i]).
__global__ void k_math_eval(uint32_t fn, const float* __restrict__ x, const float* __restrict__ y, uint64_t n,
                            float* __restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = x[i], b = y ? y[i] : 0.0f, r;
    switch (fn) {
        case TRT_MATH_COS: r = cosf(a); break;
        case TRT_MATH_SIN: r = sinf(a); break;
        case TRT_MATH_ACOS: r = acosf(a); break;
        case TRT_MATH_ATAN2: r = atan2f(a, b); break;
        default: r = __int_as_float(0x7fc00000); break;
    }
    out[i] = r;
}

// The Joe-Kuo direction numbers of Sobol dimensions 1-3, bit-reversed (the recurrence of the primitive polynomials
// x + 1, x^2 + x + 1, x^3 + x + 1 with initial numbers 1; 1, 3; 1, 3, 1).
void sobol_directions(uint32_t out[3][16]) {
    const int s_[3] = {1, 2, 3};
    const uint32_t a_[3] = {0, 1, 1};
    const uint32_t m0[3][3] = {{1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
    for (int k = 0; k < 3; ++k) {
        uint32_t m[32];
        int s = s_[k];
        for (int i = 0; i < 32; ++i) {
            if (i < s) {
                m[i] = m0[k][i];
            } else {
                uint32_t v = m[i - s] ^ (m[i - s] << s);
                for (int j = 1; j < s; ++j) v ^= ((a_[k] >> (s - 1 - j)) & 1u) * (m[i - j] << j);
                m[i] = v;
            }
        }
        for (int i = 0; i < 16; ++i) {
            uint32_t x = m[i] << (31 - i), r = 0;
            for (int b = 0; b < 32; ++b) r |= ((x >> b) & 1u) << (31 - b);
            out[k][i] = r;
        }
    }
}

}  // namespace trt

using namespace trt;

// ---- host side ------------------------------------------------------------------------------------------------------

struct trt_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<trt_scene*> scenes;  // live scenes, freed by trt_destroy
    int sm_count = 0;
    char name[256] = {0};
    std::string err;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    SkyState* sky = nullptr;  // the sky bake's tables and texels (trt_sky_bake, trt_scene_set_sky)
    cudaStream_t copy_stream = nullptr;  // asynchronous read-backs (TRT_RENDER_ASYNC_READBACK)
    cudaEvent_t copy_mark = nullptr;     // the copy stream's point the timer and synchronisation wait for
    // A render's second stream: each depth's shadow walk runs on it beside the next depth's closest-hit walk.
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // A render's second half-wave: its own stream pair, so that one half's shading shares the SMs with the other
    // half's walks.
    cudaStream_t half_stream = nullptr, half_aux = nullptr;
    cudaEvent_t half_fork = nullptr, half_join = nullptr, half_fork2 = nullptr, half_join2 = nullptr;
};

namespace trt {
// The device state of a wave: path slots, queues, the job table (one allocation).
struct Wave {
    void* work = nullptr;
    uint64_t work_bytes = 0;
    uint32_t slots = 0, shadow_alloc = 0;
    PathBufs B{};
    Queues Q{};
    Job* jobs = nullptr;
};
}  // namespace trt

struct trt_scene {
    trt_ctx* ctx = nullptr;
    void* buf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    uint64_t bytes[5] = {0, 0, 0, 0, 0};
    ushort4* env = nullptr;
    uint32_t env_w = 1, env_h = 1;
    std::vector<uint8_t> host[5];  // host copies of the buffers the wide BVH is built from
    WideBvh wide;
    float4* accum = nullptr;
    uint32_t accum_w = 0, accum_h = 0;
    // Asynchronous read-backs: a second accum, so that a render writes one while the other's copy to the host runs
    // on the context's copy stream; each buffer's event marks its last copy done (accum's and accum_alt's, swapped
    // with them). accum is always the last rendered.
    float4* accum_alt = nullptr;
    cudaEvent_t copied = nullptr, copied_alt = nullptr;
    Wave wave;  // the render's wave state
    Wave wave2; // the second half-wave's
    void* dn = nullptr;  // the denoiser's buffers, for dn_w x dn_h pixels
    uint32_t dn_w = 0, dn_h = 0;
    DenoiseBufs D{};
    float* dn_rgb = nullptr;
    unsigned long long* totals = nullptr;
    int profiling = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_extend, ev_shadow, ev_shade, ev_sort, ev_free;
    double extend_ms = 0, shadow_ms = 0, shade_ms = 0, sort_ms = 0;
    uint64_t extend_launches = 0, shadow_launches = 0, renders = 0, launches = 0;
    // The per-frame deformation (trt_deform_setup), and whether the host copies still hold what the device does.
    DeformState* deform = nullptr;
    void* em = nullptr;  // the emitter re-weigh's scratch (trt_scene_weigh_emitters)
    uint64_t em_bytes = 0;
    bool deform_stale = false;  // the nodes were written after setup: its tree checks no longer hold
    bool deformed = false;      // a deformation ran: the host copies are old (a wide BVH built from them is refit)
    uint64_t deform_gen = 0;    // deformations run (WideBvh::refit_gen: the one the wide trees were brought to)
};

namespace {

std::mutex g_sobol_mu;

int fail(trt_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}
int cuda_fail(trt_ctx* c, cudaError_t e, const char* what) {
    return fail(c, TRT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define TRT_CUDA(ctx, call)                                         \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);  \
    } while (0)

DScene scene_view(const trt_scene* s) {
    DScene S;
    S.vertices = (const float4*)s->buf[0];
    S.leaves = (const float4*)s->buf[1];
    S.nodes = (const uint4*)s->buf[2];
    S.tables = (const uint4*)s->buf[3];
    S.words = (const uint32_t*)s->buf[4];
    S.env = s->env;
    S.env_w = s->env_w;
    S.env_h = s->env_h;
    S.n_nodes = s->bytes[2] / 32;
    S.n_tris = s->bytes[1] / 48;
    S.n_table_vec4 = s->bytes[3] / 16;
    S.n_words = s->bytes[4] / 4;
    return S;
}

// Checks that what Params names lies inside the uploaded buffers (the reference trusts its own prep; a C ABI does not).
int check_params(trt_scene* s, const uint32_t* P) {
    uint64_t tv = s->bytes[3] / 16, wn = s->bytes[4] / 4;
    for (int k = 0; k < 12; ++k)
        if (P[P_TABLE_FIRST + k] > tv) return fail(s->ctx, TRT_EINVAL, "Params.table_first names a vec4 past the tables");
    for (int k = 0; k < 5; ++k)
        if (P[P_WORD_FIRST + k] > wn) return fail(s->ctx, TRT_EINVAL, "Params.word_first names a word past the words");
    uint32_t w = P[P_SIZE], h = P[P_SIZE + 1];
    if (w == 0 || h == 0 || (uint64_t)w * h > (1ull << 26)) return fail(s->ctx, TRT_EINVAL, "Params.size: 1 to 2^26 pixels");
    if (P[P_COUNTS + 2] >= MAX_DEPTH - 1) return fail(s->ctx, TRT_EINVAL, "Params.counts.z (max bounces) must be below 63");
    if (P[P_COUNTS2] > MAX_DIR_LIGHTS) return fail(s->ctx, TRT_EINVAL, "more than 4 directional lights");
    if (P[P_COUNTS] != P[P_COUNTS2]) return fail(s->ctx, TRT_EINVAL, "local lights are not part of this pass");
    uint32_t top = P[P_MOTION + 2], units = P[P_MOTION + 3];
    if (units > 0 && (uint64_t)top >= s->bytes[2] / 32) return fail(s->ctx, TRT_EINVAL, "Params.motion.z names a node past the nodes");
    if (P[P_ENV] == 0x3f800000u && ((uint32_t)bf(P[P_ENV + 1]) != s->env_w || (uint32_t)bf(P[P_ENV + 2]) != s->env_h))
        return fail(s->ctx, TRT_EINVAL, "Params.env's size is not the uploaded environment's");
    return TRT_OK;
}

// A wave's device state sized for `slots` paths with up to n_dir suns each: one allocation, laid out here.
int wave_ensure(Wave& w, uint32_t slots, uint32_t n_dir, unsigned long long* totals, cudaStream_t st, std::string& err) {
    // Shadow-ray regions: a ray a sun a path, one toward an emitter, one toward the sky.
    uint32_t caps[3] = {slots * std::max(1u, n_dir), slots, slots};
    uint32_t shadow_cap = caps[0] + caps[1] + caps[2];
    if (!w.work || w.slots < slots || w.shadow_alloc < shadow_cap) {
        uint64_t need = 0;
        auto add = [&](uint64_t b) { uint64_t at = need; need += (b + 255) / 256 * 256; return at; };
        uint64_t o_o = add(16ull * slots), o_d = add(16ull * slots), o_thr = add(16ull * slots),
                 o_rad = add(16ull * slots), o_alb = add(16ull * slots), o_nrm = add(16ull * slots),
                 o_mx = add(16ull * slots), o_mn = add(16ull * slots), o_nee = add(16ull * slots * N_SLOTS),
                 o_nt = add(16ull * slots), o_vis = add(4ull * slots), o_q0 = add(4ull * slots), o_q1 = add(4ull * slots),
                 o_ha = add(16ull * slots), o_hb = add(8ull * slots), o_so = add(16ull * shadow_cap),
                 o_sd = add(16ull * shadow_cap), o_sp = add(4ull * shadow_cap),
                 o_cnt = add(4ull * (MAX_DEPTH * CNT_STRIDE + CNT_STRIDE)), o_qx = add(4ull * slots),
                 o_kr = add(8ull * std::max(slots, shadow_cap)), o_hist = add(4ull * SORT_BINS),
                 o_start = add(4ull * SORT_BINS), o_done = add(4ull), o_perm = add(4ull * shadow_cap),
                 o_job = add(4ull * slots), o_jobs = add(sizeof(Job) * MAX_JOBS);
        if (w.work) cudaFree(w.work);
        w.work = nullptr;
        cudaError_t e = cudaMalloc(&w.work, need);
        if (e != cudaSuccess) {
            err = std::string("wave state (") + std::to_string(need >> 20) + " MiB): " + cudaGetErrorString(e);
            w.slots = w.shadow_alloc = 0;
            return TRT_ECUDA;
        }
        w.work_bytes = need;
        char* b = (char*)w.work;
        w.slots = slots;
        w.shadow_alloc = shadow_cap;
        w.B = PathBufs{(float4*)(b + o_o), (float4*)(b + o_d), (float4*)(b + o_thr), (float4*)(b + o_rad),
                       (float4*)(b + o_alb), (float4*)(b + o_nrm), (float4*)(b + o_mx), (float4*)(b + o_mn),
                       (float4*)(b + o_nee), (float4*)(b + o_nt), (uint32_t*)(b + o_vis), (uint32_t*)(b + o_job),
                       slots};
        w.jobs = (Job*)(b + o_jobs);
        w.Q.q[0] = (uint32_t*)(b + o_q0);
        w.Q.q[1] = (uint32_t*)(b + o_q1);
        w.Q.hit_a = (float4*)(b + o_ha);
        w.Q.hit_b = (uint2*)(b + o_hb);
        w.Q.so = (float4*)(b + o_so);
        w.Q.sd = (float4*)(b + o_sd);
        w.Q.sp = (uint32_t*)(b + o_sp);
        w.Q.cnt = (uint32_t*)(b + o_cnt);
        w.Q.qx = (uint32_t*)(b + o_qx);
        w.Q.sort_kr = (uint2*)(b + o_kr);
        w.Q.sort_hist = (uint32_t*)(b + o_hist);
        w.Q.sort_start = (uint32_t*)(b + o_start);
        w.Q.sort_done = (uint32_t*)(b + o_done);
        w.Q.perm = (uint32_t*)(b + o_perm);
        // The sort's counts and its finished-block count start at zero (each sort leaves them so).
        e = cudaMemsetAsync(b + o_hist, 0, o_start - o_hist, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b + o_done, 0, 4, st);
        if (e != cudaSuccess) {
            err = std::string("wave state: ") + cudaGetErrorString(e);
            return TRT_ECUDA;
        }
    }
    w.Q.totals = totals;
    w.Q.shadow_cap = shadow_cap;
    w.Q.class_base[0] = 0;
    w.Q.class_base[1] = caps[0];
    w.Q.class_base[2] = caps[0] + caps[1];
    for (int k = 0; k < 3; ++k) w.Q.class_cap[k] = caps[k];
    return TRT_OK;
}

std::pair<cudaEvent_t, cudaEvent_t> take_events(trt_scene* s) {
    if (!s->ev_free.empty()) {
        auto e = s->ev_free.back();
        s->ev_free.pop_back();
        return e;
    }
    std::pair<cudaEvent_t, cudaEvent_t> e{nullptr, nullptr};
    cudaEventCreate(&e.first);
    cudaEventCreate(&e.second);
    return e;
}

// The binary walks and the shading live on L1 hits (node records, the walks' stacks, triangle and material records)
// and use no shared memory: they ask for the whole of the SM's L1 / shared-memory split as L1, also when they share an
// SM with kernels that use shared memory (measured on the city: 1,138 -> 1,141 Mrays/s; the Cornell box 3,088-3,111 ->
// 3,116). Not the wide walks: their stacks' first entries live in shared memory, and a split that leaves it the least
// the driver may give a block would hold few of their blocks (the wide walk fell from 912-944 to 336 Mrays/s).
void prefer_l1() {
    const void* fns[] = {(const void*)k_extend<false, false, false>, (const void*)k_extend<true, false, false>,
                         (const void*)k_extend<false, false, true>,  (const void*)k_shadow<false, false, false>,
                         (const void*)k_shadow<true, false, false>,  (const void*)k_shadow<false, false, true>,
                         (const void*)k_shade<false>,                (const void*)k_shade<true>};
    for (const void* f : fns) cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaGetLastError();  // (a hint: a device that refuses it runs the kernels as they are)
}

int grid_for(const void* fn, int block, int sm_count) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0);
    return std::max(1, per_sm) * sm_count;
}

// The smallest shift that maps positions below `cap` onto at most SORT_BINS / 8 chunks.
uint32_t chunk_shift(uint32_t cap) {
    uint32_t sh = 0;
    while (cap > 0 && ((cap - 1u) >> sh) >= SORT_BINS / 8u) ++sh;
    return sh;
}

template <uint32_t KIND>
void launch_sort(trt_scene* s, Wave& W, const uint32_t* in, uint32_t* out, uint32_t depth, uint32_t cap, cudaStream_t st) {
    uint32_t shift = chunk_shift(cap);
    k_sort_count<KIND><<<(cap + SORT_ITEMS - 1u) / SORT_ITEMS, SORT_THREADS, 0, st>>>(W.jobs, W.B, W.Q, in, depth, shift);
    k_sort_scatter<KIND><<<(cap + 255u) / 256u, 256, 0, st>>>(W.Q, in, out, depth);
    s->launches += 2;
}

// A wave's launches on a stream pair (st, aux): ray generation, then each depth's walks, sorts, shading and resolve,
// then the accumulation. g_ext / g_sha: the persistent walks' grids.
template <bool COUNT, bool WIDE>
void launch_wave(trt_scene* s, Wave& W, const Job& job, uint32_t n, uint32_t last, uint32_t flags_eff,
                 cudaStream_t st, cudaStream_t aux, cudaEvent_t fork_ev, cudaEvent_t join_ev, int g_ext, int g_sha) {
    const bool sort_rays = (flags_eff & TRT_RENDER_SORT_RAYS) != 0;
    const bool sort_hits = (flags_eff & TRT_RENDER_UNSORTED_HITS) == 0;
    const bool sort_shadows = (flags_eff & TRT_RENDER_SORT_SHADOWS) != 0;
    const int blk = 128;
    auto mark = [&](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, bool begin, cudaStream_t on) {
        if (!s->profiling) return;
        if (begin) { v.push_back(take_events(s)); cudaEventRecord(v.back().first, on); }
        else cudaEventRecord(v.back().second, on);
    };
    // Each depth's shadow walk on the second stream beside the next depth's closest-hit walk: both read what the
    // depth's shading wrote and write apart (visibility bits; hit records), so their tails overlap. (Not with the ray
    // sort, whose output buffer is the previous depth's shading order, which that depth's resolve still reads.)
    const bool overlap = !sort_rays;
    k_put_job<<<1, 128, 0, st>>>(job, W.jobs, 0u);
    k_raygen<<<(n + blk - 1) / blk, blk, 0, st>>>(W.jobs, 1u, W.B, W.Q, n, nullptr);
    s->launches += 2;
    for (uint32_t depth = 0; depth <= last; ++depth) {
        // The depth's queue (raw), the order extend walks it in, the order shade takes the hits in.
        uint32_t* raw = W.Q.q[depth & 1u];
        uint32_t* next = W.Q.q[(depth + 1u) & 1u];
        uint32_t* ext_q = raw;
        if (sort_rays && depth > 0u) {
            mark(s->ev_sort, true, st);
            launch_sort<SORT_RAYS>(s, W, raw, W.Q.qx, depth, n, st);
            mark(s->ev_sort, false, st);
            ext_q = W.Q.qx;
        }
        if (!overlap || depth == 0u) {  // (past depth 0 with the overlap, launched beside the last shadow walk)
            mark(s->ev_extend, true, st);
            k_extend<COUNT, WIDE, false><<<g_ext, blk, 0, st>>>(W.jobs, job, W.B, W.Q, depth, ext_q);
            mark(s->ev_extend, false, st);
        }
        uint32_t* shade_q = ext_q;
        if (sort_hits) {
            shade_q = ext_q == raw ? W.Q.qx : raw;
            mark(s->ev_sort, true, st);
            launch_sort<SORT_HITS>(s, W, ext_q, shade_q, depth, n, st);
            mark(s->ev_sort, false, st);
        }
        mark(s->ev_shade, true, st);
        k_shade<false><<<(n + blk - 1) / blk, blk, 0, st>>>(W.jobs, job, W.B, W.Q, depth, shade_q, next);
        mark(s->ev_shade, false, st);
        const uint32_t* perm = nullptr;
        if (sort_shadows) {
            mark(s->ev_sort, true, st);
            launch_sort<SORT_SHADOWS>(s, W, nullptr, W.Q.perm, depth, W.Q.shadow_cap, st);
            mark(s->ev_sort, false, st);
            perm = W.Q.perm;
        }
        if (overlap) {
            cudaEventRecord(fork_ev, st);
            cudaStreamWaitEvent(aux, fork_ev, 0);
            mark(s->ev_shadow, true, aux);
            k_shadow<COUNT, WIDE, false><<<g_sha, blk, 0, aux>>>(W.jobs, job, W.B, W.Q, depth, perm);
            mark(s->ev_shadow, false, aux);
            if (depth < last) {
                mark(s->ev_extend, true, st);
                k_extend<COUNT, WIDE, false><<<g_ext, blk, 0, st>>>(W.jobs, job, W.B, W.Q, depth + 1u, next);
                mark(s->ev_extend, false, st);
            }
            cudaEventRecord(join_ev, aux);
            cudaStreamWaitEvent(st, join_ev, 0);
        } else {
            mark(s->ev_shadow, true, st);
            k_shadow<COUNT, WIDE, false><<<g_sha, blk, 0, st>>>(W.jobs, job, W.B, W.Q, depth, perm);
            mark(s->ev_shadow, false, st);
        }
        k_resolve<false><<<(n + blk - 1) / blk, blk, 0, st>>>(W.jobs, job, W.B, W.Q, depth, shade_q);
        s->launches += 4;
        s->extend_launches++;
        s->shadow_launches++;
    }
    k_accumulate<<<dim3((job.n_idx + blk - 1) / blk, 1), blk, 0, st>>>(W.jobs, W.B);
    s->launches++;
}

// A wave of at least this many paths runs as two half-waves (their own queues and stream pairs): one half's shading,
// latency-bound, then shares the SMs with the other half's walks, issue-bound. Each half's persistent walks are sized
// for the whole GPU (measured on the city frame: 1,134 Mrays/s, against 1,125 with half the grid each and 1,118 in
// one wave; the Cornell box 3,099, 3,228 and 3,048).
#ifndef TRT_HALF_WAVE_MIN
#define TRT_HALF_WAVE_MIN (1u << 19)
#endif

template <bool COUNT, bool WIDE>
int render_waves(trt_scene* s, const Params& P, uint32_t first_sample, uint32_t spp, uint32_t flags) {
    trt_ctx* c = s->ctx;
    cudaStream_t st = c->stream;
    uint32_t w = P.w[P_SIZE], h = P.w[P_SIZE + 1];
    uint32_t n_idx = ((w + 7u) / 8u) * ((h + 3u) / 4u) * 32u;
    // Samples a wave: enough paths to fill the GPU (about two million), at most spp.
    uint32_t K = std::max(1u, std::min(spp, (2u << 20) / std::max(1u, n_idx)));
    uint32_t n_dir = P.w[P_COUNTS2];
    // Two half-waves: the image's pixel indices (8 x 4 tiles of 32) split at a tile.
    const bool halves = (uint64_t)n_idx * K >= TRT_HALF_WAVE_MIN && n_idx >= 64u;
    const uint32_t n_idx_a = halves ? (n_idx / 2u) / 32u * 32u : n_idx, n_idx_b = n_idx - n_idx_a;
    int rc = wave_ensure(s->wave, n_idx_a * K, n_dir, s->totals, st, c->err);
    if (rc) return rc;
    if (halves) {
        rc = wave_ensure(s->wave2, n_idx_b * K, n_dir, s->totals, st, c->err);
        if (rc) return rc;
    }
    Walk wk{scene_view(s), s->wide.view(), P.w[P_MOTION + 2], P.w[P_MOTION + 3]};
    uint32_t last = P.w[P_COUNTS + 2];
    // the material table's records (18 vec4 each) between its first row and the lights' first row
    const uint32_t n_materials = (P.w[P_TABLE_FIRST + 2] - P.w[P_TABLE_FIRST + 1]) / 18u;
    const bool sort_hits = (flags & TRT_RENDER_UNSORTED_HITS) == 0 && n_materials > TRT_SORT_HITS_MIN_MATERIALS;
    const uint32_t flags_eff = (flags & ~TRT_RENDER_UNSORTED_HITS) | (sort_hits ? 0u : TRT_RENDER_UNSORTED_HITS);
    const int blk = 128;
    int g_ext = grid_for((const void*)k_extend<COUNT, WIDE, false>, blk, c->sm_count);
    int g_sha = grid_for((const void*)k_shadow<COUNT, WIDE, false>, blk, c->sm_count);
    std::vector<uint32_t> host_cnt(MAX_DEPTH * CNT_STRIDE + CNT_STRIDE, 0);
    for (uint32_t s0 = 0; s0 < spp; s0 += K) {
        uint32_t k = std::min(K, spp - s0);
        const uint32_t depth_flag = (flags & TRT_RENDER_DEPTH) ? 1u : 0u;
        Job job_a{P, wk, s->accum, 0u, n_idx_a, k, first_sample + s0, 0u, depth_flag, 0u};
        TRT_CUDA(c, cudaMemcpyAsync(s->wave.Q.cnt, host_cnt.data(), host_cnt.size() * 4, cudaMemcpyHostToDevice, st));
        if (halves) {
            // The second half on its own stream pair, after what the main stream holds so far; joined at the end.
            Job job_b{P, wk, s->accum, 0u, n_idx_b, k, first_sample + s0, 0u, depth_flag, n_idx_a};
            TRT_CUDA(c, cudaEventRecord(c->half_fork, st));
            TRT_CUDA(c, cudaStreamWaitEvent(c->half_stream, c->half_fork, 0));
            TRT_CUDA(c, cudaMemcpyAsync(s->wave2.Q.cnt, host_cnt.data(), host_cnt.size() * 4, cudaMemcpyHostToDevice,
                                        c->half_stream));
            launch_wave<COUNT, WIDE>(s, s->wave, job_a, n_idx_a * k, last, flags_eff, st, c->aux_stream, c->fork_ev,
                                     c->join_ev, g_ext, g_sha);
            launch_wave<COUNT, WIDE>(s, s->wave2, job_b, n_idx_b * k, last, flags_eff, c->half_stream, c->half_aux,
                                     c->half_fork2, c->half_join2, g_ext, g_sha);
            k_tally<<<1, 32, 0, c->half_stream>>>(s->wave2.Q, last + 1, 0u, nullptr);
            TRT_CUDA(c, cudaEventRecord(c->half_join, c->half_stream));
            TRT_CUDA(c, cudaStreamWaitEvent(st, c->half_join, 0));
        } else {
            launch_wave<COUNT, WIDE>(s, s->wave, job_a, n_idx_a * k, last, flags_eff, st, c->aux_stream, c->fork_ev,
                                     c->join_ev, g_ext, g_sha);
        }
        k_tally<<<1, 32, 0, st>>>(s->wave.Q, last + 1, w * h * k, nullptr);
        s->launches += halves ? 2 : 1;
    }
    TRT_CUDA(c, cudaGetLastError());
    return TRT_OK;
}

}  // namespace

// ---- the render without allocations --------------------------------------------------------------------------------
//
// For callers that cannot call cudaMalloc: code running inside a CUDA graph being captured, or under a memory pool
// that owns all of a device's memory (an engine's caching allocator, a process with a hard device-memory budget).
// They own the scene's buffers and the accum themselves; the wave's working state lives in this file-scope array,
// which every GPU that loads the library holds until the process exits.

// The largest wave the array holds: 65,536 path slots (a 256 x 256 image, one sample a wave) with up to 4 suns.
constexpr uint32_t NOALLOC_SLOTS = 65536u;
constexpr uint32_t NOALLOC_SHADOW = NOALLOC_SLOTS * (MAX_DIR_LIGHTS + 2u);
constexpr uint64_t na_round(uint64_t b) { return (b + 255u) / 256u * 256u; }
constexpr uint64_t NOALLOC_BYTES =
    8 * na_round(16ull * NOALLOC_SLOTS) + na_round(16ull * NOALLOC_SLOTS * N_SLOTS) + na_round(16ull * NOALLOC_SLOTS) +
    na_round(4ull * NOALLOC_SLOTS) + 2 * na_round(4ull * NOALLOC_SLOTS) + na_round(16ull * NOALLOC_SLOTS) +
    na_round(8ull * NOALLOC_SLOTS) + 2 * na_round(16ull * NOALLOC_SHADOW) + na_round(4ull * NOALLOC_SHADOW) +
    na_round(4ull * (MAX_DEPTH * CNT_STRIDE + CNT_STRIDE)) + na_round(8ull * T_COUNT) + na_round(4ull * NOALLOC_SLOTS) +
    na_round(sizeof(Job));
static_assert(NOALLOC_BYTES < (32ull << 20), "the no-allocation scratch stays under 32 MiB");

static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_BYTES];

namespace {

std::mutex g_noalloc_mu;
uint8_t* g_noalloc_ptr[256] = {nullptr};  // the array's device address, per device ordinal

int na_fail(char* err, size_t err_len, int code, const std::string& msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg.c_str());
    return code;
}

// Once per device, with it current: the array's device address (in host code its name is only a stand-in for it)
// and the sampler's tables.
int noalloc_setup(int dev, char* err, size_t err_len) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (dev < 0 || dev >= 256) return na_fail(err, err_len, TRT_EINVAL, "device ordinal out of range");
    if (g_noalloc_ptr[dev]) return TRT_OK;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return na_fail(err, err_len, TRT_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    uint32_t t[3][16], bytes[3][2][256];
    sobol_directions(t);
    for (int d = 0; d < 3; ++d)
        for (int half = 0; half < 2; ++half)
            for (uint32_t b = 0; b < 256; ++b) {
                uint32_t r = 0;
                for (int i = 0; i < 8; ++i)
                    if (b & (0x80u >> i)) r ^= t[d][half * 8 + i];
                bytes[d][half][b] = r;
            }
    e = cudaMemcpyToSymbol(g_sobol_bytes, bytes, sizeof(bytes));
    if (e != cudaSuccess) return na_fail(err, err_len, TRT_ECUDA, std::string("sampler tables: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (uint8_t*)ptr;
    return TRT_OK;
}

}  // namespace


extern "C" {

int trt_create(const trt_options* opts, trt_ctx** out) {
    if (!out) return TRT_EINVAL;
    *out = nullptr;
    auto* c = new trt_ctx();
    c->device = opts ? opts->device : 0;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    cudaDeviceProp prop;
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, c->device);
    if (e == cudaSuccess) {
        std::snprintf(c->name, sizeof(c->name), "%s", prop.name);
        if (prop.major < 10) e = cudaErrorNoKernelImageForDevice;
    }
    if (e == cudaSuccess) prefer_l1();
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> lk(g_sobol_mu);
        uint32_t t[3][16], bytes[3][2][256];
        sobol_directions(t);
        for (int d = 0; d < 3; ++d)
            for (int half = 0; half < 2; ++half)
                for (uint32_t b = 0; b < 256; ++b) {
                    uint32_t r = 0;
                    for (int i = 0; i < 8; ++i)
                        if (b & (0x80u >> i)) r ^= t[d][half * 8 + i];
                    bytes[d][half][b] = r;
                }
        e = cudaMemcpyToSymbol(g_sobol_bytes, bytes, sizeof(bytes));
    }
    if (e == cudaSuccess) e = cudaEventCreate(&c->t0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->t1);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->copy_mark, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->half_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->half_aux, cudaStreamNonBlocking);
    for (cudaEvent_t* ev : {&c->half_fork, &c->half_join, &c->half_fork2, &c->half_join2})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        // (No context to hold the message: the caller gets the code.)
        std::fprintf(stderr, "trt_create: %s\n", cudaGetErrorString(e));
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
        if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
        if (c->half_stream) cudaStreamDestroy(c->half_stream);
        if (c->half_aux) cudaStreamDestroy(c->half_aux);
        delete c;
        return TRT_ECUDA;
    }
    *out = c;
    return TRT_OK;
}

void trt_destroy(trt_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    while (!c->scenes.empty()) trt_scene_free(c->scenes.back());
    sky_free(c->sky);
    if (c->t0) cudaEventDestroy(c->t0);
    if (c->t1) cudaEventDestroy(c->t1);
    if (c->copy_mark) cudaEventDestroy(c->copy_mark);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->join_ev) cudaEventDestroy(c->join_ev);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    for (cudaEvent_t ev : {c->half_fork, c->half_join, c->half_fork2, c->half_join2})
        if (ev) cudaEventDestroy(ev);
    if (c->half_stream) cudaStreamDestroy(c->half_stream);
    if (c->half_aux) cudaStreamDestroy(c->half_aux);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* trt_last_error(const trt_ctx* c) { return c ? c->err.c_str() : "no context"; }

int trt_device_info(const trt_ctx* c, char* name, size_t name_len, int* sm_count) {
    if (!c) return TRT_EINVAL;
    if (name && name_len) std::snprintf(name, name_len, "%s", c->name);
    if (sm_count) *sm_count = c->sm_count;
    return TRT_OK;
}

int trt_scene_upload(trt_ctx* c, const trt_scene_desc* d, trt_scene** out) {
    if (!c || !d || !out) return TRT_EINVAL;
    *out = nullptr;
    cudaSetDevice(c->device);
    const void* src[5] = {d->vertices, d->leaves, d->nodes, d->tables, d->words};
    const uint64_t n[5] = {d->vertices_bytes, d->leaves_bytes, d->nodes_bytes, d->tables_bytes, d->words_bytes};
    const uint64_t unit[5] = {48, 48, 32, 16, 4};
    for (int k = 0; k < 5; ++k)
        if (!src[k] || n[k] == 0 || n[k] % unit[k] != 0)
            return fail(c, TRT_EINVAL, "scene buffer " + std::to_string(k) + ": no data, or not whole records");
    if (!d->env_half || d->env_w == 0 || d->env_h == 0) return fail(c, TRT_EINVAL, "no environment texels");
    auto* s = new trt_scene();
    s->ctx = c;
    auto cleanup = [&](int rc) { trt_scene_free(s); return rc; };
    for (int k = 0; k < 5; ++k) {
        cudaError_t e = cudaMalloc(&s->buf[k], n[k]);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->buf[k], src[k], n[k], cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return cleanup(cuda_fail(c, e, "scene upload"));
        s->bytes[k] = n[k];
        if (k >= 1 && k <= 3) s->host[k].assign((const uint8_t*)src[k], (const uint8_t*)src[k] + n[k]);
    }
    s->env_w = d->env_w;
    s->env_h = d->env_h;
    uint64_t eb = 8ull * d->env_w * d->env_h;
    cudaError_t e = cudaMalloc(&s->env, eb);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->env, d->env_half, eb, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMalloc(&s->totals, sizeof(unsigned long long) * T_COUNT);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->totals, 0, sizeof(unsigned long long) * T_COUNT, c->stream);
    if (e != cudaSuccess) return cleanup(cuda_fail(c, e, "scene upload"));
    s->wave.Q.totals = s->totals;
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cleanup(cuda_fail(c, e, "scene upload"));
    c->scenes.push_back(s);
    *out = s;
    return TRT_OK;
}

void trt_scene_free(trt_scene* s) {
    if (!s) return;
    auto& live = s->ctx->scenes;
    live.erase(std::remove(live.begin(), live.end(), s), live.end());
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    cudaStreamSynchronize(s->ctx->copy_stream);
    for (void* b : s->buf)
        if (b) cudaFree(b);
    if (s->env) cudaFree(s->env);
    if (s->accum) cudaFree(s->accum);
    if (s->accum_alt) cudaFree(s->accum_alt);
    if (s->copied) cudaEventDestroy(s->copied);
    if (s->copied_alt) cudaEventDestroy(s->copied_alt);
    if (s->wave.work) cudaFree(s->wave.work);
    if (s->wave2.work) cudaFree(s->wave2.work);
    if (s->dn) cudaFree(s->dn);
    if (s->totals) cudaFree(s->totals);
    deform_free(s->deform);
    if (s->em) cudaFree(s->em);
    s->wide.release();
    for (auto* v : {&s->ev_extend, &s->ev_shadow, &s->ev_shade, &s->ev_sort, &s->ev_free})
        for (auto& e : *v) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    delete s;
}

namespace {

// The wide BVH brought to the deformed buffers on the device (WideBvh::refit); errors go to the deformation's word.
int refit_wide(trt_scene* s, const uint32_t* params) {
    trt_ctx* c = s->ctx;
    if (s->wide.refit(params, s->buf[2], s->bytes[2] / 32, s->buf[1], s->bytes[1] / 48, s->buf[3], s->bytes[3] / 16,
                      deform_error_word(s->deform), DEFORM_E_WIDE, c->stream) != 0)
        return fail(c, TRT_ECUDA, s->wide.error);
    s->wide.refit_gen = s->deform_gen;
    return TRT_OK;
}

// The wide BVH for a walk: built from the host copies (the scene as uploaded and edited), then, on a deformed scene,
// brought to the device's buffers; a refit here waits for its error word.
int ensure_wide(trt_scene* s, const uint32_t* params) {
    trt_ctx* c = s->ctx;
    if (s->wide.ensure(params, s->host, c->stream) != 0) return fail(c, TRT_EINVAL, s->wide.error);
    if (!s->deformed || s->wide.refit_gen == s->deform_gen) return TRT_OK;
    int rc = refit_wide(s, params);
    if (rc) return rc;
    uint32_t errors = 0;
    if (deform_errors(s->deform, c->stream, &errors) != TRT_OK) return fail(c, TRT_ECUDA, "reading the deformation's errors");
    if (errors) return fail(c, TRT_EGUARD, "the deformation or the wide BVH's refit met a bad tree (error bits " + std::to_string(errors) + ")");
    return TRT_OK;
}

}  // namespace

int trt_scene_update(trt_scene* s, uint32_t which, uint64_t offset, const void* src, uint64_t bytes) {
    if (!s) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    if (which > 4 || !src || offset + bytes > s->bytes[which] || offset + bytes < offset)
        return fail(c, TRT_EINVAL, "trt_scene_update: the range is not inside the buffer");
    cudaSetDevice(c->device);
    TRT_CUDA(c, cudaMemcpyAsync((char*)s->buf[which] + offset, src, bytes, cudaMemcpyHostToDevice, c->stream));
    if (which >= 1 && which <= 3) {
        // The wide BVH is rebuilt from the edited buffers at the next render; of the tables it reads only the units'
        // mesh roots, first triangles and shadow bits, so an edit that leaves those alone (units moved by their
        // transforms) keeps it.
        if (which != 3 ||
            s->wide.reads_edit(s->host[3].data(), s->host[3].size(), offset, static_cast<const uint8_t*>(src), bytes))
            s->wide.invalidate();
        std::memcpy(s->host[which].data() + offset, src, bytes);
    }
    if (which == 2 && s->deform) s->deform_stale = true;
    return TRT_OK;
}

int trt_denoise_atrous(trt_scene* s, uint32_t iterations, float* rgb_host, float* ms) {
    if (!s || !rgb_host || iterations > 16) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    if (!s->accum) return fail(c, TRT_EINVAL, "trt_denoise_atrous: nothing rendered yet");
    cudaSetDevice(c->device);
    cudaStream_t st = c->stream;
    uint32_t w = s->accum_w, h = s->accum_h, n = w * h;
    if (!s->dn || s->dn_w != w || s->dn_h != h) {
        if (s->dn) cudaFree(s->dn);
        s->dn = nullptr;
        uint64_t need = 0;
        auto add = [&](uint64_t b) { uint64_t at = need; need += (b + 255) / 256 * 256; return at; };
        uint64_t o_c0 = add(16ull * n), o_c1 = add(16ull * n), o_v0 = add(4ull * n), o_v1 = add(4ull * n),
                 o_vf = add(4ull * n), o_a = add(16ull * n), o_n = add(16ull * n), o_rgb = add(12ull * n);
        (void)o_rgb;
        TRT_CUDA(c, cudaMalloc(&s->dn, need));
        char* b = (char*)s->dn;
        s->D = DenoiseBufs{{(float4*)(b + o_c0), (float4*)(b + o_c1)}, {(float*)(b + o_v0), (float*)(b + o_v1)},
                           (float*)(b + o_vf), (float4*)(b + o_a), (float4*)(b + o_n)};
        s->dn_rgb = (float*)(b + o_rgb);
        s->dn_w = w;
        s->dn_h = h;
    }
    const int blk = 256;
    uint32_t grid = (n + blk - 1) / blk;
    if (ms) TRT_CUDA(c, cudaEventRecord(c->t0, st));
    k_dn_prep<<<grid, blk, 0, st>>>(s->accum, n, s->D);
    uint32_t src = 0;
    for (uint32_t it = 0; it < iterations; ++it) {
        k_dn_var3<<<grid, blk, 0, st>>>(s->D.var[src], s->D.var_f, w, h);
        k_dn_atrous<<<grid, blk, 0, st>>>(s->D, src, w, h, 1 << it);
        src ^= 1u;
    }
    k_dn_remod<<<grid, blk, 0, st>>>(s->D, src, n, s->dn_rgb);
    if (ms) TRT_CUDA(c, cudaEventRecord(c->t1, st));
    TRT_CUDA(c, cudaGetLastError());
    TRT_CUDA(c, cudaMemcpyAsync(rgb_host, s->dn_rgb, 12ull * n, cudaMemcpyDeviceToHost, st));
    TRT_CUDA(c, cudaStreamSynchronize(st));
    if (ms) cudaEventElapsedTime(ms, c->t0, c->t1);
    return TRT_OK;
}

int trt_scene_read(trt_scene* s, uint32_t which, uint64_t offset, void* dst, uint64_t bytes) {
    if (!s) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    const void* base = which < 5 ? s->buf[which] : (const void*)s->env;
    uint64_t size = which < 5 ? s->bytes[which] : (uint64_t)s->env_w * s->env_h * 8;
    if (which > 5 || !dst || offset + bytes > size || offset + bytes < offset)
        return fail(c, TRT_EINVAL, "trt_scene_read: the range is not inside the buffer");
    cudaSetDevice(c->device);
    TRT_CUDA(c, cudaMemcpyAsync(dst, (const char*)base + offset, bytes, cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    return TRT_OK;
}

int trt_sky_bake(trt_ctx* c, const trt_atmosphere* a, float* texels_host, float* tables_host, trt_sky_result* out) {
    if (!c || !a) return TRT_EINVAL;
    cudaSetDevice(c->device);
    std::string err;
    int rc = sky_bake(&c->sky, c->device, c->stream, *a, texels_host, tables_host, out, &err);
    return rc ? fail(c, rc, err) : TRT_OK;
}

// lib.rs:947-1010 bake_sky + SkyBaked::write on the device, in place: the texels, the CDF, the sun's colour, Params.
int trt_scene_set_sky(trt_scene* s, const trt_atmosphere* a, int32_t sun_light, float env_nee_floor, uint32_t* P,
                      trt_sky_result* out) {
    if (!s || !a || !P) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    if (a->width != s->env_w || a->height != s->env_h)
        return fail(c, TRT_EINVAL, "trt_scene_set_sky: the scene's environment is not width x height");
    uint64_t cdf_words = (uint64_t)a->height + (uint64_t)a->width * a->height;
    uint64_t cdf_at = (uint64_t)P[P_WORD_FIRST] * 4;
    if (cdf_at + cdf_words * 4 > s->bytes[4] || cdf_at + cdf_words * 4 < cdf_at)
        return fail(c, TRT_EINVAL, "trt_scene_set_sky: the CDF's section does not fit in the words");
    uint64_t light_at = 0;
    if (sun_light >= 0) {
        if ((uint32_t)sun_light >= P[P_COUNTS]) return fail(c, TRT_EINVAL, "trt_scene_set_sky: no such light");
        light_at = ((uint64_t)P[P_TABLE_FIRST + 2] + (uint64_t)sun_light * 5 + 2) * 16;
        if (light_at + 16 > s->bytes[3]) return fail(c, TRT_EINVAL, "trt_scene_set_sky: the light is not in the tables");
    }
    cudaSetDevice(c->device);
    trt_sky_result r{};
    std::string err;
    int rc = sky_bake(&c->sky, c->device, c->stream, *a, nullptr, nullptr, &r, &err);
    if (rc) return fail(c, rc, err);
    // lib.rs:920: each row's sin(theta) as the host prep computes it, so that the CDF rounds the same.
    std::vector<float> sin_rows(a->height);
    for (uint32_t y = 0; y < a->height; ++y)
        sin_rows[y] = std::sin((((float)y) + 0.5f) / (float)a->height * 3.14159265358979323846f);
    rc = sky_env(c->sky, c->stream, sin_rows.data(), s->env, (float*)((char*)s->buf[4] + cdf_at), &r, &err);
    if (rc) return fail(c, rc, err);
    if (sun_light >= 0) {
        float col[4] = {r.sun_illuminance[0], r.sun_illuminance[1], r.sun_illuminance[2], 0.0f};
        TRT_CUDA(c, cudaMemcpyAsync((char*)s->buf[3] + light_at, col, 16, cudaMemcpyHostToDevice, c->stream));
        if (s->host[3].size() >= light_at + 16) std::memcpy(s->host[3].data() + light_at, col, 16);
        TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    auto put = [&](int w, float v) { std::memcpy(&P[w], &v, 4); };
    put(P_ENV, 1.0f);
    put(P_ENV + 1, (float)a->width);
    put(P_ENV + 2, (float)a->height);
    put(P_SKY + 3, r.horizon_v);
    P[P_COUNTS2 + 1] = r.brightest >= env_nee_floor ? 1u : 0u;
    if (out) *out = r;
    return TRT_OK;
}

int trt_deform_setup(trt_scene* s, const trt_deform_desc* desc) {
    if (!s) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    if (s->deformed) return fail(c, TRT_EINVAL, "trt_deform_setup: set up before the first deformation (the tree checks read the host copies)");
    SceneBuffers sb{{s->buf[0], s->buf[1], s->buf[2], s->buf[3], s->buf[4]},
                    {s->bytes[0], s->bytes[1], s->bytes[2], s->bytes[3], s->bytes[4]}, c->stream, s->host};
    DeformState* st = nullptr;
    std::string err;
    int rc = deform_setup(&st, sb, desc, err);
    if (rc) return fail(c, rc, err);
    deform_free(s->deform);
    s->deform = st;
    s->deform_stale = false;
    return TRT_OK;
}

int trt_deform(trt_scene* s, const uint32_t params[TRT_PARAMS_WORDS], const float* palette_rows, uint32_t n_matrices,
               uint32_t flags, trt_deform_stats* stats) {
    if (!s || !params) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    if (!s->deform) return fail(c, TRT_EINVAL, "trt_deform: no trt_deform_setup");
    if (s->deform_stale) return fail(c, TRT_EINVAL, "trt_deform: the nodes were written after trt_deform_setup: set up again");
    int rc = check_params(s, params);
    if (rc) return rc;
    SceneBuffers sb{{s->buf[0], s->buf[1], s->buf[2], s->buf[3], s->buf[4]},
                    {s->bytes[0], s->bytes[1], s->bytes[2], s->bytes[3], s->bytes[4]}, c->stream, s->host};
    std::string err;
    s->deformed = true;
    s->deform_gen++;
    rc = deform_run(s->deform, sb, params, palette_rows, n_matrices, flags, stats, err);
    if (rc) return fail(c, rc, err);
    if (s->wide.ready() && s->wide.key_matches(params)) {
        // A wide BVH in use follows the deformation at once (one built later is refit when it is built).
        if (stats) TRT_CUDA(c, cudaEventRecord(c->t0, c->stream));
        rc = refit_wide(s, params);
        if (rc) return rc;
        if (stats) {
            TRT_CUDA(c, cudaEventRecord(c->t1, c->stream));
            TRT_CUDA(c, cudaEventSynchronize(c->t1));
            cudaEventElapsedTime(&stats->wide_ms, c->t0, c->t1);
            uint32_t errors = 0;
            if (deform_errors(s->deform, c->stream, &errors) != TRT_OK) return fail(c, TRT_ECUDA, "trt_deform: reading the errors");
            stats->errors |= errors;
            if (errors) return fail(c, TRT_EGUARD, "trt_deform: the wide BVH's refit met an index out of its buffers");
        }
    }
    return TRT_OK;
}

int trt_render(trt_scene* s, const uint32_t params[TRT_PARAMS_WORDS], uint32_t first_sample, uint32_t spp,
               uint32_t flags, float* accum_host, trt_stats* stats) {
    if (!s || !params) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    int rc = check_params(s, params);
    if (rc) return rc;
    Params P;
    std::memcpy(P.w, params, sizeof(P.w));
    uint32_t w = P.w[P_SIZE], h = P.w[P_SIZE + 1];
    const bool async_back = (flags & TRT_RENDER_ASYNC_READBACK) != 0 && accum_host != nullptr;
    if (async_back && (flags & TRT_RENDER_ACCUMULATE))
        return fail(c, TRT_EINVAL, "TRT_RENDER_ASYNC_READBACK renders into a second accum: it cannot accumulate");
    if (!s->accum || s->accum_w != w || s->accum_h != h) {
        // (a size change waits for the read-backs in flight from the old buffers)
        TRT_CUDA(c, cudaStreamSynchronize(c->copy_stream));
        if (s->accum) cudaFree(s->accum);
        if (s->accum_alt) cudaFree(s->accum_alt);
        s->accum = s->accum_alt = nullptr;
        TRT_CUDA(c, cudaMalloc(&s->accum, 80ull * w * h));
        s->accum_w = w;
        s->accum_h = h;
        flags &= ~TRT_RENDER_ACCUMULATE;
    }
    if (async_back) {
        // Render into the other buffer, once its own last read-back is done; it becomes the accum.
        if (!s->accum_alt) TRT_CUDA(c, cudaMalloc(&s->accum_alt, 80ull * w * h));
        if (!s->copied) TRT_CUDA(c, cudaEventCreateWithFlags(&s->copied, cudaEventDisableTiming));
        if (!s->copied_alt) TRT_CUDA(c, cudaEventCreateWithFlags(&s->copied_alt, cudaEventDisableTiming));
        std::swap(s->accum, s->accum_alt);
        std::swap(s->copied, s->copied_alt);
    }
    // The accum may still be read back to the host by an earlier asynchronous render: wait for it on the device.
    if (s->copied) TRT_CUDA(c, cudaStreamWaitEvent(c->stream, s->copied, 0));
    if (!(flags & TRT_RENDER_ACCUMULATE)) TRT_CUDA(c, cudaMemsetAsync(s->accum, 0, 80ull * w * h, c->stream));
    unsigned long long before[T_COUNT] = {0};
    if (stats) {
        TRT_CUDA(c, cudaMemcpyAsync(before, s->totals, sizeof(before), cudaMemcpyDeviceToHost, c->stream));
        TRT_CUDA(c, cudaEventRecord(c->t0, c->stream));
    }
    uint64_t launches0 = s->launches;
    bool count = (flags & TRT_RENDER_COUNT) != 0, binary = (flags & TRT_RENDER_WIDE) == 0;
    if (!binary) {
        rc = ensure_wide(s, params);
        if (rc) return rc;
    }
    if (spp > 0) {
        if (count) rc = binary ? render_waves<true, false>(s, P, first_sample, spp, flags) : render_waves<true, true>(s, P, first_sample, spp, flags);
        else rc = binary ? render_waves<false, false>(s, P, first_sample, spp, flags) : render_waves<false, true>(s, P, first_sample, spp, flags);
        if (rc) return rc;
    }
    s->renders++;
    if (async_back) {
        // The read-back on the copy stream, after the render; the next render writes the other buffer meanwhile.
        TRT_CUDA(c, cudaEventRecord(c->copy_mark, c->stream));
        TRT_CUDA(c, cudaStreamWaitEvent(c->copy_stream, c->copy_mark, 0));
        TRT_CUDA(c, cudaMemcpyAsync(accum_host, s->accum, 80ull * w * h, cudaMemcpyDeviceToHost, c->copy_stream));
        TRT_CUDA(c, cudaEventRecord(s->copied, c->copy_stream));
    } else if (accum_host) {
        TRT_CUDA(c, cudaMemcpyAsync(accum_host, s->accum, 80ull * w * h, cudaMemcpyDeviceToHost, c->stream));
    }
    if (stats) {
        unsigned long long after[T_COUNT];
        TRT_CUDA(c, cudaEventRecord(c->t1, c->stream));
        TRT_CUDA(c, cudaMemcpyAsync(after, s->totals, sizeof(after), cudaMemcpyDeviceToHost, c->stream));
        TRT_CUDA(c, cudaStreamSynchronize(c->stream));
        float ms = 0;
        cudaEventElapsedTime(&ms, c->t0, c->t1);
        stats->closest_rays = after[T_CLOSEST] - before[T_CLOSEST];
        stats->shadow_rays = after[T_SHADOW] - before[T_SHADOW];
        stats->paths = after[T_PATHS] - before[T_PATHS];
        stats->guard_trips = (uint32_t)(after[T_GUARD] - before[T_GUARD]);
        stats->device_ms = ms;
        stats->launches = (uint32_t)(s->launches - launches0);
        if (stats->guard_trips) return fail(c, TRT_EGUARD, "a traversal stopped at its iteration limit");
    } else if (accum_host && !async_back) {
        TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return TRT_OK;
}

int trt_accum_device_ptr(trt_scene* s, void** ptr, uint64_t* bytes) {
    if (!s || !ptr) return TRT_EINVAL;
    *ptr = s->accum;
    if (bytes) *bytes = 80ull * s->accum_w * s->accum_h;
    return TRT_OK;
}

int trt_accum_read(trt_scene* s, float* accum_host, uint64_t bytes) {
    if (!s || !accum_host) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    if (bytes != 80ull * s->accum_w * s->accum_h) return fail(c, TRT_EINVAL, "trt_accum_read: wrong size");
    cudaSetDevice(c->device);
    TRT_CUDA(c, cudaMemcpyAsync(accum_host, s->accum, bytes, cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    return TRT_OK;
}

int trt_accum_copy(trt_scene* s, void* dst_device, uint64_t bytes) {
    if (!s || !dst_device) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    if (!s->accum || bytes != 80ull * s->accum_w * s->accum_h) return fail(c, TRT_EINVAL, "trt_accum_copy: wrong size");
    cudaSetDevice(c->device);
    TRT_CUDA(c, cudaMemcpyAsync(dst_device, s->accum, bytes, cudaMemcpyDeviceToDevice, c->stream));
    TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    return TRT_OK;
}

int trt_trace(trt_scene* s, const uint32_t params[TRT_PARAMS_WORDS], const trt_ray* rays, uint64_t n, uint32_t flags,
              trt_hit* hits) {
    if (!s || !params || (!rays && n) || (!hits && n)) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    int rc = check_params(s, params);
    if (rc) return rc;
    if (n == 0) return TRT_OK;
    Params P;
    std::memcpy(P.w, params, sizeof(P.w));
    trt_ray* dr = nullptr;
    trt_hit* dh = nullptr;
    TRT_CUDA(c, cudaMalloc(&dr, sizeof(trt_ray) * n));
    cudaError_t e = cudaMalloc(&dh, sizeof(trt_hit) * n);
    if (e != cudaSuccess) { cudaFree(dr); return cuda_fail(c, e, "trt_trace"); }
    e = cudaMemcpyAsync(dr, rays, sizeof(trt_ray) * n, cudaMemcpyHostToDevice, c->stream);
    bool binary = (flags & TRT_RENDER_WIDE) == 0;
    bool count = (flags & TRT_RENDER_COUNT) != 0;
    if (e == cudaSuccess && !binary) {
        rc = ensure_wide(s, params);
        if (rc) {
            cudaFree(dr);
            cudaFree(dh);
            return rc;
        }
    }
    DScene S = scene_view(s);
    Walk wk{S, s->wide.view(), P.w[P_MOTION + 2], P.w[P_MOTION + 3]};
    unsigned grid = (unsigned)((n + 127) / 128);
    if (e == cudaSuccess) {
        if (count) {
            if (binary) k_trace<true, false><<<grid, 128, 0, c->stream>>>(P, wk, dr, n, dh, s->totals);
            else k_trace<true, true><<<grid, 128, 0, c->stream>>>(P, wk, dr, n, dh, s->totals);
        } else {
            if (binary) k_trace<false, false><<<grid, 128, 0, c->stream>>>(P, wk, dr, n, dh, s->totals);
            else k_trace<false, true><<<grid, 128, 0, c->stream>>>(P, wk, dr, n, dh, s->totals);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hits, dh, sizeof(trt_hit) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(dr);
    cudaFree(dh);
    if (e != cudaSuccess) return cuda_fail(c, e, "trt_trace");
    return TRT_OK;
}

int trt_math_eval(trt_ctx* c, uint32_t fn, const float* x, const float* y, uint64_t n, float* out) {
    if (!c) return TRT_EINVAL;
    if (fn > TRT_MATH_ATAN2 || (n && (!x || !out)) || (fn == TRT_MATH_ATAN2 && n && !y))
        return fail(c, TRT_EINVAL, "trt_math_eval: a bad function or a null array");
    if (n == 0) return TRT_OK;
    cudaSetDevice(c->device);
    float* d = nullptr;
    TRT_CUDA(c, cudaMalloc(&d, 12ull * n));
    cudaError_t e = cudaMemcpyAsync(d, x, 4ull * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && y) e = cudaMemcpyAsync(d + n, y, 4ull * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        k_math_eval<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(fn, d, y ? d + n : nullptr, n, d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d + 2 * n, 4ull * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(c, e, "trt_math_eval");
    return TRT_OK;
}

int trt_scene_totals(trt_scene* s, trt_totals* out) {
    if (!s || !out) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    unsigned long long t[T_COUNT];
    TRT_CUDA(c, cudaMemcpyAsync(t, s->totals, sizeof(t), cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    auto drain = [&](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, double& acc) {
        for (auto& e : v) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) acc += ms;
            s->ev_free.push_back(e);
        }
        v.clear();
    };
    drain(s->ev_extend, s->extend_ms);
    drain(s->ev_shadow, s->shadow_ms);
    drain(s->ev_shade, s->shade_ms);
    drain(s->ev_sort, s->sort_ms);
    out->closest_rays = t[T_CLOSEST];
    out->shadow_rays = t[T_SHADOW];
    out->paths = t[T_PATHS];
    out->node_visits = t[T_E_NODES];
    out->tri_tests = t[T_E_TRIS];
    out->unit_entries = t[T_E_UNITS];
    out->shadow_node_visits = t[T_S_NODES];
    out->shadow_tri_tests = t[T_S_TRIS];
    out->shadow_unit_entries = t[T_S_UNITS];
    out->guard_trips = t[T_GUARD];
    out->renders = s->renders;
    out->launches = s->launches;
    out->extend_ms = s->extend_ms;
    out->shadow_ms = s->shadow_ms;
    out->shade_ms = s->shade_ms;
    out->sort_ms = s->sort_ms;
    out->extend_launches = s->extend_launches;
    out->shadow_launches = s->shadow_launches;
    return TRT_OK;
}

void trt_scene_reset_totals(trt_scene* s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    cudaMemsetAsync(s->totals, 0, sizeof(unsigned long long) * T_COUNT, s->ctx->stream);
    cudaStreamSynchronize(s->ctx->stream);
    for (auto* v : {&s->ev_extend, &s->ev_shadow, &s->ev_shade, &s->ev_sort}) {
        for (auto& e : *v) s->ev_free.push_back(e);
        v->clear();
    }
    s->extend_ms = s->shadow_ms = s->shade_ms = s->sort_ms = 0;
    s->extend_launches = s->shadow_launches = s->renders = s->launches = 0;
}

void trt_scene_set_profiling(trt_scene* s, int on) {
    if (s) s->profiling = on;
}

int trt_timer_start(trt_ctx* c) {
    if (!c) return TRT_EINVAL;
    TRT_CUDA(c, cudaEventRecord(c->t0, c->stream));
    return TRT_OK;
}

int trt_timer_stop(trt_ctx* c, float* ms) {
    if (!c || !ms) return TRT_EINVAL;
    // (after the read-backs still running on the copy stream, too)
    TRT_CUDA(c, cudaEventRecord(c->copy_mark, c->copy_stream));
    TRT_CUDA(c, cudaStreamWaitEvent(c->stream, c->copy_mark, 0));
    TRT_CUDA(c, cudaEventRecord(c->t1, c->stream));
    TRT_CUDA(c, cudaEventSynchronize(c->t1));
    TRT_CUDA(c, cudaEventElapsedTime(ms, c->t0, c->t1));
    return TRT_OK;
}

int trt_synchronize(trt_ctx* c) {
    if (!c) return TRT_EINVAL;
    TRT_CUDA(c, cudaStreamSynchronize(c->stream));
    TRT_CUDA(c, cudaStreamSynchronize(c->copy_stream));
    return TRT_OK;
}

int trt_render_noalloc(const trt_scene_desc* dev, const uint32_t params[TRT_PARAMS_WORDS], uint32_t first_sample,
                       uint32_t spp, uint32_t flags, float* accum_device, void* stream, char* err, size_t err_len) {
    if (err && err_len) err[0] = 0;
    if (!dev || !params || !accum_device) return na_fail(err, err_len, TRT_EINVAL, "a null argument");
    // (Its hits are always shaded unsorted, so TRT_RENDER_UNSORTED_HITS is accepted and changes nothing.)
    if (flags & ~(TRT_RENDER_ACCUMULATE | TRT_RENDER_UNSORTED_HITS))
        return na_fail(err, err_len, TRT_EINVAL, "flags: TRT_RENDER_ACCUMULATE and TRT_RENDER_UNSORTED_HITS only");
    Params P;
    std::memcpy(P.w, params, sizeof(P.w));
    // The same checks as trt_render's, against the caller's buffers, all before the first CUDA call.
    const uint64_t nb[5] = {dev->vertices_bytes, dev->leaves_bytes, dev->nodes_bytes, dev->tables_bytes, dev->words_bytes};
    const void* ptrs[5] = {dev->vertices, dev->leaves, dev->nodes, dev->tables, dev->words};
    const uint64_t unit[5] = {48, 48, 32, 16, 4};
    for (int k = 0; k < 5; ++k)
        if (!ptrs[k] || nb[k] == 0 || nb[k] % unit[k] != 0)
            return na_fail(err, err_len, TRT_EINVAL, "scene buffer " + std::to_string(k) + ": no data, or not whole records");
    if (!dev->env_half || dev->env_w == 0 || dev->env_h == 0) return na_fail(err, err_len, TRT_EINVAL, "no environment texels");
    for (int k = 0; k < 12; ++k)
        if (P.w[P_TABLE_FIRST + k] > nb[3] / 16) return na_fail(err, err_len, TRT_EINVAL, "Params.table_first names a vec4 past the tables");
    for (int k = 0; k < 5; ++k)
        if (P.w[P_WORD_FIRST + k] > nb[4] / 4) return na_fail(err, err_len, TRT_EINVAL, "Params.word_first names a word past the words");
    uint32_t w = P.w[P_SIZE], h = P.w[P_SIZE + 1];
    if (w == 0 || h == 0) return na_fail(err, err_len, TRT_EINVAL, "Params.size: an empty image");
    // Path slots in 64 bits: a size whose 32-bit count would wrap is refused like any other too large.
    const uint64_t slots64 = ((uint64_t)w + 7u) / 8u * (((uint64_t)h + 3u) / 4u) * 32u;
    if (slots64 > NOALLOC_SLOTS)
        return na_fail(err, err_len, TRT_EINVAL, "image too large for the no-allocation render: " + std::to_string(w) + " x " +
                       std::to_string(h) + " needs " + std::to_string(slots64) + " path slots (8 x 4 tiles), the most is " +
                       std::to_string(NOALLOC_SLOTS) + " (256 x 256)");
    const uint32_t n_idx = (uint32_t)slots64;
    if (P.w[P_COUNTS + 2] >= MAX_DEPTH - 1) return na_fail(err, err_len, TRT_EINVAL, "Params.counts.z (max bounces) must be below 63");
    if (P.w[P_COUNTS2] > MAX_DIR_LIGHTS) return na_fail(err, err_len, TRT_EINVAL, "more than 4 directional lights");
    if (P.w[P_COUNTS] != P.w[P_COUNTS2]) return na_fail(err, err_len, TRT_EINVAL, "local lights are not part of this pass");
    if (P.w[P_MOTION + 3] > 0 && (uint64_t)P.w[P_MOTION + 2] >= nb[2] / 32)
        return na_fail(err, err_len, TRT_EINVAL, "Params.motion.z names a node past the nodes");
    if (P.w[P_ENV] == 0x3f800000u && ((uint32_t)bf(P.w[P_ENV + 1]) != dev->env_w || (uint32_t)bf(P.w[P_ENV + 2]) != dev->env_h))
        return na_fail(err, err_len, TRT_EINVAL, "Params.env's size is not the environment's");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return na_fail(err, err_len, TRT_ECUDA, cudaGetErrorString(e));
    int rc = noalloc_setup(device, err, err_len);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t K = std::max(1u, std::min(spp, NOALLOC_SLOTS / n_idx));
    uint32_t slots = n_idx * K;
    // The array's parts, as wave_ensure lays out an allocation.
    uint8_t* b = g_noalloc_ptr[device];
    uint64_t at = 0;
    auto take = [&](uint64_t bytes) { uint8_t* p = b + at; at += na_round(bytes); return p; };
    PathBufs B;
    B.o = (float4*)take(16ull * NOALLOC_SLOTS);
    B.d = (float4*)take(16ull * NOALLOC_SLOTS);
    B.thr = (float4*)take(16ull * NOALLOC_SLOTS);
    B.rad = (float4*)take(16ull * NOALLOC_SLOTS);
    B.alb = (float4*)take(16ull * NOALLOC_SLOTS);
    B.nrm = (float4*)take(16ull * NOALLOC_SLOTS);
    B.mis_x = (float4*)take(16ull * NOALLOC_SLOTS);
    B.mis_n = (float4*)take(16ull * NOALLOC_SLOTS);
    B.nee = (float4*)take(16ull * NOALLOC_SLOTS * N_SLOTS);
    B.nee_thr = (float4*)take(16ull * NOALLOC_SLOTS);
    B.vis = (uint32_t*)take(4ull * NOALLOC_SLOTS);
    B.n = NOALLOC_SLOTS;
    Queues Q;
    Q.q[0] = (uint32_t*)take(4ull * NOALLOC_SLOTS);
    Q.q[1] = (uint32_t*)take(4ull * NOALLOC_SLOTS);
    Q.hit_a = (float4*)take(16ull * NOALLOC_SLOTS);
    Q.hit_b = (uint2*)take(8ull * NOALLOC_SLOTS);
    Q.so = (float4*)take(16ull * NOALLOC_SHADOW);
    Q.sd = (float4*)take(16ull * NOALLOC_SHADOW);
    Q.sp = (uint32_t*)take(4ull * NOALLOC_SHADOW);
    uint64_t cnt_bytes = 4ull * (MAX_DEPTH * CNT_STRIDE + CNT_STRIDE);
    Q.cnt = (uint32_t*)take(cnt_bytes);
    Q.totals = (unsigned long long*)take(8ull * T_COUNT);
    B.job = (uint32_t*)take(4ull * NOALLOC_SLOTS);
    Job* jobs = (Job*)take(sizeof(Job));
    uint32_t n_dir = P.w[P_COUNTS2];
    uint32_t caps[3] = {slots * std::max(1u, n_dir), slots, slots};
    Q.shadow_cap = caps[0] + caps[1] + caps[2];
    Q.class_base[0] = 0;
    Q.class_base[1] = caps[0];
    Q.class_base[2] = caps[0] + caps[1];
    for (int k = 0; k < 3; ++k) Q.class_cap[k] = caps[k];
    DScene S;
    S.vertices = (const float4*)dev->vertices;
    S.leaves = (const float4*)dev->leaves;
    S.nodes = (const uint4*)dev->nodes;
    S.tables = (const uint4*)dev->tables;
    S.words = (const uint32_t*)dev->words;
    S.env = (const ushort4*)dev->env_half;
    S.env_w = dev->env_w;
    S.env_h = dev->env_h;
    S.n_nodes = nb[2] / 32;
    S.n_tris = nb[1] / 48;
    S.n_table_vec4 = nb[3] / 16;
    S.n_words = nb[4] / 4;
    Walk wk{S, WideView{}, P.w[P_MOTION + 2], P.w[P_MOTION + 3]};
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return na_fail(err, err_len, TRT_ECUDA, cudaGetErrorString(e));
    const int blk = 128;
    int g_ext = grid_for((const void*)k_extend<false, false, false>, blk, sms);
    int g_sha = grid_for((const void*)k_shadow<false, false, false>, blk, sms);
    uint32_t last = P.w[P_COUNTS + 2];
    // What must start at zero: the accum (unless accumulating), the totals, each wave's counters.
    if (!(flags & TRT_RENDER_ACCUMULATE)) e = cudaMemsetAsync(accum_device, 0, 80ull * w * h, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(Q.totals, 0, 8ull * T_COUNT, st);
    for (uint32_t s0 = 0; s0 < spp && e == cudaSuccess; s0 += K) {
        uint32_t k = std::min(K, spp - s0);
        e = cudaMemsetAsync(Q.cnt, 0, cnt_bytes, st);
        if (e != cudaSuccess) break;
        uint32_t n = n_idx * k;
        Job job{P, wk, (float4*)accum_device, 0u, n_idx, k, first_sample + s0};
        k_put_job<<<1, 128, 0, st>>>(job, jobs, 0u);
        k_raygen<<<(n + blk - 1) / blk, blk, 0, st>>>(jobs, 1u, B, Q, n, nullptr);
        for (uint32_t depth = 0; depth <= last; ++depth) {
            uint32_t* queue = Q.q[depth & 1u];
            k_extend<false, false, false><<<g_ext, blk, 0, st>>>(jobs, job, B, Q, depth, queue);
            k_shade<false><<<(n + blk - 1) / blk, blk, 0, st>>>(jobs, job, B, Q, depth, queue, Q.q[(depth + 1u) & 1u]);
            k_shadow<false, false, false><<<g_sha, blk, 0, st>>>(jobs, job, B, Q, depth, nullptr);
            k_resolve<false><<<(n + blk - 1) / blk, blk, 0, st>>>(jobs, job, B, Q, depth, queue);
        }
        k_accumulate<<<dim3((n_idx + blk - 1) / blk, 1), blk, 0, st>>>(jobs, B);
        k_tally<<<1, 32, 0, st>>>(Q, last + 1, w * h * k, nullptr);
        e = cudaGetLastError();
    }
    // The walks' guard trips (the reference's loop guard, gpu.rs:4199-4205): the call waits for its work to read them
    // (a pageable copy of one word, no allocation).
    unsigned long long guard_trips = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&guard_trips, Q.totals + T_GUARD, sizeof(guard_trips), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(err, err_len, TRT_ECUDA, cudaGetErrorString(e));
    if (guard_trips)
        return na_fail(err, err_len, TRT_EGUARD, std::to_string(guard_trips) + " traversals stopped at their iteration limit");
    return TRT_OK;
}

}  // extern "C"

#include "serve.cuh"
#include "emitters.cuh"
#include "ltree.cuh"
