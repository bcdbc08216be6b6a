// The light tree built on the device (renderer/src/ltree.rs:339-386 grow, 405-470 build_with; the emitter order and
// codes of lib.rs:393-418): from the emitter records as a resident scene's tables hold them now, so that emitters
// that moved (their records written, or their instances deformed) are sampled by a tree over where they are. Included
// by pathtrace.cu after emitters.cuh; trt_scene_weigh_emitters then makes the nodes' powers, the CDF and the header.
//
// The build is the reference's: the emitters of positive power that are neither nominal nor moving, each a leaf of
// its own (LEAF_MAX 1), split at the median of their centroids along the widest axis of the centroids' bounds, node by
// node; a node is its items' bounding sphere as half floats (encode / box_sphere) with their summed power, and the
// child word of ltree.rs. Laid out for the GPU: one launch per level, one block per node of the level (its items'
// bounds by block reductions, the median split by a bitonic sort of the node's items in shared memory). A node's index
// is where ltree.rs's stack would have put it: its right subtree is grown first, so a node split with its first free
// index at a places its children at a and a + 1, and their subtrees' first free indices are a + 2 (right) and
// a + 2 * (the right child's items) (left: each split of the right subtree took two). The split's order is total:
// the centroid's coordinate by f32::total_cmp's key, then the emitter's index, so the tree does not depend on the
// sort's order of equal keys; the host prep orders its splits the same way.
#pragma once

namespace trt_lt {

constexpr uint32_t LEAF = 0x80000000u, PATH_BITS = 26u, MIN_STATIC = 256u, MAX_ITEMS = 16384u, THREADS = 256u;
constexpr uint32_t EMITTER_MOVES = 0x80000000u, EMITTER_GONE = 2u, EMITTER_NOMINAL = 4u, NO_INST = 0xffffffffu;
constexpr uint32_t INSTANCE_VEC4 = 10u, MATERIAL_VEC4 = 18u, ROW_MATERIAL = 0xffffffu, OBJECT_STRIDE = 3u;

struct Item { float lo[3], hi[3], c[3], w; };
// A node of a level still to make: its items perm[a, b), its index, its subtree's first free index, depth, path.
struct Seg { uint32_t a, b, node, alloc, depth, path; };

struct Build {
    const uint4* tables;
    uint4* rw;
    const uint32_t* words;
    uint64_t n_tables, n_words;
    uint32_t n_emitters, list, entries, tree, tree_cap, instances, materials, objects, rows;
    Item* items;        // per emitter
    uint32_t* eligible; // per emitter: 1 if it goes into the tree
    uint32_t* perm;     // the tree's items (emitter indices), in the order the splits leave them
    uint32_t* rest;     // the emitters outside the tree, in index order
    uint32_t* code;     // per tree entry
    uint32_t* n_tree;   // the tree's items
    uint32_t* err;
};

__device__ __forceinline__ uint4 tget(const Build& B, uint64_t i) {
    if (i >= B.n_tables) {
        atomicOr(B.err, 1u);
        return make_uint4(0u, 0u, 0u, 0u);
    }
    return B.tables[i];
}
__device__ __forceinline__ void tput(const Build& B, uint64_t i, uint4 v) {
    if (i >= B.n_tables) {
        atomicOr(B.err, 1u);
        return;
    }
    B.rw[i] = v;
}

// binary32 -> binary16, round to nearest even (half::f16::from_f32), as the host prep's float_to_half.
__device__ __forceinline__ uint32_t f2h(float f) {
    uint32_t x = __float_as_uint(f);
    uint32_t sign = (x >> 16) & 0x8000u, exp = (x >> 23) & 0xffu, man = x & 0x7fffffu;
    if (exp == 0xffu) return sign | 0x7c00u | (man ? 0x200u : 0u);
    int32_t e = (int32_t)exp - 127 + 15;
    if (e >= 31) return sign | 0x7c00u;
    if (e <= 0) {
        if (e < -10) return sign;
        man |= 0x800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t hm = man >> shift, rem = man & ((1u << shift) - 1u), halfway = 1u << (shift - 1);
        if (rem > halfway || (rem == halfway && (hm & 1u))) hm++;
        return sign | hm;
    }
    uint32_t hm = man >> 13, rem = man & 0x1fffu;
    uint32_t out = sign | ((uint32_t)e << 10) | hm;
    if (rem > 0x1000u || (rem == 0x1000u && (hm & 1u))) out++;
    return out;
}
__device__ __forceinline__ float h2f(uint32_t h) {
    uint32_t s = (h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    if (e == 0) {
        if (m == 0) return __uint_as_float(s);
        float f = (float)m * (1.0f / 16777216.0f);
        return s ? -f : f;
    }
    if (e == 31) return __uint_as_float(s | 0x7f800000u | (m << 13));
    return __uint_as_float(s | ((e + 112u) << 23) | (m << 13));
}

// ltree.rs:121-137 encode of box_sphere: the box's bounding sphere, centre and radius as half floats (the radius
// grown by the centre's rounding and rounded up).
__device__ __forceinline__ uint2 box_sphere(const float lo[3], const float hi[3]) {
    float c[3];
    for (int k = 0; k < 3; ++k) c[k] = 0.5f * (lo[k] + hi[k]);
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    float r = 0.5f * sqrtf(dx * dx + dy * dy + dz * dz);
    float hc[3];
    for (int k = 0; k < 3; ++k) hc[k] = h2f(f2h(c[k]));
    float gx = hc[0] - c[0], gy = hc[1] - c[1], gz = hc[2] - c[2];
    float grow = sqrtf(gx * gx + gy * gy + gz * gz);
    uint32_t hr = f2h(r + grow);
    if (h2f(hr) < r + grow) hr = (hr + 1u) & 0xffffu;
    return make_uint2(f2h(hc[0]) | (f2h(hc[1]) << 16), f2h(hc[2]) | (hr << 16));
}

// f32::total_cmp as an unsigned key.
__device__ __forceinline__ uint32_t total_key(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Each emitter's item: its power (area x emissive luminance x its object's power, as emitter_weights.wgsl weighs it
// without the light LOD), the bounds of its triangle's vertices v0, v0 + e1, v0 + e2 (GpuEmitterTri::vertices,
// lib.rs:175-178) and their centroid; eligible when the power is positive and it is neither nominal nor moving.
__global__ void k_lt_items(Build B) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_emitters) return;
    uint64_t r = (uint64_t)B.list + (uint64_t)i * 4u;
    uint4 r0 = tget(B, r), r1 = tget(B, r + 1), r2 = tget(B, r + 2), r3 = tget(B, r + 3);
    float v0[3] = {__uint_as_float(r0.x), __uint_as_float(r0.y), __uint_as_float(r0.z)};
    float e1[3] = {__uint_as_float(r1.x), __uint_as_float(r1.y), __uint_as_float(r1.z)};
    float e2[3] = {__uint_as_float(r2.x), __uint_as_float(r2.y), __uint_as_float(r2.z)};
    float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
    float area = 0.5f * sqrtf(cx * cx + cy * cy + cz * cz);
    float w = 0.0f;
    bool ok = (r3.y & (EMITTER_GONE | EMITTER_NOMINAL)) == 0u && (r2.w & EMITTER_MOVES) == 0u && r1.w != NO_INST;
    if (ok) {
        uint4 info = tget(B, (uint64_t)B.instances + (uint64_t)r1.w * INSTANCE_VEC4 + 6u);
        uint64_t wi = (uint64_t)B.rows + ((uint64_t)info.w + r3.x) * 4u;
        uint32_t m = 0u;
        if (wi < B.n_words) m = B.words[wi] & ROW_MATERIAL;
        else atomicOr(B.err, 1u);
        uint4 em = tget(B, (uint64_t)B.materials + (uint64_t)m * MATERIAL_VEC4 + 1u);
        float power = __uint_as_float(tget(B, (uint64_t)B.objects + (uint64_t)info.y * OBJECT_STRIDE).w);
        w = area * (__uint_as_float(em.x) * 0.2126f + __uint_as_float(em.y) * 0.7152f + __uint_as_float(em.z) * 0.0722f) *
            power;
    }
    Item it;
    float vs[3][3];
    for (int k = 0; k < 3; ++k) {
        vs[0][k] = v0[k];
        vs[1][k] = v0[k] + e1[k];
        vs[2][k] = v0[k] + e2[k];
    }
    for (int k = 0; k < 3; ++k) {
        it.lo[k] = fminf(fminf(vs[0][k], vs[1][k]), vs[2][k]);
        it.hi[k] = fmaxf(fmaxf(vs[0][k], vs[1][k]), vs[2][k]);
        it.c[k] = (vs[0][k] + vs[1][k] + vs[2][k]) / 3.0f;
    }
    it.w = w;
    B.items[i] = it;
    B.eligible[i] = (ok && w > 0.0f) ? 1u : 0u;
}

// The eligible emitters in index order (perm[0, n)) and the others (rest), and the first's count (every emitter goes
// to rest when `tree` is 0): one block, running counts by chunks.
__global__ void __launch_bounds__(THREADS) k_lt_compact(Build B, uint32_t tree) {
    __shared__ uint32_t warp_sums[2][THREADS / 32u];
    __shared__ uint32_t base[2];
    if (threadIdx.x == 0) base[0] = base[1] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    for (uint32_t c0 = 0; c0 < B.n_emitters; c0 += THREADS) {
        uint32_t i = c0 + threadIdx.x;
        bool valid = i < B.n_emitters;
        bool in = valid && tree && B.eligible[i] != 0u;
        unsigned m_in = __ballot_sync(0xffffffffu, in), m_out = __ballot_sync(0xffffffffu, valid && !in);
        if (lane == 0) {
            warp_sums[0][wid] = (uint32_t)__popc(m_in);
            warp_sums[1][wid] = (uint32_t)__popc(m_out);
        }
        __syncthreads();
        uint32_t off_in = base[0], off_out = base[1];
        for (uint32_t w = 0; w < wid; ++w) {
            off_in += warp_sums[0][w];
            off_out += warp_sums[1][w];
        }
        const unsigned below = (1u << lane) - 1u;
        if (in && off_in + (uint32_t)__popc(m_in & below) < MAX_ITEMS) B.perm[off_in + __popc(m_in & below)] = i;
        if (valid && !in) B.rest[off_out + __popc(m_out & below)] = i;
        __syncthreads();
        if (threadIdx.x == 0)
            for (uint32_t w = 0; w < THREADS / 32u; ++w) {
                base[0] += warp_sums[0][w];
                base[1] += warp_sums[1][w];
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) *B.n_tree = base[0];
}

// One level: a block per node (segment). Its items' bounds and power, its sphere; a leaf's entry and code, or the
// median split (a bitonic sort of (key, emitter) pairs in shared memory) and its two children for the next level.
__global__ void __launch_bounds__(THREADS) k_lt_level(Build B, const Seg* __restrict__ segs, uint32_t n_segs,
                                                      Seg* __restrict__ next) {
    extern __shared__ unsigned long long sort_buf[];
    __shared__ float red[6][THREADS / 32u];
    __shared__ float red_w[THREADS / 32u];
    __shared__ int axis_s;
    const uint32_t si = blockIdx.x;
    if (si >= n_segs) return;
    const Seg sg = segs[si];
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    if (sg.b <= sg.a) {  // (no node here: the next level's children of a leaf)
        if (threadIdx.x == 0) {
            next[2 * si] = Seg{0, 0, 0, 0, 0, 0};
            next[2 * si + 1] = Seg{0, 0, 0, 0, 0, 0};
        }
        return;
    }
    const uint32_t len = sg.b - sg.a;
    // The items' bounds (min / max: exact in any order) and centroid bounds, then their power.
    float lo[3] = {3.4028235e38f, 3.4028235e38f, 3.4028235e38f}, hi[3] = {-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
    float clo[3] = {3.4028235e38f, 3.4028235e38f, 3.4028235e38f}, chi[3] = {-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
    float w = 0.0f;
    for (uint32_t k = threadIdx.x; k < len; k += THREADS) {
        const Item& it = B.items[B.perm[sg.a + k]];
        for (int d = 0; d < 3; ++d) {
            lo[d] = fminf(lo[d], it.lo[d]);
            hi[d] = fmaxf(hi[d], it.hi[d]);
            clo[d] = fminf(clo[d], it.c[d]);
            chi[d] = fmaxf(chi[d], it.c[d]);
        }
        w += it.w;
    }
    float vals[12] = {lo[0], lo[1], lo[2], clo[0], clo[1], clo[2], hi[0], hi[1], hi[2], chi[0], chi[1], chi[2]};
    float outv[12];
    for (int q = 0; q < 12; ++q) {
        float v = vals[q];
        for (int o = 16; o > 0; o >>= 1) {
            float u = __shfl_xor_sync(0xffffffffu, v, o);
            v = q < 6 ? fminf(v, u) : fmaxf(v, u);
        }
        if (lane == 0) red[q % 6][wid] = v;
        __syncthreads();
        float acc = red[q % 6][0];
        for (uint32_t k = 1; k < THREADS / 32u; ++k) acc = q < 6 ? fminf(acc, red[q % 6][k]) : fmaxf(acc, red[q % 6][k]);
        outv[q] = acc;
        __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (lane == 0) red_w[wid] = w;
    __syncthreads();
    float power = 0.0f;
    for (uint32_t k = 0; k < THREADS / 32u; ++k) power += red_w[k];
    for (int d = 0; d < 3; ++d) {
        lo[d] = outv[d];
        clo[d] = outv[3 + d];
        hi[d] = outv[6 + d];
        chi[d] = outv[9 + d];
    }
    uint32_t word;
    if (len <= 1u) {
        word = LEAF | sg.a;
        if (threadIdx.x == 0) {
            if (sg.depth > PATH_BITS) atomicOr(B.err, 2u);
            B.code[sg.a] = ((sg.depth + 1u) << PATH_BITS) | sg.path;
            next[2 * si] = Seg{0, 0, 0, 0, 0, 0};
            next[2 * si + 1] = Seg{0, 0, 0, 0, 0, 0};
        }
    } else {
        // ltree.rs:368-375: the widest axis of the centroids' bounds (the last of equals), the median split.
        if (threadIdx.x == 0) {
            int ax = 0;
            for (int d = 1; d < 3; ++d)
                if ((chi[d] - clo[d]) >= (chi[ax] - clo[ax])) ax = d;
            axis_s = ax;
        }
        __syncthreads();
        const int ax = axis_s;
        uint32_t n2 = 1u;
        while (n2 < len) n2 <<= 1;
        for (uint32_t k = threadIdx.x; k < n2; k += THREADS) {
            unsigned long long key = ~0ull;
            if (k < len) {
                uint32_t e = B.perm[sg.a + k];
                key = ((unsigned long long)total_key(B.items[e].c[ax]) << 32) | e;
            }
            sort_buf[k] = key;
        }
        __syncthreads();
        for (uint32_t size = 2u; size <= n2; size <<= 1) {
            for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                for (uint32_t k = threadIdx.x; k < n2; k += THREADS) {
                    uint32_t j = k ^ stride;
                    if (j > k) {
                        unsigned long long x = sort_buf[k], y = sort_buf[j];
                        bool up = (k & size) == 0u;
                        if ((x > y) == up) {
                            sort_buf[k] = y;
                            sort_buf[j] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t k = threadIdx.x; k < len; k += THREADS) B.perm[sg.a + k] = (uint32_t)(sort_buf[k] & 0xffffffffu);
        const uint32_t mid = len / 2u, len_r = len - mid;
        word = sg.alloc;
        if (threadIdx.x == 0) {
            next[2 * si] = Seg{sg.a, sg.a + mid, sg.alloc, sg.alloc + 2u * len_r, sg.depth + 1u, sg.path};
            next[2 * si + 1] = Seg{sg.a + mid, sg.b, sg.alloc + 1u, sg.alloc + 2u, sg.depth + 1u, sg.path | (1u << sg.depth)};
        }
    }
    if (threadIdx.x == 0) {
        if (sg.node >= B.tree_cap) {
            atomicOr(B.err, 4u);
        } else {
            uint2 sph = box_sphere(lo, hi);
            tput(B, (uint64_t)B.tree + sg.node, make_uint4(sph.x, sph.y, __float_as_uint(power), word));
        }
    }
}

// The emitter table in the tree's leaf order, then the other emitters in index order (lib.rs:393-402 emitter_order);
// each triangle's code: its path in the tree, or its entry's position (lib.rs:404-418), the moving flag kept.
__global__ void k_lt_order(Build B, uint32_t n_tree) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B.n_emitters) return;
    uint32_t e = k < n_tree ? B.perm[k] : B.rest[k - n_tree];
    uint4 ent = tget(B, (uint64_t)B.entries + k);
    ent.x = e;
    tput(B, (uint64_t)B.entries + k, ent);
    uint64_t r = (uint64_t)B.list + (uint64_t)e * 4u + 2u;
    uint4 r2 = tget(B, r);
    r2.w = (r2.w & EMITTER_MOVES) | (k < n_tree ? B.code[k] : k);
    tput(B, r, r2);
}

}  // namespace trt_lt

// ltree.rs:405-470 build on the device, with the emitter order and codes (lib.rs:393-418) and Params' tree words.
int trt_scene_build_light_tree(trt_scene* s, uint32_t* P, uint32_t* tree_nodes, float* ms) {
    using namespace trt_lt;
    if (!s || !P || !tree_nodes) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    *tree_nodes = 0;
    const uint32_t n = P[P_COUNTS + 1];
    const uint64_t tv = s->bytes[3] / 16;
    Build B{};
    B.n_emitters = n;
    B.tree = P[P_TABLE_FIRST + 0];
    B.tree_cap = P[P_TABLE_FIRST + 1] > B.tree ? P[P_TABLE_FIRST + 1] - B.tree : 0u;
    B.materials = P[P_TABLE_FIRST + 1];
    B.entries = P[P_TABLE_FIRST + 4];
    B.objects = P[P_TABLE_FIRST + 6];
    B.instances = P[P_TABLE_FIRST + 7];
    B.list = P[P_TABLE_FIRST + 11];
    B.rows = P[P_WORD_FIRST + 3];
    if (n == 0) return TRT_OK;
    if ((uint64_t)B.list + 4ull * n > tv || (uint64_t)B.entries + n > tv || (uint64_t)B.tree + B.tree_cap > tv)
        return fail(c, TRT_EINVAL, "trt_scene_build_light_tree: the emitter records, entries or tree are not inside the tables");
    cudaSetDevice(c->device);
    cudaStream_t st = c->stream;
    // Scratch: items, flags, the two orders, codes, counters, two levels of segments.
    const uint32_t max_levels = 16u;
    uint64_t need = 0;
    auto add = [&](uint64_t b) { uint64_t at = need; need += (b + 255) / 256 * 256; return at; };
    const uint64_t o_items = add(sizeof(Item) * n), o_elig = add(4ull * n), o_perm = add(4ull * MAX_ITEMS),
                   o_rest = add(4ull * n), o_code = add(4ull * MAX_ITEMS), o_cnt = add(16),
                   o_seg0 = add(sizeof(Seg) * (2ull << max_levels)), o_seg1 = add(sizeof(Seg) * (2ull << max_levels));
    void* scratch = nullptr;
    TRT_CUDA(c, cudaMalloc(&scratch, need));
    char* b = (char*)scratch;
    B.tables = (const uint4*)s->buf[3];
    B.rw = (uint4*)s->buf[3];
    B.words = (const uint32_t*)s->buf[4];
    B.n_tables = tv;
    B.n_words = s->bytes[4] / 4;
    B.items = (Item*)(b + o_items);
    B.eligible = (uint32_t*)(b + o_elig);
    B.perm = (uint32_t*)(b + o_perm);
    B.rest = (uint32_t*)(b + o_rest);
    B.code = (uint32_t*)(b + o_code);
    B.n_tree = (uint32_t*)(b + o_cnt);
    B.err = B.n_tree + 1;
    Seg* segs[2] = {(Seg*)(b + o_seg0), (Seg*)(b + o_seg1)};
    auto done = [&](int rc) { cudaStreamSynchronize(st); cudaFree(scratch); return rc; };
    uint32_t counts[2] = {0, 0};
    cudaError_t e = cudaMemsetAsync(B.n_tree, 0, 16, st);
    if (ms) cudaEventRecord(c->t0, st);
    k_lt_items<<<(n + 127) / 128, 128, 0, st>>>(B);
    k_lt_compact<<<1, THREADS, 0, st>>>(B, 1u);
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts, B.n_tree, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(c, e, "trt_scene_build_light_tree"));
    if (counts[1]) return done(fail(c, TRT_EINVAL, "trt_scene_build_light_tree: an emitter record points outside the scene's buffers"));
    uint32_t nt = counts[0];
    if (nt > MAX_ITEMS)
        return done(fail(c, TRT_EINVAL, "trt_scene_build_light_tree: more than 16,384 emitters for the tree (the device build's limit)"));
    if (nt < MIN_STATIC) {
        nt = 0;  // ltree.rs:421: the CDF alone below MIN_STATIC emitters
        k_lt_compact<<<1, THREADS, 0, st>>>(B, 0u);
    } else {
        if (2ull * nt - 1 > B.tree_cap)
            return done(fail(c, TRT_EINVAL, "trt_scene_build_light_tree: the tables' tree section holds fewer nodes than the tree needs"));
        Seg root{0u, nt, 0u, 1u, 0u, 0u};
        e = cudaMemcpyAsync(segs[0], &root, sizeof(root), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_lt_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(8u * MAX_ITEMS));
        int cur = 0;
        for (uint32_t level = 0; level < max_levels && e == cudaSuccess; ++level) {
            uint32_t max_len = (nt + (1u << level) - 1u) >> level;  // the right halves get the odd item
            uint32_t n2 = 1u;
            while (n2 < max_len) n2 <<= 1;
            k_lt_level<<<1u << level, THREADS, max_len >= 2u ? 8u * n2 : 0u, st>>>(B, segs[cur], 1u << level, segs[cur ^ 1]);
            e = cudaGetLastError();
            cur ^= 1;
            if (max_len <= 1u) break;
        }
    }
    if (e == cudaSuccess) {
        k_lt_order<<<(n + 127) / 128, 128, 0, st>>>(B, nt);
        e = cudaGetLastError();
    }
    if (ms && e == cudaSuccess) e = cudaEventRecord(c->t1, st);
    uint32_t err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, B.err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(c, e, "trt_scene_build_light_tree"));
    if (ms) cudaEventElapsedTime(ms, c->t0, c->t1);
    if (err) return done(fail(c, TRT_EINVAL, "trt_scene_build_light_tree: a record outside the tables, or a tree too deep"));
    // The host copy of the tables follows the device's (the re-weigh reads the tree's levels from it).
    if (s->host[3].size() >= s->bytes[3]) {
        auto back = [&](uint64_t first, uint64_t count) {
            if (e == cudaSuccess && count)
                e = cudaMemcpyAsync(s->host[3].data() + first * 16, (const char*)s->buf[3] + first * 16, count * 16,
                                    cudaMemcpyDeviceToHost, st);
        };
        back(B.tree, nt ? 2ull * nt - 1 : 0);
        back(B.entries, n);
        back(B.list, 4ull * n);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return done(cuda_fail(c, e, "trt_scene_build_light_tree"));
        s->wide.invalidate();
    }
    // Params' tree words (lib.rs:735-740): the tree's entries and the candidates resampled at camera hits.
    const float ris = nt ? 6.0f : 0.0f;
    P[P_LTREE + 1] = nt;
    std::memcpy(&P[P_LTREE + 3], &ris, 4);
    *tree_nodes = nt ? 2u * nt - 1u : 0u;
    return done(TRT_OK);
}
