// The light list's weights made again on the device from what the pass shades with: each emitter's weight (its
// triangle's area as its record has it now x its material's emissive luminance x its object's power, x the light LOD
// when one is given), the cumulative table and its guide, the light tree's node powers, the table's header (the
// total, the share outside the tree). renderer/shaders/emitter_weights.wgsl as gpu.rs:3219-3285 weigh_emitters
// runs it, after object-power, material or emitter-record edits; what lib.rs:451-485 emitter_cdf and ltree.rs:260-272
// refit make on the CPU at load. Included by pathtrace.cu (it writes a resident scene's tables).
//
// The rounding is the reference kernel's: the cumulative weights summed sequentially within blocks of 256 entries,
// the blocks' sums sequentially, then each entry's prefix as (its block's offset + its in-block sum) / total.
#pragma once

namespace trt_em {

constexpr uint32_t INSTANCE_VEC4 = 10u, MATERIAL_VEC4 = 18u, NO_INST = 0xffffffffu, EMITTER_MOVES = 0x80000000u,
                   EMITTER_GONE = 2u, EMITTER_NOMINAL = 4u, ROW_MATERIAL = 0xffffffu, LEAF = 0x80000000u,
                   GUIDE = 65536u, BLOCK = 256u, LEVELS = 32u;

// emitter_weights.wgsl Params: where each table starts (vec4s), the light LOD and its cull.
struct Weigh {
    uint32_t n, nodes, stride, flags;
    uint32_t list, entries, tree, instances, materials, objects, rows;
    float4 lod, cull, dir;
    const uint4* tables;  // the scene's tables (read-write through `rw`)
    uint4* rw;
    const uint32_t* words;
    uint64_t n_tables, n_words;
    float4* blocks;       // ceil(n / 256) + 1
    uint32_t* err;        // set when a record points outside the buffers
};

__device__ __forceinline__ uint4 tget(const Weigh& W, uint64_t i) {
    if (i >= W.n_tables) {
        atomicOr(W.err, 1u);
        return make_uint4(0u, 0u, 0u, 0u);
    }
    return W.tables[i];
}
__device__ __forceinline__ float4 tgetf(const Weigh& W, uint64_t i) {
    uint4 v = tget(W, i);
    return make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w));
}
__device__ __forceinline__ void tput(const Weigh& W, uint64_t i, float4 v) {
    if (i >= W.n_tables) {
        atomicOr(W.err, 1u);
        return;
    }
    W.rw[i] = make_uint4(__float_as_uint(v.x), __float_as_uint(v.y), __float_as_uint(v.z), __float_as_uint(v.w));
}

// emitter_weights.wgsl light_lod (lib.rs emitter_lod): the LOD's falloff and its cull.
__device__ __forceinline__ float light_lod(const Weigh& W, float cx, float cy, float cz) {
    float dx = cx - W.lod.x, dy = cy - W.lod.y, dz = cz - W.lod.z;
    float d = sqrtf(dx * dx + dy * dy + dz * dz);
    if (W.cull.x > 0.0f && d > W.cull.x &&
        !(d <= W.cull.y && dx * W.dir.x + dy * W.dir.y + dz * W.dir.z >= W.cull.z * d))
        return 0.0f;
    float k = W.lod.w / fmaxf(d, W.lod.w);
    return k * k;
}

// weigh: an entry's weight and area from its emitter's record, instance, material and object.
__global__ void k_em_weigh(Weigh W) {
    uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= W.n) return;
    uint4 e = tget(W, (uint64_t)W.entries + id);
    uint64_t r = (uint64_t)W.list + (uint64_t)e.x * 4u;
    uint4 r0 = tget(W, r), r1 = tget(W, r + 1), r2 = tget(W, r + 2), r3 = tget(W, r + 3);
    float e1x = __uint_as_float(r1.x), e1y = __uint_as_float(r1.y), e1z = __uint_as_float(r1.z);
    float e2x = __uint_as_float(r2.x), e2y = __uint_as_float(r2.y), e2z = __uint_as_float(r2.z);
    float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
    float area = 0.5f * sqrtf(cx * cx + cy * cy + cz * cz);
    if ((r3.y & EMITTER_NOMINAL) != 0u) area = __uint_as_float(r3.z);
    float w = 0.0f;
    if ((r3.y & EMITTER_GONE) != 0u || r1.w == NO_INST) {
        area = 0.0f;
    } else {
        // (The instance's record: its seventh vec4 has its object and its rows.)
        uint4 info = tget(W, (uint64_t)W.instances + (uint64_t)r1.w * INSTANCE_VEC4 + 6u);
        uint64_t wi = (uint64_t)W.rows + ((uint64_t)info.w + r3.x) * 4u;
        uint32_t m = 0u;
        if (wi < W.n_words) m = W.words[wi] & ROW_MATERIAL;
        else atomicOr(W.err, 1u);
        float4 em = tgetf(W, (uint64_t)W.materials + (uint64_t)m * MATERIAL_VEC4 + 1u);
        float power = tgetf(W, (uint64_t)W.objects + (uint64_t)info.y * W.stride).w;
        w = area * (em.x * 0.2126f + em.y * 0.7152f + em.z * 0.0722f) * power;
        if ((W.flags & 1u) != 0u && (r2.w & EMITTER_MOVES) == 0u)
            w *= light_lod(W, __uint_as_float(r0.x) + (e1x + e2x) / 3.0f, __uint_as_float(r0.y) + (e1y + e2y) / 3.0f,
                           __uint_as_float(r0.z) + (e1z + e2z) / 3.0f);
    }
    tput(W, (uint64_t)W.entries + id, make_float4(__uint_as_float(e.x), 0.0f, fmaxf(w, 0.0f), area));
}

// scan_a: each block of 256 entries' running sum, in order; the block's sum. A warp a block: its lanes stage the
// weights in shared memory, one lane adds them up in entry order (the reference's rounding), the lanes write back.
constexpr uint32_t SCAN_WARPS = 4u;
__global__ void __launch_bounds__(32u * SCAN_WARPS) k_em_scan_a(Weigh W) {
    __shared__ float run[SCAN_WARPS][BLOCK];
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
    const uint32_t b = blockIdx.x * SCAN_WARPS + wi;
    const uint32_t nb = (W.n + BLOCK - 1u) / BLOCK;
    if (b >= nb) return;  // (whole warps)
    const uint32_t lo = b * BLOCK, cnt = min(BLOCK, W.n - lo);
    float* r = run[wi];
    for (uint32_t k = lane; k < cnt; k += 32u) r[k] = tgetf(W, (uint64_t)W.entries + lo + k).z;
    __syncwarp();
    if (lane == 0) {
        float sum = 0.0f;
#pragma unroll 8
        for (uint32_t k = 0; k < cnt; ++k) {
            sum += r[k];
            r[k] = sum;
        }
        W.blocks[b] = make_float4(sum, 0.0f, 0.0f, 0.0f);
    }
    __syncwarp();
    for (uint32_t k = lane; k < cnt; k += 32u) {
        float4 e = tgetf(W, (uint64_t)W.entries + lo + k);
        e.y = r[k];
        tput(W, (uint64_t)W.entries + lo + k, e);
    }
}

// scan_b: the blocks' offsets, in order; after the last, the total. One thread.
__global__ void k_em_scan_b(Weigh W) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t nb = (W.n + BLOCK - 1u) / BLOCK;
    float sum = 0.0f;
    for (uint32_t b = 0; b < nb; ++b) {
        W.blocks[b].y = sum;
        sum += W.blocks[b].x;
    }
    W.blocks[nb] = make_float4(sum, 0.0f, 0.0f, 0.0f);
}

// scan_c: the cumulative weights over the total (exactly 1 from the last entry that weighs something on).
__global__ void k_em_scan_c(Weigh W) {
    uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= W.n) return;
    uint32_t nb = (W.n + BLOCK - 1u) / BLOCK;
    float total = W.blocks[nb].x;
    float4 e = tgetf(W, (uint64_t)W.entries + id);
    float c = W.blocks[id / BLOCK].y + e.y;
    e.y = total > 0.0f ? (c >= total ? 1.0f : c / total) : 0.0f;
    tput(W, (uint64_t)W.entries + id, e);
}

// guide: index k is the first entry whose cumulative weight is not below k / GUIDE; four a vec4, a vec4 a thread.
__global__ void k_em_guide(Weigh W) {
    uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id > GUIDE / 4u) return;
    uint32_t out[4] = {0u, 0u, 0u, 0u};
    for (uint32_t c = 0; c < 4u; ++c) {
        uint32_t k = id * 4u + c;
        if (k > GUIDE) break;
        float u = (float)k / (float)GUIDE;
        uint32_t lo = 0u, hi = W.n;
        for (uint32_t s = 0; s < 32u && lo < hi; ++s) {
            uint32_t mid = (lo + hi) / 2u;
            if (tgetf(W, (uint64_t)W.entries + mid).y < u) lo = mid + 1u;
            else hi = mid;
        }
        out[c] = lo;
    }
    uint64_t at = (uint64_t)W.entries + W.n + id;
    if (at >= W.n_tables) {
        atomicOr(W.err, 1u);
        return;
    }
    W.rw[at] = make_uint4(out[0], out[1], out[2], out[3]);
}

// tree: the nodes' powers, the deepest level first (ltree.rs levels), a leaf's from its entries, a node's from its
// two children. One block walks the levels; a level's nodes are independent. `levels`: per level (first, count) into
// `list`, `n_levels` of them.
__global__ void k_em_tree(Weigh W, const uint32_t* __restrict__ levels, uint32_t n_levels,
                          const uint32_t* __restrict__ list) {
    if (W.nodes == 0u) return;
    uint32_t top = min(n_levels, LEVELS);
    for (uint32_t l = 0; l < top; ++l) {
        uint32_t first = levels[2 * l], count = levels[2 * l + 1];
        for (uint32_t j = threadIdx.x; j < count; j += blockDim.x) {
            uint32_t i = list[first + j];
            float4 nd = tgetf(W, (uint64_t)W.tree + i);
            uint32_t w = __float_as_uint(nd.w);
            float power = 0.0f;
            if ((w & LEAF) != 0u) {
                uint32_t lo = w & 0x1fffffffu, hi = lo + ((w >> 29) & 3u) + 1u;
                for (uint32_t k = lo; k < hi; ++k) {
                    if (k >= W.n) {
                        atomicOr(W.err, 1u);
                        break;
                    }
                    power += tgetf(W, (uint64_t)W.entries + k).z;
                }
            } else {
                power = tgetf(W, (uint64_t)W.tree + w).z + tgetf(W, (uint64_t)W.tree + w + 1u).z;
            }
            nd.z = power;
            tput(W, (uint64_t)W.tree + i, nd);
        }
        __syncthreads();
    }
}

// finish: the header: the total, and the share of it that is not the tree's.
__global__ void k_em_finish(Weigh W) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t nb = (W.n + BLOCK - 1u) / BLOCK;
    float total = W.blocks[nb].x;
    float tail = 0.0f;
    if (W.nodes > 0u && total > 0.0f) tail = fmaxf((total - tgetf(W, W.tree).z) / total, 0.0f);
    tput(W, (uint64_t)W.entries + W.n + GUIDE / 4u + 1u, make_float4(total, tail, 0.0f, 0.0f));
}

}  // namespace trt_em

// ltree.rs:233-256 LightTree::levels from the tree's node words (host copy of the tables): the reachable nodes by
// depth, the deepest first (index order within a depth); per level (first, count).
static void em_levels(const uint4* nodes, uint32_t n, std::vector<uint32_t>& list, std::vector<uint32_t>& levels) {
    std::vector<uint32_t> depth(n, 0xffffffffu);
    if (n > 0) depth[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t w = nodes[i].w;
        if (depth[i] != 0xffffffffu && (w & trt_em::LEAF) == 0u && (uint64_t)w + 1 < n)
            depth[w] = depth[w + 1] = depth[i] + 1;
    }
    list.clear();
    for (uint32_t i = 0; i < n; ++i)
        if (depth[i] != 0xffffffffu) list.push_back(i);
    std::stable_sort(list.begin(), list.end(), [&](uint32_t a, uint32_t b) { return depth[a] > depth[b]; });
    levels.clear();
    for (size_t k = 0; k < list.size(); ++k) {
        if (k == 0 || depth[list[k]] != depth[list[k - 1]]) {
            levels.push_back((uint32_t)k);
            levels.push_back(0u);
        }
        levels.back() += 1;
    }
}

int trt_scene_weigh_emitters(trt_scene* s, const uint32_t* P, uint32_t tree_nodes, const float* lod, const float* cull,
                             float* ms) {
    using namespace trt_em;
    if (!s || !P) return TRT_EINVAL;
    trt_ctx* c = s->ctx;
    uint32_t n = P[P_COUNTS + 1];
    if (n == 0) return TRT_OK;
    uint64_t tv = s->bytes[3] / 16;
    uint64_t entries = P[P_TABLE_FIRST + 4], tree = P[P_TABLE_FIRST + 0];
    if (entries + n + GUIDE / 4u + 2u > tv || tree + tree_nodes > tv)
        return fail(c, TRT_EINVAL, "trt_scene_weigh_emitters: the emitter table or the tree is not inside the tables");
    if (tree_nodes > 0 && s->host[3].size() < (tree + tree_nodes) * 16)
        return fail(c, TRT_EINVAL, "trt_scene_weigh_emitters: no host copy of the tree");
    std::vector<uint32_t> list, levels;
    em_levels(reinterpret_cast<const uint4*>(s->host[3].data()) + tree, tree_nodes, list, levels);
    uint32_t nb = (n + BLOCK - 1u) / BLOCK;
    uint64_t need = (uint64_t)(nb + 1) * 16 + 16 + (levels.size() + list.size() + 2) * 4;
    cudaSetDevice(c->device);
    if (need > s->em_bytes) {
        if (s->em) cudaFree(s->em);
        s->em = nullptr;
        s->em_bytes = 0;
        TRT_CUDA(c, cudaMalloc(&s->em, need));
        s->em_bytes = need;
    }
    char* base = (char*)s->em;
    Weigh W{};
    W.n = n;
    W.nodes = tree_nodes;
    W.stride = 3;  // vec4s an object (lib.rs object_stride: the power row and two more)
    W.flags = (lod && lod[3] > 0.0f) ? 1u : 0u;
    W.list = P[P_TABLE_FIRST + 11];
    W.entries = (uint32_t)entries;
    W.tree = (uint32_t)tree;
    W.instances = P[P_TABLE_FIRST + 7];
    W.materials = P[P_TABLE_FIRST + 1];
    W.objects = P[P_TABLE_FIRST + 6];
    W.rows = P[P_WORD_FIRST + 3];
    W.lod = lod ? make_float4(lod[0], lod[1], lod[2], lod[3]) : make_float4(0, 0, 0, 0);
    W.cull = cull ? make_float4(cull[0], cull[1], cull[2], 0.0f) : make_float4(0, 0, 0, 0);
    W.dir = cull ? make_float4(cull[3], cull[4], cull[5], 0.0f) : make_float4(0, 0, 0, 0);
    W.tables = (const uint4*)s->buf[3];
    W.rw = (uint4*)s->buf[3];
    W.words = (const uint32_t*)s->buf[4];
    W.n_tables = tv;
    W.n_words = s->bytes[4] / 4;
    W.blocks = (float4*)base;
    W.err = (uint32_t*)(base + (uint64_t)(nb + 1) * 16);
    uint32_t* d_levels = W.err + 4;
    uint32_t* d_list = d_levels + levels.size();
    cudaStream_t st = c->stream;
    std::vector<uint32_t> up(levels);
    up.insert(up.end(), list.begin(), list.end());
    TRT_CUDA(c, cudaMemsetAsync(W.err, 0, 4, st));
    if (!up.empty()) TRT_CUDA(c, cudaMemcpyAsync(d_levels, up.data(), up.size() * 4, cudaMemcpyHostToDevice, st));
    if (ms) TRT_CUDA(c, cudaEventRecord(c->t0, st));
    k_em_weigh<<<(n + 63) / 64, 64, 0, st>>>(W);
    k_em_scan_a<<<(nb + SCAN_WARPS - 1u) / SCAN_WARPS, 32u * SCAN_WARPS, 0, st>>>(W);
    k_em_scan_b<<<1, 32, 0, st>>>(W);
    k_em_scan_c<<<(n + 63) / 64, 64, 0, st>>>(W);
    k_em_guide<<<(GUIDE / 4u + 1u + 127u) / 128u, 128, 0, st>>>(W);
    k_em_tree<<<1, 256, 0, st>>>(W, d_levels, (uint32_t)(levels.size() / 2), d_list);
    k_em_finish<<<1, 32, 0, st>>>(W);
    if (ms) TRT_CUDA(c, cudaEventRecord(c->t1, st));
    TRT_CUDA(c, cudaGetLastError());
    uint32_t err = 0;
    TRT_CUDA(c, cudaMemcpyAsync(&err, W.err, 4, cudaMemcpyDeviceToHost, st));
    TRT_CUDA(c, cudaStreamSynchronize(st));
    if (ms) cudaEventElapsedTime(ms, c->t0, c->t1);
    // The host copy of the tables follows the device's (the wide BVH reads its instance records from it).
    if (s->host[3].size() >= s->bytes[3]) {
        TRT_CUDA(c, cudaMemcpyAsync(s->host[3].data() + entries * 16, (const char*)s->buf[3] + entries * 16,
                                    ((uint64_t)n + GUIDE / 4u + 2u) * 16, cudaMemcpyDeviceToHost, st));
        if (tree_nodes)
            TRT_CUDA(c, cudaMemcpyAsync(s->host[3].data() + tree * 16, (const char*)s->buf[3] + tree * 16,
                                        (uint64_t)tree_nodes * 16, cudaMemcpyDeviceToHost, st));
        TRT_CUDA(c, cudaStreamSynchronize(st));
    }
    if (err) return fail(c, TRT_EINVAL, "trt_scene_weigh_emitters: an emitter record points outside the scene's buffers");
    return TRT_OK;
}
