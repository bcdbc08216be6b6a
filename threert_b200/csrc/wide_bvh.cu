// Builds the wide BVH (wide_bvh.cuh) from the reference's binary trees: each mesh tree a unit names, and the units'
// top tree. A binary node's children are opened, the one with the largest box first, until a wide node has eight
// (bvh.rs trees' leaves stay whole, with their triangles in the tree's order); child boxes are quantised against the
// node's own box.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "wide_bvh.cuh"

namespace trt {
namespace {

struct BinNode { float bmin[3]; uint32_t left_or_first; float bmax[3]; uint32_t count; };
static_assert(sizeof(BinNode) == 32, "the reference's GpuNode");

struct WNode { uint32_t w[20]; };

float area_of(const BinNode& n) {
    float e[3];
    for (int k = 0; k < 3; ++k) e[k] = std::max(n.bmax[k] - n.bmin[k], 0.0f);
    return 2.0f * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0]);
}

struct Builder {
    const BinNode* nodes;
    uint64_t n_nodes;
    std::vector<WNode> out;
    std::string error;

    // Quantises the child boxes of one wide node (wide_encode) and writes its header.
    void encode(WNode& W, const std::vector<const BinNode*>& ch, const std::vector<bool>& interior, uint32_t child_base,
                uint32_t leaf_base, const std::vector<uint32_t>& counts, float tree_pad) {
        float bmin[8][3], bmax[8][3];
        uint32_t present = 0, imask = 0, cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (size_t i = 0; i < ch.size() && i < 8; ++i) {
            if (!ch[i]) continue;
            present |= 1u << i;
            for (int k = 0; k < 3; ++k) { bmin[i][k] = ch[i]->bmin[k]; bmax[i][k] = ch[i]->bmax[k]; }
            if (interior[i]) imask |= 1u << i;
            else cnt[i] = counts[i];
        }
        wide_encode(W.w, bmin, bmax, present, imask, child_base, leaf_base, cnt, tree_pad);
    }

    // The children in slots by octant: slot s (bit k set: the upper half along axis k) takes the child whose centre
    // lies most that way from the node's centre, so that a walk visiting slots in the order k ^ (the ray's sign bits)
    // meets them nearly front to back without sorting. Greedy assignment by score; unused slots are empty (index
    // UINT32_MAX).
    std::vector<uint32_t> octant_slots(const std::vector<uint32_t>& ch) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t c : ch)
            for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], nodes[c].bmin[k]); hi[k] = std::max(hi[k], nodes[c].bmax[k]); }
        struct Cand { float score; int child, slot; };
        std::vector<Cand> cands;
        for (size_t j = 0; j < ch.size(); ++j) {
            float v[3];
            for (int k = 0; k < 3; ++k) {
                float e = std::max(hi[k] - lo[k], 1e-30f);
                v[k] = ((nodes[ch[j]].bmin[k] + nodes[ch[j]].bmax[k]) - (lo[k] + hi[k])) / e;
            }
            for (int sl = 0; sl < 8; ++sl) {
                float sc = 0.0f;
                for (int k = 0; k < 3; ++k) sc += (sl >> k & 1) ? v[k] : -v[k];
                cands.push_back({sc, (int)j, sl});
            }
        }
        std::stable_sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) { return a.score > b.score; });
        std::vector<uint32_t> slots(8, UINT32_MAX);
        std::vector<bool> placed(ch.size(), false);
        for (const Cand& c : cands)
            if (!placed[c.child] && slots[c.slot] == UINT32_MAX) { slots[c.slot] = ch[c.child]; placed[c.child] = true; }
        return slots;
    }

    // Collapses the binary tree rooted at `root` (child indices from `root`); `leaf(node, items)` appends a binary
    // leaf's items and returns their count. Returns the wide root's index, or UINT32_MAX on a malformed tree.
    // What a refit reads (WideBvh::slot_host, pad_host), by wide node.
    std::vector<uint32_t> slots;
    std::vector<float> pads;

    template <class Leaf>
    uint32_t collapse(uint32_t root, Leaf&& leaf, uint32_t max_leaf_items, bool top_tree) {
        if (root >= n_nodes) { error = "a tree's root is past the nodes"; return UINT32_MAX; }
        // A slab test rounds with the distance to the box: a box far from the ray's origin but small (a few
        // millimetres of a 10 m mesh seen from 1 km) needs more margin than its own size gives, so every box of a
        // tree is widened by at least 2^-14 of the tree's extent.
        float tree_pad;
        {
            const BinNode& r0 = nodes[root];
            float ext = 0.0f;
            for (int k = 0; k < 3; ++k) ext = std::max(ext, r0.bmax[k] - r0.bmin[k]);
            tree_pad = std::isfinite(ext) ? ext * (1.0f / 16384.0f) : 0.0f;
        }
        const float pad_of_tree = tree_pad;  // (a nested collapse of a unit's mesh tree has its own)
        uint32_t wroot = (uint32_t)out.size();
        out.emplace_back();
        std::vector<std::pair<uint32_t, uint32_t>> work{{root, wroot}};
        uint64_t visited = 0;
        while (!work.empty()) {
            auto [b, w] = work.back();
            work.pop_back();
            if (++visited > 4 * n_nodes + 8) { error = "a tree is not a tree (a node is reached twice)"; return UINT32_MAX; }
            std::vector<uint32_t> ch;
            const BinNode& n = nodes[b];
            if (n.count > 0) {
                ch.push_back(b);
            } else {
                uint32_t l = root + n.left_or_first;
                if (l <= b || (uint64_t)l + 1 >= n_nodes) { error = "a node's children are not after it"; return UINT32_MAX; }
                ch = {l, l + 1};
                for (;;) {
                    if (ch.size() >= 8) break;
                    int best = -1;
                    float best_area = -1.0f;
                    for (size_t i = 0; i < ch.size(); ++i) {
                        const BinNode& c = nodes[ch[i]];
                        if (c.count == 0 && area_of(c) > best_area) { best_area = area_of(c); best = (int)i; }
                    }
                    if (best < 0) break;
                    uint32_t cl = root + nodes[ch[best]].left_or_first;
                    if (cl <= ch[best] || (uint64_t)cl + 1 >= n_nodes) { error = "a node's children are not after it"; return UINT32_MAX; }
                    ch[best] = cl;
                    ch.insert(ch.begin() + best + 1, cl + 1);
                }
            }
            ch = octant_slots(ch);
            std::vector<const BinNode*> cp;
            std::vector<bool> interior;
            std::vector<uint32_t> counts;
            uint32_t n_interior = 0;
            for (uint32_t c : ch) {
                cp.push_back(c == UINT32_MAX ? nullptr : &nodes[c]);
                interior.push_back(c != UINT32_MAX && nodes[c].count == 0);
                if (c != UINT32_MAX && nodes[c].count == 0) n_interior++;
            }
            uint32_t child_base = (uint32_t)out.size();
            out.resize(out.size() + n_interior);
            uint32_t leaf_base = UINT32_MAX, k = 0;
            for (size_t i = 0; i < ch.size(); ++i) {
                if (ch[i] == UINT32_MAX) {
                    counts.push_back(0);
                } else if (interior[i]) {
                    work.push_back({ch[i], child_base + k++});
                    counts.push_back(0);
                } else {
                    if (nodes[ch[i]].count > max_leaf_items) { error = "a leaf holds more items than a tree's leaves may"; return UINT32_MAX; }
                    uint32_t first = leaf(nodes[ch[i]]);
                    if (first == UINT32_MAX) return UINT32_MAX;
                    if (leaf_base == UINT32_MAX) leaf_base = first;
                    counts.push_back(nodes[ch[i]].count);

                }
            }
            if (leaf_base == UINT32_MAX) leaf_base = 0;
            encode(out[w], cp, interior, child_base, leaf_base, counts, pad_of_tree);
            if (slots.size() < 8 * out.size()) {
                slots.resize(8 * out.size(), WIDE_SLOT_EMPTY);
                pads.resize(out.size(), 0.0f);
            }
            for (int i = 0; i < 8; ++i) slots[8ull * w + i] = top_tree ? WIDE_SLOT_TOP : ch[i];
            pads[w] = pad_of_tree;

        }
        return wroot;
    }
};

constexpr uint32_t P_MOTION_Z = 70, P_MOTION_W = 71, P_T_INSTANCES = 124 + 7, P_W_INDICES = 136 + 4;

// ---- the refit after a deformation --------------------------------------------------------------------------------

// A binary node (the reference's GpuNode, two vec4s): its box, left_or_first and count.
__device__ __forceinline__ void bin_node(const uint4* __restrict__ bin, uint32_t i, float mn[3], float mx[3],
                                         uint32_t* lof, uint32_t* count) {
    const uint4 a = bin[2ull * i], b = bin[2ull * i + 1];
    mn[0] = __uint_as_float(a.x); mn[1] = __uint_as_float(a.y); mn[2] = __uint_as_float(a.z);
    mx[0] = __uint_as_float(b.x); mx[1] = __uint_as_float(b.y); mx[2] = __uint_as_float(b.z);
    *lof = a.w;
    *count = b.w;
}

__device__ __forceinline__ void put_node(uint4* __restrict__ wn, uint32_t w, const uint32_t W[20]) {
#pragma unroll
    for (int j = 0; j < 5; ++j) wn[5ull * w + j] = make_uint4(W[4 * j], W[4 * j + 1], W[4 * j + 2], W[4 * j + 3]);
}

// Every built node of a mesh tree quantised again over its slots' binary boxes (the topology, its child and leaf
// indices and counts are the build's). A thread a node; the top tree's nodes are skipped.
__global__ void k_wide_refit(const uint4* __restrict__ bin, uint64_t n_bin, const uint32_t* __restrict__ slots,
                             const float* __restrict__ pads, uint4* wn, uint32_t n_nodes, uint32_t* err, uint32_t err_bit) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < n_nodes; w += gridDim.x * blockDim.x) {
        const uint32_t* sl = slots + 8ull * w;
        if (sl[0] == WIDE_SLOT_TOP) continue;
        uint32_t W[20];
#pragma unroll
        for (int j = 0; j < 5; ++j) {
            const uint4 q = wn[5ull * w + j];
            W[4 * j] = q.x; W[4 * j + 1] = q.y; W[4 * j + 2] = q.z; W[4 * j + 3] = q.w;
        }
        float bmin[8][3], bmax[8][3];
        uint32_t present = 0, counts[8];
        bool bad = false;
        for (int i = 0; i < 8; ++i) {
            counts[i] = (W[6 + (i >> 2)] >> (8 * (i & 3))) & 0xffu;
            const uint32_t b = sl[i];
            if (b == WIDE_SLOT_EMPTY) continue;
            if (b >= n_bin) { bad = true; continue; }
            uint32_t lof, cnt;
            bin_node(bin, b, bmin[i], bmax[i], &lof, &cnt);
            present |= 1u << i;
        }
        if (bad) { atomicOr(err, err_bit); continue; }
        uint32_t out[20];
        wide_encode(out, bmin, bmax, present, W[3] >> 24, W[4], W[5], counts, pads[w]);
        put_node(wn, w, out);
    }
}

// The wide triangle copies gathered again from the deformed leaves (each copy keeps its reference index in the third
// vec4's w).
__global__ void k_wide_tris(const float4* __restrict__ leaves, uint64_t n_leaf_tris, float4* tris, uint32_t n_tris,
                            uint32_t* err, uint32_t err_bit) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_tris; i += gridDim.x * blockDim.x) {
        const uint32_t ti = __float_as_uint(tris[3ull * i + 2].w);
        if (ti >= n_leaf_tris) { atomicOr(err, err_bit); continue; }
        float4 c = leaves[3ull * ti + 2];
        c.w = __uint_as_float(ti);
        tris[3ull * i] = leaves[3ull * ti];
        tris[3ull * i + 1] = leaves[3ull * ti + 1];
        tris[3ull * i + 2] = c;
    }
}

struct TopCollapse {
    const uint4* bin;
    uint64_t n_bin;
    uint32_t top;           // the binary top tree's root; its children are at top + left_or_first
    const uint4* tables;
    uint64_t n_table_vec4;
    uint32_t t_instances;   // the units' records, 10 vec4s each
    uint4* wn;
    uint32_t base, cap;     // the top region: nodes [base, base + cap)
    uint32_t* items;        // the top tree's leaf items (unit record | shadow bit)
    uint32_t n_items;
    uint2* front;           // two frontiers of cap entries
    uint32_t* err;
    uint32_t err_bit;
};

constexpr uint32_t TOP_THREADS = 256, TOP_WARPS_C = TOP_THREADS / 32;

// Exclusive prefix of v over the block, and the block's total; `part` is TOP_WARPS_C words of shared memory.
__device__ __forceinline__ uint32_t block_prefix(uint32_t v, uint32_t* total, uint32_t* part) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) part[warp] = x;
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (uint32_t k = 0; k < TOP_WARPS_C; ++k) {
        before += k < warp ? part[k] : 0u;
        all += part[k];
    }
    *total = all;
    return before + x - v;
}

// One binary node of the top tree opened into a wide node's children as the host build opens it (the child of
// largest surface area first, up to eight; a leaf stays whole), then placed in slots by octant (the greedy assignment
// of (child, slot) pairs by score, ties to the lower child and slot). False on a malformed tree.
__device__ bool top_slots(const TopCollapse& T, uint32_t b, uint32_t slot[8]) {
    uint32_t ch[8], n;
    float mn[3], mx[3];
    uint32_t lof, cnt;
    bin_node(T.bin, b, mn, mx, &lof, &cnt);
    if (cnt > 0) {
        ch[0] = b;
        n = 1;
    } else {
        const uint32_t l = T.top + lof;
        if (l <= b || (uint64_t)l + 1 >= T.n_bin) return false;
        ch[0] = l;
        ch[1] = l + 1;
        n = 2;
        while (n < 8) {
            int best = -1;
            float best_area = -1.0f;
            for (uint32_t i = 0; i < n; ++i) {
                bin_node(T.bin, ch[i], mn, mx, &lof, &cnt);
                float e[3];
                for (int k = 0; k < 3; ++k) e[k] = wmax(mx[k] - mn[k], 0.0f);
                const float area = 2.0f * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0]);
                if (cnt == 0 && area > best_area) { best_area = area; best = (int)i; }
            }
            if (best < 0) break;
            bin_node(T.bin, ch[best], mn, mx, &lof, &cnt);
            const uint32_t cl = T.top + lof;
            if (cl <= ch[best] || (uint64_t)cl + 1 >= T.n_bin) return false;
            for (uint32_t i = n; i > (uint32_t)best + 1; --i) ch[i] = ch[i - 1];
            ch[best] = cl;
            ch[best + 1] = cl + 1;
            ++n;
        }
    }
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float v[8][3];
    for (uint32_t j = 0; j < n; ++j) {
        bin_node(T.bin, ch[j], mn, mx, &lof, &cnt);
        for (int k = 0; k < 3; ++k) { lo[k] = wmin(lo[k], mn[k]); hi[k] = wmax(hi[k], mx[k]); }
    }
    for (uint32_t j = 0; j < n; ++j) {
        bin_node(T.bin, ch[j], mn, mx, &lof, &cnt);
        for (int k = 0; k < 3; ++k) {
            const float e = wmax(hi[k] - lo[k], 1e-30f);
            v[j][k] = ((mn[k] + mx[k]) - (lo[k] + hi[k])) / e;
        }
    }
    for (int i = 0; i < 8; ++i) slot[i] = WIDE_SLOT_EMPTY;
    uint32_t placed = 0, taken = 0;
    for (uint32_t round = 0; round < n; ++round) {
        int bj = -1, bs = -1;
        float bsc = 0.0f;
        for (uint32_t j = 0; j < n; ++j) {
            if (placed >> j & 1u) continue;
            for (int sl = 0; sl < 8; ++sl) {
                if (taken >> sl & 1u) continue;
                float sc = 0.0f;
                for (int k = 0; k < 3; ++k) sc += (sl >> k & 1) ? v[j][k] : -v[j][k];
                if (bj < 0 || sc > bsc) { bj = (int)j; bs = sl; bsc = sc; }
            }
        }
        slot[bs] = ch[bj];
        placed |= 1u << bj;
        taken |= 1u << bs;
    }
    return true;
}

// The rebuilt top tree collapsed again into the top region, one CTA, a level of wide nodes at a time: each thread
// opens a frontier node, the block's prefix sums give its children's nodes and its leaf items their places (a node's
// interior children consecutive, its leaf items consecutive in slot order), and the children form the next frontier.
__global__ void __launch_bounds__(TOP_THREADS) k_wide_top(TopCollapse T) {
    __shared__ uint32_t part_n[TOP_WARPS_C], part_i[TOP_WARPS_C];
    __shared__ uint32_t next_free, items_next, next_count, failed;
    const uint32_t tid = threadIdx.x;
    if (T.top >= T.n_bin || T.cap == 0) {
        if (tid == 0) atomicOr(T.err, T.err_bit);
        return;
    }
    float mn[3], mx[3];
    uint32_t lof, cnt;
    bin_node(T.bin, T.top, mn, mx, &lof, &cnt);
    float ext = 0.0f;
    for (int k = 0; k < 3; ++k) ext = wmax(ext, mx[k] - mn[k]);
    const float tree_pad = isfinite(ext) ? ext * (1.0f / 16384.0f) : 0.0f;
    if (tid == 0) {
        T.front[0] = make_uint2(T.top, T.base);
        next_free = 1;
        items_next = 0;
        failed = 0;
    }
    __syncthreads();
    uint2* cur = T.front;
    uint2* nxt = T.front + T.cap;
    uint32_t count = 1;
    for (uint32_t level = 0; count > 0; ++level) {
        if (level >= 64) {
            if (tid == 0) atomicOr(T.err, T.err_bit);
            return;
        }
        if (tid == 0) next_count = 0;
        __syncthreads();
        for (uint32_t chunk = 0; chunk < count; chunk += TOP_THREADS) {
            const uint32_t i = chunk + tid;
            uint32_t slot[8], n_int = 0, n_items = 0;
            uint2 item = make_uint2(0, 0);
            bool ok = i < count;
            if (ok) {
                item = cur[i];
                ok = top_slots(T, item.x, slot);
                if (!ok) failed = 1;
            }
            if (ok)
                for (int s = 0; s < 8; ++s) {
                    if (slot[s] == WIDE_SLOT_EMPTY) continue;
                    bin_node(T.bin, slot[s], mn, mx, &lof, &cnt);
                    if (cnt == 0) n_int++;
                    else if (cnt > 16) { ok = false; failed = 1; }
                    else n_items += cnt;
                }
            if (!ok) n_int = n_items = 0;
            uint32_t tot_n, tot_i;
            const uint32_t pn = block_prefix(n_int, &tot_n, part_n);
            const uint32_t pi = block_prefix(n_items, &tot_i, part_i);
            const uint32_t nf = next_free, it0 = items_next, nc = next_count;
            const bool room = nf + tot_n <= T.cap && it0 + tot_i <= T.n_items;
            if (ok && room) {
                const uint32_t child_base = T.base + nf + pn, leaf_base = it0 + pi;
                float bmin[8][3], bmax[8][3];
                uint32_t present = 0, imask = 0, counts[8], k = 0, off = 0;
                for (int s = 0; s < 8; ++s) {
                    counts[s] = 0;
                    if (slot[s] == WIDE_SLOT_EMPTY) continue;
                    bin_node(T.bin, slot[s], bmin[s], bmax[s], &lof, &cnt);
                    present |= 1u << s;
                    if (cnt == 0) {
                        imask |= 1u << s;
                        nxt[nc + pn + k] = make_uint2(slot[s], child_base + k);
                        ++k;
                    } else {
                        counts[s] = cnt;
                        for (uint32_t j = 0; j < cnt; ++j) {
                            const uint32_t rec = lof + j;
                            const uint64_t r = (uint64_t)T.t_instances + 10ull * rec;
                            uint32_t bits = 0;
                            if (r + 10 > T.n_table_vec4) failed = 1;
                            else bits = T.tables[r + 4].w;
                            T.items[leaf_base + off++] = rec | ((bits & UNIT_SHADOW) ? WIDE_UNIT_BIT : 0u);
                        }
                    }
                }
                uint32_t W[20];
                wide_encode(W, bmin, bmax, present, imask, child_base, n_items ? leaf_base : 0u, counts, tree_pad);
                put_node(T.wn, item.y, W);
            }
            __syncthreads();
            if (tid == 0) {
                if (!room) failed = 1;
                next_free = nf + tot_n;
                items_next = it0 + tot_i;
                next_count = nc + tot_n;
            }
            __syncthreads();
            if (failed) {
                if (tid == 0) atomicOr(T.err, T.err_bit);
                return;
            }
        }
        count = next_count;
        uint2* t = cur;
        cur = nxt;
        nxt = t;
        __syncthreads();
    }
}

}  // namespace

int WideBvh::refit(const uint32_t* P, const void* bin_nodes, uint64_t n_bin, const void* leaves, uint64_t n_leaf_tris,
                   const void* tables, uint64_t n_table_vec4, uint32_t* err, uint32_t err_bit, cudaStream_t st) {
    if (!built) { error = "the wide BVH is not built"; return 1; }
    cudaError_t e = cudaSuccess;
    if (!slot_dev) {
        e = cudaMalloc(&slot_dev, std::max<size_t>(slot_host.size() * 4, 16));
        if (e == cudaSuccess) e = cudaMalloc(&pad_dev, std::max<size_t>(pad_host.size() * 4, 16));
        if (e == cudaSuccess && top_cap) e = cudaMalloc(&frontier, 2ull * top_cap * sizeof(uint2));
        if (e == cudaSuccess) e = cudaMemcpyAsync(slot_dev, slot_host.data(), slot_host.size() * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(pad_dev, pad_host.data(), pad_host.size() * 4, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { error = std::string("wide BVH refit: ") + cudaGetErrorString(e); return 1; }
    }
    const uint4* bin = static_cast<const uint4*>(bin_nodes);
    if (n_built) {
        unsigned g = (unsigned)std::min<uint64_t>((n_built + 255) / 256, 148ull * 8);
        k_wide_refit<<<g, 256, 0, st>>>(bin, n_bin, slot_dev, pad_dev, nodes, n_built, err, err_bit);
    }
    if (v.n_tris) {
        unsigned g = (unsigned)std::min<uint64_t>((v.n_tris + 255) / 256, 148ull * 8);
        k_wide_tris<<<g, 256, 0, st>>>(static_cast<const float4*>(leaves), n_leaf_tris, tris, v.n_tris, err, err_bit);
    }
    if (top_cap && v.n_units) {
        TopCollapse T{bin, n_bin, P[P_MOTION_Z], static_cast<const uint4*>(tables), n_table_vec4, P[P_T_INSTANCES],
                      nodes, n_built, top_cap, units, v.n_units, frontier, err, err_bit};
        k_wide_top<<<1, TOP_THREADS, 0, st>>>(T);
        v.top_root = n_built;
        v.n_nodes = n_built + top_cap;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) { error = std::string("wide BVH refit: ") + cudaGetErrorString(e); return 1; }
    return 0;
}

void WideBvh::release() {
    for (void* p : {(void*)nodes, (void*)tris, (void*)units, (void*)unit_root, (void*)slot_dev, (void*)pad_dev, (void*)frontier})
        if (p) cudaFree(p);
    nodes = nullptr;
    tris = nullptr;
    units = nullptr;
    unit_root = nullptr;
    slot_dev = nullptr;
    pad_dev = nullptr;
    frontier = nullptr;
    slot_host.clear();
    pad_host.clear();
    n_built = top_cap = 0;
    refit_gen = 0;
    built = false;
}

bool WideBvh::key_matches(const uint32_t* P) const {
    const uint32_t k[6] = {P[P_MOTION_Z], P[P_MOTION_W], P[P_T_INSTANCES], P[P_W_INDICES], 0, 0};
    return std::memcmp(k, key, sizeof(k)) == 0;
}

bool WideBvh::reads_edit(const uint8_t* old_tables, uint64_t tables_bytes, uint64_t offset, const uint8_t* src,
                         uint64_t bytes) const {
    if (!built || bytes == 0) return false;
    const uint64_t t_inst = key[2], end = offset + bytes;
    const uint64_t first = t_inst * 16;
    if (first >= tables_bytes) return false;
    const uint64_t n_units = std::min<uint64_t>(key[1], (tables_bytes - first) / 160);  // (records inside the copy)
    const uint64_t last = first + 160 * n_units;  // the unit records' bytes
    if (end <= first || offset >= last) return false;
    const uint64_t r0 = (std::max(offset, first) - first) / 160, r1 = std::min(n_units, (end - first + 159) / 160);
    // A record's words the build reads: vec4 3's w (the mesh root), vec4 6's x (the first triangle), and of vec4 4's
    // w (the bits) the shadow bit.
    const uint64_t words[3] = {3 * 16 + 12, 6 * 16, 4 * 16 + 12};
    const uint32_t masks[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, UNIT_SHADOW};
    for (uint64_t r = r0; r < r1; ++r)
        for (int j = 0; j < 3; ++j) {
            const uint64_t a = first + 160 * r + words[j];
            uint8_t now[4];
            std::memcpy(now, old_tables + a, 4);
            for (uint64_t b = std::max(a, offset); b < std::min(a + 4, end); ++b) now[b - a] = src[b - offset];
            uint32_t was, is;
            std::memcpy(&was, old_tables + a, 4);
            std::memcpy(&is, now, 4);
            if ((was ^ is) & masks[j]) return true;
        }
    return false;
}

int WideBvh::ensure(const uint32_t* P, const std::vector<uint8_t>* host, cudaStream_t st) {
    uint32_t k[6] = {P[P_MOTION_Z], P[P_MOTION_W], P[P_T_INSTANCES], P[P_W_INDICES], 0, 0};
    if (built && std::memcmp(k, key, sizeof(k)) == 0) return 0;
    auto t0 = std::chrono::steady_clock::now();
    release();
    const BinNode* bn = reinterpret_cast<const BinNode*>(host[2].data());
    uint64_t n_bin = host[2].size() / 32;
    const float* leaves = reinterpret_cast<const float*>(host[1].data());
    uint64_t n_leaf_tris = host[1].size() / 48;
    const uint32_t* tables = reinterpret_cast<const uint32_t*>(host[3].data());
    uint64_t n_tv = host[3].size() / 16;
    Builder B{bn, n_bin, {}, {}};
    std::vector<float> wtris;
    std::vector<uint32_t> top_items;
    uint32_t top = P[P_MOTION_Z], n_units = P[P_MOTION_W];
    uint32_t t_inst = P[P_T_INSTANCES];
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> mesh_root;  // (binary root, first triangle) -> wide root
    std::vector<uint32_t> unit_roots;
    uint32_t top_root = 0;
    if (n_units > 0) {
        // The top tree's leaves name unit records; a record's mesh tree is at its n0.w, its triangles from info.x.
        auto unit_leaf = [&](const BinNode& n) -> uint32_t {
            uint32_t first = (uint32_t)top_items.size();
            for (uint32_t j = 0; j < n.count; ++j) {
                uint32_t rec = n.left_or_first + j;
                uint64_t b = (uint64_t)t_inst + (uint64_t)rec * 10u;
                if (b + 10 > n_tv) { B.error = "a unit's record is past the tables"; return UINT32_MAX; }
                const uint32_t* r = tables + 4 * b;
                uint32_t bits = r[4 * 4 + 3];
                top_items.push_back(rec | ((bits & UNIT_SHADOW) ? WIDE_UNIT_BIT : 0u));
                uint32_t root = r[3 * 4 + 3], first_tri = r[6 * 4 + 0];
                auto key2 = std::make_pair(root, first_tri);
                uint32_t wr;
                auto it = mesh_root.find(key2);
                if (it == mesh_root.end()) {
                    auto tri_leaf = [&](const BinNode& m) -> uint32_t {
                        uint32_t f = (uint32_t)(wtris.size() / 12);
                        for (uint32_t q = 0; q < m.count; ++q) {
                            uint64_t ti = (uint64_t)first_tri + m.left_or_first + q;
                            if (ti >= n_leaf_tris) { B.error = "a leaf names a triangle past the leaves"; return UINT32_MAX; }
                            const float* l = leaves + 12 * ti;
                            float rec12[12];
                            std::memcpy(rec12, l, 48);
                            uint32_t tiu = (uint32_t)ti;
                            std::memcpy(&rec12[11], &tiu, 4);
                            wtris.insert(wtris.end(), rec12, rec12 + 12);
                        }
                        return f;
                    };
                    wr = B.collapse(root, tri_leaf, 16, false);
                    if (wr == UINT32_MAX) return UINT32_MAX;
                    mesh_root.emplace(key2, wr);
                } else {
                    wr = it->second;
                }
                if (unit_roots.size() <= rec) unit_roots.resize(rec + 1, 0);
                unit_roots[rec] = wr;
            }
            return first;
        };
        // Collapse the top tree with its unit leaves (mesh trees are collapsed as their units are met).
        top_root = B.collapse(top, unit_leaf, 16, true);
        if (top_root == UINT32_MAX) {
            error = B.error;
            return 1;
        }
    }
    uint32_t n_wn = (uint32_t)B.out.size();
    // Room after the built nodes for the top tree collapsed again after a deformation: at most a node a unit.
    uint32_t cap = n_units > 0 ? n_units + 1u : 0u;
    cudaError_t e = cudaSuccess;
    auto upload = [&](void** dst, const void* src, size_t bytes, size_t room = 0) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(dst, std::max<size_t>(bytes + room, 16));
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && room) e = cudaMemsetAsync((char*)*dst + bytes, 0, room, st);
    };
    if (top_items.empty()) top_items.push_back(0);
    if (unit_roots.empty()) unit_roots.push_back(0);
    upload((void**)&nodes, B.out.data(), B.out.size() * sizeof(WNode), (size_t)cap * sizeof(WNode));
    upload((void**)&tris, wtris.data(), wtris.size() * 4);
    upload((void**)&units, top_items.data(), top_items.size() * 4);
    upload((void**)&unit_root, unit_roots.data(), unit_roots.size() * 4);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        error = std::string("wide BVH upload: ") + cudaGetErrorString(e);
        release();
        return 1;
    }
    v = WideView{nodes, tris, units, unit_root, top_root, n_wn, (uint32_t)(wtris.size() / 12),
                 (uint32_t)top_items.size(), (uint32_t)unit_roots.size()};
    if (n_units == 0) v.n_units = 0;
    slot_host = std::move(B.slots);
    pad_host = std::move(B.pads);
    slot_host.resize(8ull * n_wn, WIDE_SLOT_EMPTY);
    pad_host.resize(n_wn, 0.0f);
    n_built = n_wn;
    top_cap = cap;
    refit_gen = 0;
    std::memcpy(key, k, sizeof(k));
    built = true;
    build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

}  // namespace trt
