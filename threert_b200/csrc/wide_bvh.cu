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

    // Quantises the child boxes of one wide node (wide_bvh.cuh's layout) and writes its header.
    void encode(WNode& W, const std::vector<const BinNode*>& ch, const std::vector<bool>& interior, uint32_t child_base,
                uint32_t leaf_base, const std::vector<uint32_t>& counts, float tree_pad) {
        std::memset(&W, 0, sizeof(W));
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (const BinNode* c : ch)
            if (c)
                for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], c->bmin[k]); hi[k] = std::max(hi[k], c->bmax[k]); }
        float origin[3];
        int ex[3];
        for (int k = 0; k < 3; ++k) {
            float ext = hi[k] - lo[k];
            float mag = std::max(std::fabs(lo[k]), std::fabs(hi[k]));
            // A step's margin on every side is added per child; this pad keeps the widened boxes inside 0..255 and
            // gives flat boxes a width of some 2^-16 of their coordinates.
            float pad = ext * (1.0f / 253.0f) + mag * (1.0f / 65536.0f) + tree_pad + 1e-20f;
            origin[k] = lo[k] - pad;
            float range = (hi[k] + pad) - origin[k];
            int e;
            std::frexp(range / 255.0f, &e);  // range / 255 < 2^e
            while (std::ldexp(255.0f, e) < range) ++e;
            ex[k] = std::max(-126, std::min(127, e));
        }
        uint8_t qlo[3][8], qhi[3][8];
        for (int i = 0; i < 8; ++i)
            for (int k = 0; k < 3; ++k) { qlo[k][i] = 255; qhi[k][i] = 0; }
        for (size_t i = 0; i < ch.size(); ++i) {
            if (!ch[i]) continue;
            for (int k = 0; k < 3; ++k) {
                float s = std::ldexp(1.0f, ex[k]);
                double a = std::floor((double)(ch[i]->bmin[k] - origin[k]) / s) - 1.0;
                double b = std::ceil((double)(ch[i]->bmax[k] - origin[k]) / s) + 1.0;
                qlo[k][i] = (uint8_t)std::max(0.0, std::min(255.0, a));
                qhi[k][i] = (uint8_t)std::max(0.0, std::min(255.0, b));
            }
        }
        uint32_t imask = 0;
        for (size_t i = 0; i < ch.size(); ++i)
            if (interior[i]) imask |= 1u << i;
        std::memcpy(&W.w[0], origin, 12);
        W.w[3] = (uint32_t)(ex[0] + 127) | ((uint32_t)(ex[1] + 127) << 8) | ((uint32_t)(ex[2] + 127) << 16) | (imask << 24);
        W.w[4] = child_base;
        W.w[5] = leaf_base;
        uint8_t cnt[8] = {0};
        for (size_t i = 0; i < ch.size(); ++i) cnt[i] = (interior[i] || !ch[i]) ? 0 : (uint8_t)counts[i];
        std::memcpy(&W.w[6], cnt, 8);
        uint8_t* q = reinterpret_cast<uint8_t*>(&W.w[8]);
        for (int k = 0; k < 3; ++k) std::memcpy(q + 8 * k, qlo[k], 8);
        for (int k = 0; k < 3; ++k) std::memcpy(q + 24 + 8 * k, qhi[k], 8);
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
    template <class Leaf>
    uint32_t collapse(uint32_t root, Leaf&& leaf, uint32_t max_leaf_items) {
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

        }
        return wroot;
    }
};

constexpr uint32_t P_MOTION_Z = 70, P_MOTION_W = 71, P_T_INSTANCES = 124 + 7, P_W_INDICES = 136 + 4;

}  // namespace

void WideBvh::release() {
    if (nodes) cudaFree(nodes);
    if (tris) cudaFree(tris);
    if (units) cudaFree(units);
    if (unit_root) cudaFree(unit_root);
    nodes = nullptr;
    tris = nullptr;
    units = nullptr;
    unit_root = nullptr;
    built = false;
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
                    wr = B.collapse(root, tri_leaf, 16);
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
        top_root = B.collapse(top, unit_leaf, 16);
        if (top_root == UINT32_MAX) {
            error = B.error;
            return 1;
        }
    }
    uint32_t n_wn = (uint32_t)B.out.size();
    cudaError_t e = cudaSuccess;
    auto upload = [&](void** dst, const void* src, size_t bytes) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(dst, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st);
    };
    if (top_items.empty()) top_items.push_back(0);
    if (unit_roots.empty()) unit_roots.push_back(0);
    upload((void**)&nodes, B.out.data(), B.out.size() * sizeof(WNode));
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
    std::memcpy(key, k, sizeof(k));
    built = true;
    build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

}  // namespace trt
