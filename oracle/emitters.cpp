// Test infrastructure, not product code: the CPU oracle of the emitters' re-weigh.
//
// renderer/shaders/emitter_weights.wgsl (weigh 67-90, scan_a 93-106, scan_b 108-119, scan_c 121-131, guide 135-153,
// tree 157-177, finish 185-192) with the levels of ltree.rs:233-256, restated on host arrays: the scene's tables and
// words after trt_prep, the Params' table and word offsets. The device re-weigh (threert_b200/csrc/emitters.cuh) is
// held to it bit for bit; it is held to the prep's own tables (lib.rs:451-485 emitter_cdf, ltree.rs:260-272 refit) to
// float rounding (the blocked scan rounds otherwise than one running sum).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

const uint32_t INSTANCE_VEC4 = 10, MATERIAL_VEC4 = 18, NO_INST = 0xffffffffu, EMITTER_MOVES = 0x80000000u,
               EMITTER_GONE = 2, EMITTER_NOMINAL = 4, ROW_MATERIAL = 0xffffffu, LEAF = 0x80000000u, GUIDE = 65536,
               BLOCK = 256, LEVELS = 32;

float fb(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
uint32_t bu(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

struct Tables {
    uint32_t* t;  // 4 words a vec4
    uint64_t n;
    uint32_t* v(uint64_t i) { return t + 4 * i; }
};

}  // namespace

extern "C" void orc_weigh_emitters(uint32_t* tables, uint64_t n_vec4, const uint32_t* words, uint64_t n_words,
                                   const uint32_t* P, uint32_t tree_nodes, const float* lod, const float* cull) {
    (void)n_words;
    Tables T{tables, n_vec4};
    const uint32_t n = P[21];  // counts.y: the emitters
    if (n == 0) return;
    const uint32_t list = P[124 + 11], entries = P[124 + 4], tree = P[124 + 0], instances = P[124 + 7],
                   materials = P[124 + 1], objects = P[124 + 6], rows = P[136 + 3], stride = 3;
    const bool use_lod = lod && lod[3] > 0.0f;
    auto light_lod = [&](float cx, float cy, float cz) {
        float dx = cx - lod[0], dy = cy - lod[1], dz = cz - lod[2];
        float d = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (cull && cull[0] > 0.0f && d > cull[0] && !(d <= cull[1] && dx * cull[3] + dy * cull[4] + dz * cull[5] >= cull[2] * d))
            return 0.0f;
        float k = lod[3] / std::max(d, lod[3]);
        return k * k;
    };
    // weigh
    for (uint32_t id = 0; id < n; ++id) {
        uint32_t* e = T.v(entries + id);
        uint64_t r = list + (uint64_t)e[0] * 4;
        const uint32_t *r0 = T.v(r), *r1 = T.v(r + 1), *r2 = T.v(r + 2), *r3 = T.v(r + 3);
        float e1x = fb(r1[0]), e1y = fb(r1[1]), e1z = fb(r1[2]), e2x = fb(r2[0]), e2y = fb(r2[1]), e2z = fb(r2[2]);
        float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
        float area = 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
        if (r3[1] & EMITTER_NOMINAL) area = fb(r3[2]);
        float w = 0.0f;
        if ((r3[1] & EMITTER_GONE) || r1[3] == NO_INST) {
            area = 0.0f;
        } else {
            const uint32_t* info = T.v(instances + (uint64_t)r1[3] * INSTANCE_VEC4 + 6);
            uint32_t m = words[rows + ((uint64_t)info[3] + r3[0]) * 4] & ROW_MATERIAL;
            const uint32_t* em = T.v(materials + (uint64_t)m * MATERIAL_VEC4 + 1);
            float power = fb(T.v(objects + (uint64_t)info[1] * stride)[3]);
            w = area * (fb(em[0]) * 0.2126f + fb(em[1]) * 0.7152f + fb(em[2]) * 0.0722f) * power;
            if (use_lod && !(r2[3] & EMITTER_MOVES))
                w *= light_lod(fb(r0[0]) + (e1x + e2x) / 3.0f, fb(r0[1]) + (e1y + e2y) / 3.0f,
                               fb(r0[2]) + (e1z + e2z) / 3.0f);
        }
        uint32_t ex = e[0];
        e[0] = ex;
        e[1] = bu(0.0f);
        e[2] = bu(std::max(w, 0.0f));
        e[3] = bu(area);
    }
    // scan_a, scan_b
    uint32_t nb = (n + BLOCK - 1) / BLOCK;
    std::vector<float> bsum(nb + 1), boff(nb + 1);
    for (uint32_t b = 0; b < nb; ++b) {
        uint32_t lo = b * BLOCK, hi = std::min(lo + BLOCK, n);
        float sum = 0.0f;
        for (uint32_t k = lo; k < hi; ++k) {
            uint32_t* e = T.v(entries + k);
            sum += fb(e[2]);
            e[1] = bu(sum);
        }
        bsum[b] = sum;
    }
    float sum = 0.0f;
    for (uint32_t b = 0; b < nb; ++b) {
        boff[b] = sum;
        sum += bsum[b];
    }
    float total = sum;
    // scan_c
    for (uint32_t id = 0; id < n; ++id) {
        uint32_t* e = T.v(entries + id);
        float c = boff[id / BLOCK] + fb(e[1]);
        e[1] = bu(total > 0.0f ? (c >= total ? 1.0f : c / total) : 0.0f);
    }
    // guide
    for (uint32_t id = 0; id <= GUIDE / 4; ++id) {
        uint32_t out[4] = {0, 0, 0, 0};
        for (uint32_t c = 0; c < 4; ++c) {
            uint32_t k = id * 4 + c;
            if (k > GUIDE) break;
            float u = (float)k / (float)GUIDE;
            uint32_t lo = 0, hi = n;
            for (uint32_t s = 0; s < 32 && lo < hi; ++s) {
                uint32_t mid = (lo + hi) / 2;
                if (fb(T.v(entries + mid)[1]) < u) lo = mid + 1;
                else hi = mid;
            }
            out[c] = lo;
        }
        std::memcpy(T.v(entries + n + id), out, 16);
    }
    // tree, by ltree.rs levels: the reachable nodes, the deepest first
    if (tree_nodes > 0) {
        std::vector<uint32_t> depth(tree_nodes, 0xffffffffu);
        depth[0] = 0;
        for (uint32_t i = 0; i < tree_nodes; ++i) {
            uint32_t w = T.v(tree + i)[3];
            if (depth[i] != 0xffffffffu && !(w & LEAF) && (uint64_t)w + 1 < tree_nodes) depth[w] = depth[w + 1] = depth[i] + 1;
        }
        std::vector<uint32_t> order;
        for (uint32_t i = 0; i < tree_nodes; ++i)
            if (depth[i] != 0xffffffffu) order.push_back(i);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return depth[a] > depth[b]; });
        uint32_t levels_seen = 0;
        for (size_t k = 0; k < order.size(); ++k) {
            if (k == 0 || depth[order[k]] != depth[order[k - 1]]) ++levels_seen;
            if (levels_seen > LEVELS) break;
            uint32_t i = order[k];
            uint32_t* nd = T.v(tree + i);
            uint32_t w = nd[3];
            float power = 0.0f;
            if (w & LEAF) {
                uint32_t lo = w & 0x1fffffffu, hi = lo + ((w >> 29) & 3) + 1;
                for (uint32_t j = lo; j < hi; ++j) power += fb(T.v(entries + j)[2]);
            } else {
                power = fb(T.v(tree + w)[2]) + fb(T.v(tree + w + 1)[2]);
            }
            nd[2] = bu(power);
        }
    }
    // finish
    float tail = 0.0f;
    if (tree_nodes > 0 && total > 0.0f) tail = std::max((total - fb(T.v(tree)[2])) / total, 0.0f);
    uint32_t* h = T.v(entries + n + GUIDE / 4 + 1);
    h[0] = bu(total);
    h[1] = bu(tail);
    h[2] = bu(0.0f);
    h[3] = bu(0.0f);
}
