// Host prep: a scene description to the reference's packed buffers (include/threert_prep.h says which reference
// functions each part restates). Plain C++17, single-threaded where the reference is, no CUDA.
#include "threert_prep.h"

#include <algorithm>
#include <array>
#include <memory>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_error;

inline float bf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t bu(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
constexpr float F_INF = std::numeric_limits<float>::infinity();
constexpr float PI_F = 3.14159265358979f;

struct V3 {
    float x = 0, y = 0, z = 0;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 mk(float x, float y, float z) { V3 v; v.x = x; v.y = y; v.z = z; return v; }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
// glam's Vec3A::min / max (SSE minps / maxps): the first operand where it is smaller (larger), else the second.
inline float gmin(float a, float b) { return a < b ? a : b; }
inline float gmax(float a, float b) { return a > b ? a : b; }
inline V3 vmin(V3 a, V3 b) { return mk(gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return mk(gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)); }
// f32::total_cmp's key: orders every float, -0 before +0.
inline int32_t total_key(float f) {
    int32_t b;
    std::memcpy(&b, &f, 4);
    return b ^ (int32_t)(((uint32_t)(b >> 31)) >> 1);
}
inline V3 splat(float s) { return mk(s, s, s); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline bool finite3(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline float max_elem(V3 a) { return std::max(a.x, std::max(a.y, a.z)); }
inline V3 vabs(V3 a) { return mk(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }

// IEEE binary32 -> binary16, round to nearest even (half::f16::from_f32).
uint16_t float_to_half(float f) {
    uint32_t x = bu(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xffu;
    uint32_t man = x & 0x7fffffu;
    if (exp == 0xffu) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u : 0u));
    int32_t e = (int32_t)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t half_man = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u);
        uint32_t halfway = 1u << (shift - 1);
        if (rem > halfway || (rem == halfway && (half_man & 1u))) half_man++;
        return (uint16_t)(sign | half_man);
    }
    uint32_t half_man = man >> 13;
    uint32_t rem = man & 0x1fffu;
    uint32_t out = sign | ((uint32_t)e << 10) | half_man;
    if (rem > 0x1000u || (rem == 0x1000u && (half_man & 1u))) out++;
    return (uint16_t)out;
}
float half_to_float(uint16_t h) {
    uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    if (e == 0) {
        if (m == 0) return bf(s);
        float f = (float)m * (1.0f / 16777216.0f);
        return s ? -f : f;
    }
    if (e == 31) return bf(s | 0x7f800000u | (m << 13));
    return bf(s | ((e + 112u) << 23) | (m << 13));
}

// ------------------------------------------------------------------------------------------------------------------
// Trees (bvh.rs, units.rs)

struct GpuNode { float bmin[3]; uint32_t left_or_first; float bmax[3]; uint32_t count; };
static_assert(sizeof(GpuNode) == 32, "GpuNode is 32 bytes");
// bvh.rs:57 EMPTY / units.rs:48 FILL: a leaf of one item without a box.
const GpuNode EMPTY_NODE = {{0, 0, 0}, 0, {0, 0, 0}, 1};
const GpuNode ZERO_NODE = {{0, 0, 0}, 0, {0, 0, 0}, 0};

struct Aabb {
    V3 lo = splat(F_INF), hi = splat(-F_INF);
    void grow(V3 p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void merge(const Aabb& o) { lo = vmin(lo, o.lo); hi = vmax(hi, o.hi); }
    // bvh.rs:32-35
    float area() const {
        V3 e = vmax(hi - lo, splat(0.0f));
        return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
    }
    // bvh.rs:124-128
    bool finite() const { return finite3(lo) && finite3(hi) && lo.x <= hi.x && lo.y <= hi.y && lo.z <= hi.z; }
};
inline GpuNode make_node(V3 lo, uint32_t lf, V3 hi, uint32_t count) {
    GpuNode n;
    n.bmin[0] = lo.x; n.bmin[1] = lo.y; n.bmin[2] = lo.z;
    n.bmax[0] = hi.x; n.bmax[1] = hi.y; n.bmax[2] = hi.z;
    n.left_or_first = lf;
    n.count = count;
    return n;
}

constexpr size_t BINS = 16, MAX_LEAF = 4, SAH_LEAF = 16, BVH_STACK = 48;  // bvh.rs:47-55
constexpr size_t UNITS_STACK = 64, TOP_DEPTH = 19, MESH_DEPTH = UNITS_STACK - TOP_DEPTH;  // units.rs:30-37
constexpr size_t MAX_UNITS = size_t(1) << (TOP_DEPTH - 1);
constexpr uint32_t UNIT_MAX_LEAF = 16;
constexpr size_t TOP_BINS = 32;  // units.rs:138

// Rust's `f as usize`: saturating, NaN to 0.
inline size_t to_usize(float f) {
    if (!(f > 0.0f)) return 0;
    if (f >= 1.8e19f) return std::numeric_limits<size_t>::max();
    return (size_t)f;
}
// bvh.rs:115-117 levels
size_t levels(size_t count) {
    size_t c = (count + MAX_LEAF - 1) / MAX_LEAF;
    size_t p = 1, lv = 0;
    while (p < c) { p <<= 1; lv++; }
    return lv;
}

struct Bvh { std::vector<GpuNode> nodes; std::vector<uint32_t> order; size_t depth = 0; };

// bvh.rs:131-239 build_from
Bvh build_from(const std::vector<Aabb>& boxes, const std::vector<V3>& centroids, size_t max_depth) {
    Bvh out;
    for (uint32_t i = 0; i < boxes.size(); ++i)
        if (boxes[i].finite()) out.order.push_back(i);
    size_t n = out.order.size();
    for (uint32_t i = 0; i < boxes.size(); ++i)
        if (!boxes[i].finite()) out.order.push_back(i);
    out.nodes.push_back(ZERO_NODE);
    if (n == 0) return out;
    if (levels(n) > max_depth) throw std::runtime_error("items do not fit a tree of the asked depth");
    struct Task { size_t ni, start, end, depth; };
    std::vector<Task> stack{{0, 0, n, 0}};
    std::vector<uint32_t>& order = out.order;
    while (!stack.empty()) {
        Task tk = stack.back();
        stack.pop_back();
        out.depth = std::max(out.depth, tk.depth);
        Aabb bounds, cb;
        for (size_t k = tk.start; k < tk.end; ++k) {
            bounds.merge(boxes[order[k]]);
            cb.grow(centroids[order[k]]);
        }
        size_t count = tk.end - tk.start;
        auto make_leaf = [&]() { out.nodes[tk.ni] = make_node(bounds.lo, (uint32_t)tk.start, bounds.hi, (uint32_t)count); };
        if (count <= MAX_LEAF) { make_leaf(); continue; }
        V3 ext = cb.hi - cb.lo;
        float best_cost = F_INF;
        int best_axis = 0;
        size_t best_split = 0;
        for (int axis = 0; axis < 3; ++axis) {
            if (ext[axis] <= 1e-9f) continue;
            Aabb bin_box[BINS];
            size_t bin_cnt[BINS] = {};
            float scale = (float)BINS / ext[axis];
            for (size_t k = tk.start; k < tk.end; ++k) {
                uint32_t t = order[k];
                size_t b = std::min(to_usize((centroids[t][axis] - cb.lo[axis]) * scale), BINS - 1);
                bin_cnt[b]++;
                bin_box[b].merge(boxes[t]);
            }
            float left_area[BINS];
            size_t left_cnt[BINS];
            Aabb acc;
            size_t c = 0;
            for (size_t i = 0; i < BINS; ++i) {
                acc.merge(bin_box[i]);
                c += bin_cnt[i];
                left_area[i] = acc.area();
                left_cnt[i] = c;
            }
            Aabb racc;
            c = 0;
            for (size_t i = BINS - 1; i >= 1; --i) {
                racc.merge(bin_box[i]);
                c += bin_cnt[i];
                float cost = left_area[i - 1] * (float)left_cnt[i - 1] + racc.area() * (float)c;
                bool fits = tk.depth + 1 + levels(std::max(left_cnt[i - 1], c)) <= max_depth;
                if (left_cnt[i - 1] > 0 && c > 0 && cost < best_cost && fits) {
                    best_cost = cost;
                    best_axis = axis;
                    best_split = i;
                }
            }
        }
        float leaf_cost = bounds.area() * (float)count;
        bool splittable = std::isfinite(best_cost);
        if (count <= SAH_LEAF && (!splittable || best_cost >= leaf_cost)) { make_leaf(); continue; }
        size_t mid;
        if (splittable) {
            float scale = (float)BINS / ext[best_axis];
            size_t i = tk.start;
            for (size_t j = tk.start; j < tk.end; ++j) {
                size_t b = std::min(to_usize((centroids[order[j]][best_axis] - cb.lo[best_axis]) * scale), BINS - 1);
                if (b < best_split) { std::swap(order[i], order[j]); i++; }
            }
            mid = i;
        } else if (ext.x <= 1e-9f && ext.y <= 1e-9f && ext.z <= 1e-9f) {
            mid = tk.start + count / 2;
        } else {
            int axis = 0;
            for (int k = 1; k < 3; ++k)
                if (ext[k] >= ext[axis]) axis = k;  // max_by keeps the last of equals
            size_t half = count / 2;
            std::nth_element(order.begin() + tk.start, order.begin() + tk.start + half, order.begin() + tk.end,
                             [&](uint32_t p, uint32_t q) { return centroids[p][axis] < centroids[q][axis]; });
            mid = tk.start + half;
        }
        size_t left = out.nodes.size();
        out.nodes.push_back(ZERO_NODE);
        out.nodes.push_back(ZERO_NODE);
        out.nodes[tk.ni] = make_node(bounds.lo, (uint32_t)left, bounds.hi, 0);
        stack.push_back({left + 1, mid, tk.end, tk.depth + 1});
        stack.push_back({left, tk.start, mid, tk.depth + 1});
    }
    return out;
}

// bvh.rs:81-98 build_tris
Bvh build_tris(const std::vector<std::array<V3, 3>>& tris, size_t max_depth) {
    if (tris.empty()) {
        Bvh b;
        b.nodes.push_back(EMPTY_NODE);
        return b;
    }
    std::vector<Aabb> boxes;
    std::vector<V3> cent;
    boxes.reserve(tris.size());
    cent.reserve(tris.size());
    for (const auto& t : tris) {
        Aabb b;
        if (finite3(t[0]) && finite3(t[1]) && finite3(t[2]))
            for (const V3& p : t) b.grow(p);
        boxes.push_back(b);
        V3 s = t[0] + t[1] + t[2];
        cent.push_back(mk(s.x / 3.0f, s.y / 3.0f, s.z / 3.0f));  // bvh.rs:93: (a + b + c) / 3
    }
    Bvh b = build_from(boxes, cent, max_depth);
    if (b.nodes.size() == 1 && b.nodes[0].count == 0) {
        Bvh e;
        e.nodes.push_back(EMPTY_NODE);
        e.order = b.order;
        return e;
    }
    return b;
}

// bvh.rs:246-285 check_tree; returns depth or -1 with g_error.
long check_tree(const GpuNode* nodes, size_t n_nodes, size_t max_depth, uint32_t max_leaf, uint64_t n_items) {
    if (n_nodes == 0) { g_error = "a tree without nodes"; return -1; }
    std::vector<char> seen(n_nodes, 0);
    std::vector<std::pair<size_t, size_t>> stack{{0, 0}};
    size_t deepest = 0, reached = 0;
    while (!stack.empty()) {
        auto [i, depth] = stack.back();
        stack.pop_back();
        if (seen[i]) { g_error = "node " + std::to_string(i) + " is reached twice"; return -1; }
        seen[i] = 1;
        reached++;
        deepest = std::max(deepest, depth);
        const GpuNode& n = nodes[i];
        if (n.count > 0) {
            if (n.count > max_leaf || (uint64_t)n.left_or_first + n.count > n_items) {
                g_error = "leaf " + std::to_string(i) + ": items out of range";
                return -1;
            }
            continue;
        }
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(n.bmin[k]) || !std::isfinite(n.bmax[k]) || n.bmin[k] > n.bmax[k]) {
                g_error = "node " + std::to_string(i) + "'s box is not finite";
                return -1;
            }
        size_t l = n.left_or_first;
        if (l <= i || l + 1 >= n_nodes) { g_error = "children not after their parent"; return -1; }
        if (depth + 1 > max_depth) { g_error = "deeper than allowed"; return -1; }
        stack.push_back({l, depth + 1});
        stack.push_back({l + 1, depth + 1});
    }
    if (reached != n_nodes) { g_error = "nodes not reached"; return -1; }
    return (long)deepest;
}

using Box = std::pair<V3, V3>;

// units.rs:84-122 build_median
void build_median(const std::vector<Box>& boxes, size_t max_leaf, std::vector<GpuNode>& nodes, std::vector<uint32_t>& order) {
    order.resize(boxes.size());
    std::iota(order.begin(), order.end(), 0u);
    nodes.assign(1, EMPTY_NODE);
    if (boxes.empty()) return;
    auto centre = [&](uint32_t k) { return (boxes[k].first + boxes[k].second) * 0.5f; };
    struct T { size_t ni, start, end; };
    std::vector<T> stack{{0, 0, boxes.size()}};
    while (!stack.empty()) {
        T t = stack.back();
        stack.pop_back();
        V3 lo = splat(F_INF), hi = splat(-F_INF), clo = lo, chi = hi;
        for (size_t k = t.start; k < t.end; ++k) {
            lo = vmin(lo, boxes[order[k]].first);
            hi = vmax(hi, boxes[order[k]].second);
            clo = vmin(clo, centre(order[k]));
            chi = vmax(chi, centre(order[k]));
        }
        size_t count = t.end - t.start;
        if (count <= max_leaf) { nodes[t.ni] = make_node(lo, (uint32_t)t.start, hi, (uint32_t)count); continue; }
        V3 ext = chi - clo;
        int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
        size_t mid = count / 2;
        std::nth_element(order.begin() + t.start, order.begin() + t.start + mid, order.begin() + t.end,
                         [&](uint32_t a, uint32_t b) {
                             float ca = centre(a)[axis], cb = centre(b)[axis];
                             return ca < cb || (ca == cb && a < b);
                         });
        size_t left = nodes.size();
        nodes.push_back(EMPTY_NODE);
        nodes.push_back(EMPTY_NODE);
        nodes[t.ni] = make_node(lo, (uint32_t)left, hi, 0);
        stack.push_back({left + 1, t.start + mid, t.end});
        stack.push_back({left, t.start, t.start + mid});
    }
}

inline float box_area(V3 lo, V3 hi) {
    V3 e = vmax(hi - lo, splat(0.0f));
    return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
}

// units.rs:140-224 build_sah (one box a leaf, at most max_depth deep)
void build_sah(const std::vector<Box>& boxes, size_t max_depth, std::vector<GpuNode>& nodes, std::vector<uint32_t>& order) {
    order.resize(boxes.size());
    std::iota(order.begin(), order.end(), 0u);
    nodes.assign(1, EMPTY_NODE);
    if (boxes.empty()) return;
    std::vector<V3> centres(boxes.size());
    for (size_t k = 0; k < boxes.size(); ++k) centres[k] = (boxes[k].first + boxes[k].second) * 0.5f;
    struct T { size_t ni, start, end, depth; };
    std::vector<T> stack{{0, 0, boxes.size(), 0}};
    while (!stack.empty()) {
        T t = stack.back();
        stack.pop_back();
        V3 lo = splat(F_INF), hi = splat(-F_INF), clo = lo, chi = hi;
        for (size_t k = t.start; k < t.end; ++k) {
            uint32_t b = order[k];
            lo = vmin(lo, boxes[b].first);
            hi = vmax(hi, boxes[b].second);
            clo = vmin(clo, centres[b]);
            chi = vmax(chi, centres[b]);
        }
        size_t count = t.end - t.start;
        if (count == 1) { nodes[t.ni] = make_node(lo, (uint32_t)t.start, hi, 1); continue; }
        size_t shift = max_depth - t.depth - 1;
        size_t room = shift >= 63 ? std::numeric_limits<size_t>::max() : (size_t(1) << shift);
        V3 ext = chi - clo;
        auto bin = [&](uint32_t k, int axis) {
            return std::min(to_usize((centres[k][axis] - clo[axis]) * ((float)TOP_BINS / ext[axis])), TOP_BINS - 1);
        };
        float best_cost = F_INF;
        int best_axis = 0;
        size_t best_split = 0;
        for (int axis = 0; axis < 3; ++axis) {
            if (!(ext[axis] > 0.0f)) continue;
            V3 blo[TOP_BINS], bhi[TOP_BINS];
            size_t bc[TOP_BINS] = {};
            for (size_t i = 0; i < TOP_BINS; ++i) { blo[i] = splat(F_INF); bhi[i] = splat(-F_INF); }
            for (size_t k = t.start; k < t.end; ++k) {
                size_t b = bin(order[k], axis);
                blo[b] = vmin(blo[b], boxes[order[k]].first);
                bhi[b] = vmax(bhi[b], boxes[order[k]].second);
                bc[b]++;
            }
            float right[TOP_BINS] = {};
            V3 alo = splat(F_INF), ahi = splat(-F_INF);
            for (size_t i = TOP_BINS - 1; i >= 1; --i) {
                alo = vmin(alo, blo[i]);
                ahi = vmax(ahi, bhi[i]);
                right[i] = box_area(alo, ahi);
            }
            alo = splat(F_INF);
            ahi = splat(-F_INF);
            size_t nl = 0;
            for (size_t i = 1; i < TOP_BINS; ++i) {
                alo = vmin(alo, blo[i - 1]);
                ahi = vmax(ahi, bhi[i - 1]);
                nl += bc[i - 1];
                size_t nr = count - nl;
                if (nl == 0 || nr == 0 || nl > room || nr > room) continue;
                float cost = box_area(alo, ahi) * (float)nl + right[i] * (float)nr;
                if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = i; }
            }
        }
        size_t mid;
        if (std::isfinite(best_cost)) {
            size_t i = 0;
            for (size_t j = 0; j < count; ++j) {
                if (bin(order[t.start + j], best_axis) < best_split) {
                    std::swap(order[t.start + i], order[t.start + j]);
                    i++;
                }
            }
            mid = i;
        } else {
            int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
            std::nth_element(order.begin() + t.start, order.begin() + t.start + count / 2, order.begin() + t.end,
                             [&](uint32_t a, uint32_t b) {
                                 int32_t ka = total_key(centres[a][axis]), kb = total_key(centres[b][axis]);
                                 return ka < kb || (ka == kb && a < b);
                             });
            mid = count / 2;
        }
        size_t left = nodes.size();
        nodes.push_back(EMPTY_NODE);
        nodes.push_back(EMPTY_NODE);
        nodes[t.ni] = make_node(lo, (uint32_t)left, hi, 0);
        stack.push_back({left + 1, t.start + mid, t.end, t.depth + 1});
        stack.push_back({left, t.start, t.start + mid, t.depth + 1});
    }
}

struct MeshTree { std::vector<GpuNode> nodes; std::vector<uint32_t> order; size_t depth = 0; V3 lo, hi; };

// units.rs:231-248 mesh_tree
MeshTree mesh_tree(const std::vector<std::array<V3, 3>>& tris) {
    if (tris.empty()) throw std::runtime_error("a mesh without triangles has no tree");
    for (const auto& t : tris)
        for (const V3& v : t)
            if (!finite3(v)) throw std::runtime_error("a mesh's vertex is not finite");
    MeshTree mt;
    Bvh b = build_tris(tris, BVH_STACK);
    long d = check_tree(b.nodes.data(), b.nodes.size(), MESH_DEPTH, UNIT_MAX_LEAF, tris.size());
    if (d >= 0) {
        mt.nodes = std::move(b.nodes);
        mt.order = std::move(b.order);
    } else {
        std::vector<Box> boxes;
        for (const auto& t : tris) boxes.push_back({vmin(vmin(t[0], t[1]), t[2]), vmax(vmax(t[0], t[1]), t[2])});
        build_median(boxes, 4, mt.nodes, mt.order);
    }
    d = check_tree(mt.nodes.data(), mt.nodes.size(), MESH_DEPTH, UNIT_MAX_LEAF, tris.size());
    if (d < 0) throw std::runtime_error("mesh tree: " + g_error);
    mt.depth = (size_t)d;
    mt.lo = splat(F_INF);
    mt.hi = splat(-F_INF);
    for (const auto& t : tris)
        for (const V3& v : t) { mt.lo = vmin(mt.lo, v); mt.hi = vmax(mt.hi, v); }
    return mt;
}

// A row-major 3x4 world matrix.
struct Mat34 { float m[3][4]; };
inline V3 transform_point(const Mat34& w, V3 p) {
    // glam's Mat4 * point: x_axis * x + y_axis * y + z_axis * z + w_axis
    return mk(w.m[0][0] * p.x + w.m[0][1] * p.y + w.m[0][2] * p.z + w.m[0][3],
              w.m[1][0] * p.x + w.m[1][1] * p.y + w.m[1][2] * p.z + w.m[1][3],
              w.m[2][0] * p.x + w.m[2][1] * p.y + w.m[2][2] * p.z + w.m[2][3]);
}

// units.rs:288-300 UnitBox::new
Box unit_box(const Mat34& world, V3 lo, V3 hi) {
    V3 a = splat(F_INF), b = splat(-F_INF);
    for (int c = 0; c < 8; ++c) {
        V3 p = transform_point(world, mk((c & 1) == 0 ? lo.x : hi.x, (c & 2) == 0 ? lo.y : hi.y, (c & 4) == 0 ? lo.z : hi.z));
        a = vmin(a, p);
        b = vmax(b, p);
    }
    float pad = max_elem(b - a) * 1e-4f + max_elem(vmax(vabs(a), vabs(b))) * 1e-5f + 1e-6f;
    return {a - splat(pad), b + splat(pad)};
}

// ------------------------------------------------------------------------------------------------------------------
// Records

constexpr uint32_t UNIT_SHADOW = 1, UNIT_SHIFTED = 2, INST_MIRRORED = 4;
constexpr uint32_t INST_BITS = 4 | 16 | 32 | 64 | 128;  // scene.rs:270
constexpr uint32_t NO_EMITTER = 0xffffffffu, NO_INST = 0xffffffffu;
constexpr uint32_t EMITTER_GUIDE = 65536;
constexpr uint32_t LT_LEAF = 0x80000000u, LT_PATH_BITS = 26;
constexpr size_t LT_MIN_STATIC = 256, LT_LEAF_MAX = 1;
constexpr uint32_t RIS_OFFLINE = 6;
constexpr uint32_t EMITTER_CARD = 1;

struct GpuInstance { float m[3][4]; float n[3][4]; uint32_t info[4]; float p[3][4]; };
static_assert(sizeof(GpuInstance) == 160, "GpuInstance is 160 bytes");
struct GpuMaterial { float base_color[4], emissive[4], params[4]; int32_t tex0[4], tex1[4]; float uv[4], uv2[4], layer[4], mp[8][4]; int32_t mt[8]; };
static_assert(sizeof(GpuMaterial) == 288, "GpuMaterial is 288 bytes");
struct GpuLight { float pos[4], dir[4], color[4], ext[4], x[4]; };
static_assert(sizeof(GpuLight) == 80, "GpuLight is 80 bytes");
struct GpuEmitterTri { float v0[3]; uint32_t tri; float e1[3]; uint32_t inst; float e2[3]; uint32_t code; uint32_t part, flags, nominal, spare; };
static_assert(sizeof(GpuEmitterTri) == 64, "GpuEmitterTri is 64 bytes");

// scene.rs:239-247 Instance::gpu: world rows, normal rows (inverse transpose of the 3x3, glam's Mat3::inverse:
// the columns' cross products over the determinant), info (first triangle, object, first vertex, rows' first).
GpuInstance instance_gpu(const Mat34& w, uint32_t first_tri, uint32_t object, uint32_t verts, uint32_t rows, uint32_t bits) {
    GpuInstance r;
    std::memset(&r, 0, sizeof(r));
    V3 cx = mk(w.m[0][0], w.m[1][0], w.m[2][0]), cy = mk(w.m[0][1], w.m[1][1], w.m[2][1]), cz = mk(w.m[0][2], w.m[1][2], w.m[2][2]);
    V3 t0 = cross(cy, cz), t1 = cross(cz, cx), t2 = cross(cx, cy);
    float det = dot(cz, t2);
    float inv = 1.0f / det;
    // nm = from_cols(t0, t1, t2) * inv_det; nrow(r) = [nm.x_axis[r], nm.y_axis[r], nm.z_axis[r]]
    V3 c0 = t0 * inv, c1 = t1 * inv, c2 = t2 * inv;
    bool mirrors = det < 0.0f;
    for (int k = 0; k < 3; ++k) {
        for (int c = 0; c < 4; ++c) { r.m[k][c] = w.m[k][c]; r.p[k][c] = w.m[k][c]; }
        r.n[k][0] = c0[k]; r.n[k][1] = c1[k]; r.n[k][2] = c2[k];
    }
    r.n[0][3] = 0.0f;
    r.n[1][3] = bf(bits | (mirrors ? INST_MIRRORED : 0u));
    r.n[2][3] = bf(0u);
    r.info[0] = first_tri; r.info[1] = object; r.info[2] = verts; r.info[3] = rows;
    return r;
}
// units.rs:343-345 translation_alone
bool translation_alone(const GpuInstance& r) {
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c)
            if (r.n[k][c] != (k == c ? 1.0f : 0.0f)) return false;
    return true;
}
// units.rs:329-334 unit_record
void unit_record(GpuInstance& r, uint32_t root, bool cast_shadow) {
    r.n[0][3] = bf(root);
    r.n[1][3] = bf((bu(r.n[1][3]) & INST_BITS) | (cast_shadow ? UNIT_SHADOW : 0u) | (translation_alone(r) ? UNIT_SHIFTED : 0u));
}

// ------------------------------------------------------------------------------------------------------------------
// Light tree (ltree.rs)

// ltree.rs:121-130 encode
void lt_encode(const float c[3], float r, float out[2]) {
    float hc[3];
    for (int k = 0; k < 3; ++k) hc[k] = half_to_float(float_to_half(c[k]));
    float gx = hc[0] - c[0], gy = hc[1] - c[1], gz = hc[2] - c[2];
    float grow = std::sqrt(gx * gx + gy * gy + gz * gz);
    uint16_t hr = float_to_half(r + grow);
    if (half_to_float(hr) < r + grow) hr = (uint16_t)(hr + 1);
    out[0] = bf((uint32_t)float_to_half(hc[0]) | ((uint32_t)float_to_half(hc[1]) << 16));
    out[1] = bf((uint32_t)float_to_half(hc[2]) | ((uint32_t)hr << 16));
}
// ltree.rs:133-137 box_sphere
void lt_box_sphere(const float lo[3], const float hi[3], float out[2]) {
    float c[3];
    for (int k = 0; k < 3; ++k) c[k] = 0.5f * (lo[k] + hi[k]);
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    float r = 0.5f * std::sqrt(dx * dx + dy * dy + dz * dz);
    lt_encode(c, r, out);
}

struct LtItem { uint32_t e; float lo[3], hi[3], c[3]; float w; };
struct LightTree {
    std::vector<std::array<float, 4>> nodes;
    std::vector<std::pair<uint32_t, uint32_t>> ranges;
    std::vector<uint32_t> order, code;
    float power = 0.0f;

    // ltree.rs:339-386 grow
    void grow(std::vector<LtItem>& items, size_t first, size_t root, uint32_t depth0, uint32_t path0) {
        struct T { size_t a, b, ni; uint32_t depth, path; };
        std::vector<T> stack{{0, items.size(), root, depth0, path0}};
        while (!stack.empty()) {
            T t = stack.back();
            stack.pop_back();
            float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(), std::numeric_limits<float>::max()};
            float hi[3] = {std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest()};
            float w = 0.0f;
            for (size_t i = t.a; i < t.b; ++i) {
                for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], items[i].lo[k]); hi[k] = std::max(hi[k], items[i].hi[k]); }
                w += items[i].w;
            }
            float s[2];
            lt_box_sphere(lo, hi, s);
            nodes[t.ni] = {s[0], s[1], w, 0.0f};
            ranges[t.ni] = {(uint32_t)(first + t.a), (uint32_t)(first + t.b)};
            size_t len = t.b - t.a;
            if (len <= LT_LEAF_MAX) {
                nodes[t.ni][3] = bf(LT_LEAF | ((uint32_t)(len - 1) << 29) | (uint32_t)(first + t.a));
                if (t.depth > LT_PATH_BITS) throw std::runtime_error("light tree deeper than its path bits");
                for (size_t k = 0; k < len; ++k) {
                    order[first + t.a + k] = items[t.a + k].e;
                    code[first + t.a + k] = ((t.depth + 1) << LT_PATH_BITS) | t.path;
                }
                continue;
            }
            float clo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(), std::numeric_limits<float>::max()};
            float chi[3] = {std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest()};
            for (size_t i = t.a; i < t.b; ++i)
                for (int k = 0; k < 3; ++k) { clo[k] = std::min(clo[k], items[i].c[k]); chi[k] = std::max(chi[k], items[i].c[k]); }
            int axis = 0;
            for (int k = 1; k < 3; ++k)
                if ((chi[k] - clo[k]) >= (chi[axis] - clo[axis])) axis = k;
            size_t mid = len / 2;
            // (ltree.rs orders by the centroid's coordinate under f32::total_cmp; equal ones here by their emitter's
            // index, so that the split does not depend on the selection's order of equals and the device build, which
            // orders them so, makes the same tree.)
            auto key = [&](const LtItem& p) {
                uint32_t b = bu(p.c[axis]);
                return ((uint64_t)((b & 0x80000000u) ? ~b : (b | 0x80000000u)) << 32) | p.e;
            };
            std::nth_element(items.begin() + t.a, items.begin() + t.a + mid, items.begin() + t.b,
                             [&](const LtItem& p, const LtItem& q) { return key(p) < key(q); });
            size_t left = nodes.size();
            nodes.push_back({0, 0, 0, 0});
            nodes.push_back({0, 0, 0, 0});
            ranges.push_back({0, 0});
            ranges.push_back({0, 0});
            nodes[t.ni][3] = bf((uint32_t)left);
            stack.push_back({t.a, t.a + mid, left, t.depth + 1, t.path});
            stack.push_back({t.a + mid, t.b, left + 1, t.depth + 1, t.path | (1u << t.depth)});
        }
    }
};

// ------------------------------------------------------------------------------------------------------------------
// Energy table (lib.rs:1041-1104)

void specular_albedo(double mu, double alpha, size_t nr, size_t nphi, double out[2]) {
    mu = std::min(std::max(mu, 1e-4), 1.0);
    if (alpha < 1e-6) {
        double fc = std::pow(1.0 - mu, 5);
        out[0] = 1.0 - fc;
        out[1] = fc;
        return;
    }
    double vx = std::sqrt(std::max(1.0 - mu * mu, 0.0)), vz = mu;
    double k = std::sqrt(alpha * alpha * vx * vx + vz * vz);
    double hx = alpha * vx / k, hz = vz / k;
    double s = 0.5 * (1.0 + hz);
    double inv_g1 = 0.5 * (1.0 + std::sqrt(1.0 + alpha * alpha * (1.0 - mu * mu) / (mu * mu)));
    double a = 0.0, b = 0.0;
    const double pi = 3.14159265358979323846;
    for (size_t i = 0; i < nr; ++i) {
        double t = ((double)i + 0.5) / (double)nr;
        double r = std::sqrt(1.0 - (1.0 - t) * (1.0 - t)), w = 2.0 * (1.0 - t);
        for (size_t j = 0; j < nphi; ++j) {
            double phi = pi * (((double)j + 0.5) / (double)nphi - 0.5);
            double p1 = r * std::cos(phi);
            double p2 = (1.0 - s) * std::sqrt(std::max(1.0 - p1 * p1, 0.0)) + s * r * std::sin(phi);
            double pz = std::sqrt(std::max(1.0 - p1 * p1 - p2 * p2, 0.0));
            double m0 = alpha * (pz * hx - p2 * hz), m1 = alpha * p1, m2 = std::max(p2 * hx + pz * hz, 0.0);
            double len = std::sqrt(m0 * m0 + m1 * m1 + m2 * m2);
            double voh = (vx * m0 + vz * m2) / len;
            double nol = 2.0 * voh * m2 / len - vz;
            if (nol <= 0.0 || voh <= 0.0) continue;
            double g2 = 2.0 * mu * nol / (nol * (mu * (1.0 - alpha) + alpha) + mu * (nol * (1.0 - alpha) + alpha));
            double fc = std::pow(1.0 - voh, 5);
            a += w * (1.0 - fc) * g2;
            b += w * fc * g2;
        }
    }
    double kk = inv_g1 / (double)(nr * nphi);
    out[0] = a * kk;
    out[1] = b * kk;
}
std::vector<std::array<float, 4>> energy_lut() {
    const size_t n = 32;
    std::vector<float> vals;
    vals.reserve(2 * n * n);
    for (size_t iy = 0; iy < n; ++iy) {
        double r = (double)iy / (double)(n - 1);
        for (size_t ix = 0; ix < n; ++ix) {
            double x = (double)ix / (double)(n - 1);
            double o[2];
            specular_albedo(x * x, r * r, 48, 8, o);
            vals.push_back((float)o[0]);
            vals.push_back((float)o[1]);
        }
    }
    std::vector<std::array<float, 4>> out;
    for (size_t i = 0; i < vals.size(); i += 4) out.push_back({vals[i], vals[i + 1], vals[i + 2], vals[i + 3]});
    return out;
}

// ------------------------------------------------------------------------------------------------------------------
// Sky (sky.rs:941-975 bake_gradient without glow or clouds; lib.rs:916-944 build_env_cdf)

struct EnvMap { uint32_t w = 1, h = 1; std::vector<std::array<float, 4>> texels; };

EnvMap bake_gradient(const trt_sky_spec& g) {
    EnvMap e;
    e.w = g.width ? g.width : 1024;
    e.h = g.height ? g.height : 512;
    e.texels.resize((size_t)e.w * e.h);
    V3 zen = mk(g.zenith[0], g.zenith[1], g.zenith[2]), hor = mk(g.horizon[0], g.horizon[1], g.horizon[2]),
       gnd = mk(g.ground[0], g.ground[1], g.ground[2]);
    auto lerp = [](V3 a, V3 b, float t) { return a + (b - a) * t; };  // glam's lerp: self + (rhs - self) * s
    for (size_t i = 0; i < e.texels.size(); ++i) {
        float x = (float)(i % e.w) + 0.5f, y = (float)(i / e.w) + 0.5f;
        float theta = y / (float)e.h * PI_F;
        float phi = (x / (float)e.w - 0.5f) * 2.0f * PI_F;
        V3 d = mk(std::sin(theta) * std::sin(phi), std::cos(theta), -std::sin(theta) * std::cos(phi));
        V3 l;
        if (d.y < 0.0f) {
            float k = std::min(-d.y / 0.08f, 1.0f);
            l = lerp(hor, gnd, k);
        } else {
            float el = std::asin(d.y);
            l = lerp(hor, zen, std::pow(el / (0.5f * PI_F), 0.45f));
        }
        e.texels[i] = {l.x, l.y, l.z, 1.0f};
    }
    return e;
}

std::vector<float> build_env_cdf(const EnvMap& env) {
    size_t w = env.w, h = env.h;
    std::vector<float> cond(w * h), rows(h);
    for (size_t y = 0; y < h; ++y) {
        float sin_t = std::sin((((float)y) + 0.5f) / (float)h * PI_F);
        float acc = 0.0f;
        for (size_t x = 0; x < w; ++x) {
            const auto& t = env.texels[y * w + x];
            acc += std::max(0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2], 0.0f) * sin_t + 1e-12f;
            cond[y * w + x] = acc;
        }
        rows[y] = acc;
        for (size_t x = 0; x < w; ++x) cond[y * w + x] /= acc;
    }
    float total = 0.0f;
    for (float r : rows) total += r;
    std::vector<float> out(h);
    float acc = 0.0f;
    for (size_t y = 0; y < h; ++y) {
        acc += rows[y] / total;
        out[y] = acc;
    }
    out.insert(out.end(), cond.begin(), cond.end());
    return out;
}

// heap.rs:127-135 place: sections of at least 512 bytes, each starting at a multiple of 256.
std::vector<uint64_t> place(const std::vector<uint64_t>& bytes, uint64_t& size) {
    std::vector<uint64_t> at;
    uint64_t end = 0;
    for (uint64_t b : bytes) {
        uint64_t cap = std::max<uint64_t>(b, 512);
        cap = (cap + 255) / 256 * 256;
        at.push_back(end);
        end += cap;
    }
    size = end;
    return at;
}

}  // namespace

// ------------------------------------------------------------------------------------------------------------------

struct trt_prepared {
    std::vector<std::array<float, 4>> vertices, leaves;
    std::vector<GpuNode> nodes;
    std::vector<uint32_t> tables, words;
    std::vector<uint16_t> env_half;
    uint32_t env_w = 1, env_h = 1;
    uint32_t params[156];
    trt_prep_info info;
    std::vector<uint32_t> lt_order, lt_code;
};

extern "C" {

const char* trt_prep_last_error(void) { return g_error.c_str(); }

int trt_prep_build(const trt_scene_spec* spec, trt_prepared** out) {
    try {
        auto P = std::make_unique<trt_prepared>();
        std::memset(P->params, 0, sizeof(P->params));
        std::memset(&P->info, 0, sizeof(P->info));
        const trt_scene_spec& S = *spec;
        if (S.n_meshes == 0 || S.n_instances == 0) throw std::runtime_error("a scene needs a mesh and an instance");
        // Objects: (pivot, power), (bounds size, time of its last power edit), custom data (scene.rs OBJECT_STRIDE 3).
        uint32_t n_objects = std::max<uint32_t>(S.n_objects, 1);
        for (uint32_t i = 0; i < S.n_instances; ++i) n_objects = std::max(n_objects, S.instances[i].object + 1);
        std::vector<std::array<float, 4>> objects((size_t)n_objects * 3, std::array<float, 4>{0, 0, 0, 0});
        for (uint32_t o = 0; o < n_objects; ++o) {
            objects[o * 3][3] = (S.object_power && o < S.n_objects) ? S.object_power[o] : 1.0f;
            objects[o * 3 + 1][3] = -1.0e9f;
        }
        auto obj_power = [&](uint32_t o) { return objects[(size_t)o * 3][3]; };

        // Materials (scene.rs:480-491).
        std::vector<GpuMaterial> mats(std::max<uint32_t>(S.n_materials, 1));
        for (auto& m : mats) {
            std::memset(&m, 0, sizeof(m));
            for (int k = 0; k < 4; ++k) { m.tex0[k] = -1; m.tex1[k] = -1; }
            m.tex1[2] = 0; m.tex1[3] = 0;
            m.uv[0] = 1.0f; m.uv[1] = 1.0f;
            for (int k = 0; k < 8; ++k) m.mt[k] = -1;
            m.base_color[3] = 1.0f;
            m.params[1] = 1.0f; m.params[3] = 1.0f;
        }
        for (uint32_t i = 0; i < S.n_materials; ++i) {
            const trt_material_spec& s = S.materials[i];
            GpuMaterial& m = mats[i];
            for (int k = 0; k < 4; ++k) m.base_color[k] = s.base_color[k];
            for (int k = 0; k < 3; ++k) m.emissive[k] = s.emissive[k];
            m.params[0] = s.metallic; m.params[1] = s.roughness; m.params[2] = s.specular; m.params[3] = 1.0f;
            m.tex1[2] = s.card ? 2 : 0;
        }
        auto lum = [](const float* c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; };
        auto emits = [&](uint32_t mi) { return mi < mats.size() && lum(mats[mi].emissive) > 0.0f; };

        // Mesh trees (lib.rs:865-943 unit_trees): each mesh's triangles put in its tree's order, ranked in sections.
        struct Mesh {
            uint32_t first = 0, count = 0, vfirst = 0, n_vertices = 0, n_sections = 1, root = 0;
            uint32_t like = NO_INST;  // the mesh whose triangles, tree and attributes this one repeats
            std::vector<std::array<V3, 3>> tris;
            std::vector<std::array<float, 4>> attr_n0, attr_n1, attr_n2;  // per corner normal + uv
            std::vector<uint32_t> section, rank;
            MeshTree tree;
        };
        std::vector<Mesh> meshes(S.n_meshes);
        // A mesh's triangles, tree and attributes: its own, or those of the mesh it repeats.
        auto data = [&](const Mesh& m) -> const Mesh& { return m.like == NO_INST ? m : meshes[m.like]; };
        uint32_t tri_total = 0;
        for (uint32_t mi = 0; mi < S.n_meshes; ++mi) {
            const trt_mesh_spec& ms = S.meshes[mi];
            Mesh& m = meshes[mi];
            if (ms.like) {
                if (ms.like - 1 >= mi) throw std::runtime_error("a mesh repeats one that is not before it");
                m.like = meshes[ms.like - 1].like == NO_INST ? ms.like - 1 : meshes[ms.like - 1].like;
                m.count = meshes[m.like].count;
                m.n_sections = meshes[m.like].n_sections;
                m.first = tri_total;
                tri_total += m.count;
                continue;
            }
            m.count = ms.n_tris;
            m.n_sections = std::max<uint32_t>(ms.n_sections, 1);
            std::vector<std::array<V3, 3>> tris(ms.n_tris);
            for (uint32_t t = 0; t < ms.n_tris; ++t)
                for (int c = 0; c < 3; ++c)
                    tris[t][c] = mk(ms.positions[t * 9 + c * 3], ms.positions[t * 9 + c * 3 + 1], ms.positions[t * 9 + c * 3 + 2]);
            m.tree = mesh_tree(tris);
            m.tris.resize(ms.n_tris);
            m.attr_n0.resize(ms.n_tris * 3);
            m.section.resize(ms.n_tris);
            m.rank.resize(ms.n_tris);
            std::vector<uint32_t> seen(m.n_sections, 0);
            for (uint32_t k = 0; k < ms.n_tris; ++k) {
                uint32_t src = m.tree.order[k];
                m.tris[k] = tris[src];
                V3 fn = cross(tris[src][1] - tris[src][0], tris[src][2] - tris[src][0]);
                float fl = std::sqrt(dot(fn, fn));
                if (fl > 0.0f) fn = mk(fn.x / fl, fn.y / fl, fn.z / fl);
                for (int c = 0; c < 3; ++c) {
                    V3 n = ms.normals ? mk(ms.normals[src * 9 + c * 3], ms.normals[src * 9 + c * 3 + 1], ms.normals[src * 9 + c * 3 + 2]) : fn;
                    float u = ms.uvs ? ms.uvs[src * 6 + c * 2] : 0.0f, v = ms.uvs ? ms.uvs[src * 6 + c * 2 + 1] : 0.0f;
                    // (normal, u) kept here with v in the 4th slot of the next: packed below as vertex records.
                    m.attr_n0[k * 3 + c] = {n.x, n.y, n.z, 0.0f};
                    m.attr_n0[k * 3 + c][3] = u;
                    (void)v;
                }
                uint32_t s = ms.sections ? ms.sections[src] : 0u;
                if (s >= m.n_sections) throw std::runtime_error("a triangle's section is past its mesh's sections");
                m.section[k] = s;
                m.rank[k] = seen[s]++;  // scene.rs:2406-2416 rank_in_sections
            }
            // (uvs' v kept separately: the vertex record holds (position, u), (normal, v).)
            m.attr_n1.resize(ms.n_tris * 3);
            for (uint32_t k = 0; k < ms.n_tris; ++k) {
                uint32_t src = m.tree.order[k];
                for (int c = 0; c < 3; ++c) m.attr_n1[k * 3 + c] = {ms.uvs ? ms.uvs[src * 6 + c * 2 + 1] : 0.0f, 0, 0, 0};
            }
            m.first = tri_total;
            tri_total += m.count;
            P->info.max_mesh_depth = std::max<uint32_t>(P->info.max_mesh_depth, (uint32_t)m.tree.depth);
        }

        // Shared vertices (indexed.rs): a mesh's corners that are the same record are one vertex; a triangle's
        // indices count from its mesh's first vertex. Leaves: (v0, section), (e1, rank), (e2, 0) (lib.rs:762-764).
        std::vector<uint32_t> indices;
        indices.reserve((size_t)tri_total * 3);
        P->leaves.reserve((size_t)tri_total * 3);
        for (Mesh& m : meshes) {
            m.vfirst = (uint32_t)(P->vertices.size() / 3);
            if (m.like != NO_INST) {
                // A repeat: the original's vertex records, indices (counted from the mesh's first vertex) and leaves.
                const Mesh& o = meshes[m.like];
                m.n_vertices = o.n_vertices;
                auto repeat = [](auto& v, size_t a, size_t b) {
                    size_t n = b - a, at = v.size();
                    v.resize(at + n);
                    std::copy(v.begin() + a, v.begin() + b, v.begin() + at);
                };
                repeat(P->vertices, 3ull * o.vfirst, 3ull * (o.vfirst + o.n_vertices));
                repeat(indices, 3ull * o.first, 3ull * (o.first + o.count));
                repeat(P->leaves, 3ull * o.first, 3ull * (o.first + o.count));
                continue;
            }
            std::unordered_map<std::string, uint32_t> seen;
            uint32_t nv = 0;
            for (uint32_t k = 0; k < m.count; ++k) {
                for (int c = 0; c < 3; ++c) {
                    const V3& p = m.tris[k][c];
                    const auto& na = m.attr_n0[k * 3 + c];
                    float u = na[3], v = m.attr_n1[k * 3 + c][0];
                    float rec[12] = {p.x, p.y, p.z, u, na[0], na[1], na[2], v, 0.0f, 0.0f, 0.0f, 0.0f};
                    std::string key(reinterpret_cast<const char*>(rec), sizeof(rec));
                    auto it = seen.find(key);
                    uint32_t idx;
                    if (it == seen.end()) {
                        idx = nv++;
                        seen.emplace(std::move(key), idx);
                        P->vertices.push_back({rec[0], rec[1], rec[2], rec[3]});
                        P->vertices.push_back({rec[4], rec[5], rec[6], rec[7]});
                        P->vertices.push_back({rec[8], rec[9], rec[10], rec[11]});
                    } else {
                        idx = it->second;
                    }
                    indices.push_back(idx);
                }
                V3 v0 = m.tris[k][0], e1 = m.tris[k][1] - v0, e2 = m.tris[k][2] - v0;
                P->leaves.push_back({v0.x, v0.y, v0.z, bf(m.section[k])});
                P->leaves.push_back({e1.x, e1.y, e1.z, bf(m.rank[k])});
                P->leaves.push_back({e2.x, e2.y, e2.z, 0.0f});
            }
            m.n_vertices = nv;
        }

        // Node buffer: the mesh trees side by side, then the top tree (units.rs Layout).
        for (Mesh& m : meshes) {
            m.root = (uint32_t)P->nodes.size();
            const auto& tn = data(m).tree.nodes;
            P->nodes.insert(P->nodes.end(), tn.begin(), tn.end());
        }
        uint32_t top_first = (uint32_t)P->nodes.size();

        // Instances: records, rows, unit boxes.
        std::vector<GpuInstance> insts;
        std::vector<std::array<uint32_t, 4>> rows;
        std::vector<Mat34> worlds(S.n_instances);
        std::vector<uint32_t> inst_rows(S.n_instances);
        std::vector<Box> unit_boxes;
        std::vector<uint32_t> unit_records;
        for (uint32_t r = 0; r < S.n_instances; ++r) {
            const trt_instance_spec& is = S.instances[r];
            if (is.mesh >= S.n_meshes) throw std::runtime_error("an instance names a mesh that is not there");
            Mesh& m = meshes[is.mesh];
            std::memcpy(worlds[r].m, is.world, sizeof(float) * 12);
            inst_rows[r] = (uint32_t)rows.size();
            for (uint32_t s = 0; s < m.n_sections; ++s) {
                uint32_t mat = is.section_materials ? is.section_materials[s] : 0u;
                if (mat >= mats.size()) throw std::runtime_error("an instance names a material that is not there");
                uint32_t sfirst = m.first;
                for (uint32_t k = 0; k < m.count; ++k)
                    if (data(m).section[k] == s) { sfirst = m.first + k; break; }
                rows.push_back({mat, sfirst, NO_EMITTER, 0u});  // scene.rs:115-118 row_of (class 0: opaque)
            }
            GpuInstance g = instance_gpu(worlds[r], m.first, is.object, m.vfirst, inst_rows[r], 0u);
            unit_record(g, m.root, is.cast_shadow != 0);
            insts.push_back(g);
            unit_boxes.push_back(unit_box(worlds[r], data(m).tree.lo, data(m).tree.hi));
            unit_records.push_back(r);
        }
        if (unit_boxes.size() > MAX_UNITS) throw std::runtime_error("more units than a top tree holds");
        // units.rs:303-326 top_tree: SAH down to one unit a leaf, a level less deep than TOP_DEPTH.
        std::vector<GpuNode> top;
        std::vector<uint32_t> top_order;
        build_sah(unit_boxes, TOP_DEPTH - 1, top, top_order);
        for (GpuNode& n : top)
            if (n.count > 0) n.left_or_first = unit_records[top_order[n.left_or_first]];
        long td = check_tree(top.data(), top.size(), TOP_DEPTH, 1, S.n_instances);
        if (td < 0) throw std::runtime_error("top tree: " + g_error);
        P->info.top_depth = (uint32_t)td;
        P->nodes.insert(P->nodes.end(), top.begin(), top.end());

        // Emitters (lib.rs:605-639, 190-214): an instance at a time, its emissive sections' triangles, a section
        // after another, each section's by rank.
        struct ETri { uint32_t tri, mat, obj; float area; float c[3]; uint32_t inst, part; bool card; };
        std::vector<ETri> etris;
        std::vector<GpuEmitterTri> getris;
        for (uint32_t r = 0; r < S.n_instances; ++r) {
            const trt_instance_spec& is = S.instances[r];
            Mesh& m = meshes[is.mesh];
            std::vector<int64_t> starts(m.n_sections, -1);
            std::vector<uint32_t> sec_count(m.n_sections, 0);
            const Mesh& md = data(m);
            for (uint32_t k = 0; k < m.count; ++k) sec_count[md.section[k]]++;
            uint32_t at = 0;
            for (uint32_t s = 0; s < m.n_sections; ++s)
                if (emits(rows[inst_rows[r] + s][0])) { starts[s] = at; at += sec_count[s]; }
            if (at == 0) continue;
            uint32_t first = (uint32_t)etris.size();
            for (uint32_t s = 0; s < m.n_sections; ++s)
                if (starts[s] >= 0) rows[inst_rows[r] + s][2] = first + (uint32_t)starts[s];
            std::vector<ETri> out(at);
            std::vector<GpuEmitterTri> gout(at);
            for (uint32_t k = 0; k < m.count; ++k) {
                uint32_t s = md.section[k];
                if (starts[s] < 0) continue;
                uint32_t slot = (uint32_t)starts[s] + md.rank[k];
                uint32_t mat = rows[inst_rows[r] + s][0];
                V3 w[3];
                for (int c = 0; c < 3; ++c) w[c] = transform_point(worlds[r], md.tris[k][c]);
                V3 cr = cross(w[1] - w[0], w[2] - w[0]);
                float area = 0.5f * std::sqrt(dot(cr, cr));
                V3 cen = w[0] + w[1] + w[2];
                ETri e{m.first + k, mat, is.object, area, {cen.x / 3.0f, cen.y / 3.0f, cen.z / 3.0f}, r, s, mats[mat].tex1[2] == 2};
                out[slot] = e;
                GpuEmitterTri g;
                std::memset(&g, 0, sizeof(g));
                V3 e1 = w[1] - w[0], e2 = w[2] - w[0];
                g.v0[0] = w[0].x; g.v0[1] = w[0].y; g.v0[2] = w[0].z;
                g.e1[0] = e1.x; g.e1[1] = e1.y; g.e1[2] = e1.z;
                g.e2[0] = e2.x; g.e2[1] = e2.y; g.e2[2] = e2.z;
                g.tri = e.tri;
                g.inst = r;
                g.part = s;
                g.flags = e.card ? EMITTER_CARD : 0u;
                gout[slot] = g;
            }
            etris.insert(etris.end(), out.begin(), out.end());
            getris.insert(getris.end(), gout.begin(), gout.end());
        }
        auto emitter_power = [&](const ETri& e) { return e.area * lum(mats[e.mat].emissive) * obj_power(e.obj); };

        // Light tree (ltree.rs:405-470; lib.rs:256-265 light_tree_of with every emitter on).
        LightTree lt;
        bool have_tree = false;
        if (S.use_light_tree) {
            std::vector<LtItem> fixed;
            for (uint32_t i = 0; i < etris.size(); ++i) {
                float w = emitter_power(etris[i]);
                if (!(w > 0.0f)) continue;
                // GpuEmitterTri::vertices (lib.rs:175-178): v0, v0 + e1, v0 + e2.
                const GpuEmitterTri& g = getris[i];
                float vs[3][3];
                for (int k = 0; k < 3; ++k) { vs[0][k] = g.v0[k]; vs[1][k] = g.v0[k] + g.e1[k]; vs[2][k] = g.v0[k] + g.e2[k]; }
                LtItem it;
                it.e = i;
                for (int k = 0; k < 3; ++k) {
                    it.lo[k] = std::min(std::min(std::min(std::numeric_limits<float>::max(), vs[0][k]), vs[1][k]), vs[2][k]);
                    it.hi[k] = std::max(std::max(std::max(std::numeric_limits<float>::lowest(), vs[0][k]), vs[1][k]), vs[2][k]);
                    // The centroid of the record's vertices (the reference takes the world vertices' before the record
                    // rounds them to v0, e1, e2: the same point to an ulp). A device build has only the record.
                    it.c[k] = (vs[0][k] + vs[1][k] + vs[2][k]) / 3.0f;
                }
                it.w = w;
                fixed.push_back(it);
            }
            if (fixed.size() >= LT_MIN_STATIC) {
                if (fixed.size() >= (1u << 29)) throw std::runtime_error("light tree entries beyond the child word");
                lt.nodes.assign(1, {0, 0, 0, 0});
                lt.ranges.assign(1, {0, 0});
                lt.order.assign(fixed.size(), 0);
                lt.code.assign(fixed.size(), 0);
                lt.grow(fixed, 0, 0, 0, 0);
                lt.power = lt.nodes[0][2];
                have_tree = true;
            }
        }
        // lib.rs:393-418 emitter_order, emitter_codes
        std::vector<uint32_t> order;
        std::vector<char> placed(etris.size(), 0);
        if (have_tree)
            for (uint32_t i : lt.order) { order.push_back(i); placed[i] = 1; }
        for (uint32_t i = 0; i < etris.size(); ++i)
            if (!placed[i]) order.push_back(i);
        size_t in_tree = have_tree ? lt.order.size() : 0;
        for (size_t k = 0; k < order.size(); ++k) getris[order[k]].code = k < in_tree ? lt.code[k] : (uint32_t)k;
        // lib.rs:437-479 emitter_cdf
        std::vector<std::array<float, 4>> emitters;
        float total = 0.0f, power = 0.0f;
        for (uint32_t i : order) {
            float p = emitter_power(etris[i]);
            power += p;
            total += p * 1.0f;
            emitters.push_back({bf(i), total, p * 1.0f, etris[i].area});
        }
        if (total > 0.0f)
            for (auto& e : emitters) e[1] /= total;
        {
            size_t n = emitters.size(), i = 0;
            std::vector<uint32_t> guide(EMITTER_GUIDE + 1);
            for (uint32_t k = 0; k <= EMITTER_GUIDE; ++k) {
                float u = (float)k / (float)EMITTER_GUIDE;
                while (i < n && emitters[i][1] < u) i++;
                guide[k] = (uint32_t)i;
            }
            for (size_t k = 0; k < guide.size(); k += 4) {
                std::array<float, 4> v{0, 0, 0, 0};
                for (size_t j = 0; j < 4; ++j) v[j] = bf(k + j < guide.size() ? guide[k + j] : 0u);
                emitters.push_back(v);
            }
            emitters.push_back({total, 0.0f, 0.0f, 0.0f});
        }
        float ltree_param[4] = {0, 0, 0, 0};
        if (have_tree) {
            ltree_param[1] = bf((uint32_t)lt.order.size());
            ltree_param[2] = total > 0.0f ? std::max((total - lt.power) / total, 0.0f) : 0.0f;
            ltree_param[3] = (float)RIS_OFFLINE;
        }
        emitters[etris.size() + (EMITTER_GUIDE + 1 + 3) / 4][1] = ltree_param[2];
        float all_power = 0.0f, em_area = 0.0f;
        for (const ETri& e : etris) all_power += emitter_power(e);
        for (size_t k = 0; k < etris.size(); ++k) em_area += emitters[k][3];

        // Sky (lib.rs:947-1000 bake_sky, 1005-1010 SkyBaked::write, 1012-1022).
        EnvMap env;
        V3 sky_color = mk(0, 0, 0);
        bool has_env = false;
        if (S.sky.kind == 2) {
            env = bake_gradient(S.sky);
            has_env = true;
        } else if (S.sky.kind == 3) {
            // The atmosphere (lib.rs:960-982): baked on the device (trt_sky_bake) and written over this black map of
            // the bake's size, its CDF, the sun's colour and Params (trt_prep_env, or trt_scene_set_sky in place).
            env.w = S.sky.width ? S.sky.width : 1024;
            env.h = S.sky.height ? S.sky.height : 512;
            env.texels.assign((size_t)env.w * env.h, {0.0f, 0.0f, 0.0f, 1.0f});
            has_env = true;
        } else {
            if (S.sky.kind == 1) sky_color = mk(S.sky.color[0], S.sky.color[1], S.sky.color[2]);
            env.texels.push_back({sky_color.x, sky_color.y, sky_color.z, S.sky.kind == 1 ? 1.0f : 0.0f});
        }
        std::vector<float> env_cdf = build_env_cdf(env);
        float env_nee_floor = etris.empty() ? 0.0f : 0.01f * all_power / std::max(em_area, 1e-6f);
        float brightest = 0.0f;
        for (const auto& t : env.texels) brightest = std::max(brightest, 0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2]);
        brightest = std::max(brightest, 0.2126f * sky_color.x + 0.7152f * sky_color.y + 0.0722f * sky_color.z);
        bool env_sampled = brightest >= env_nee_floor;
        P->env_w = env.w;
        P->env_h = env.h;
        P->env_half.resize(env.texels.size() * 4);
        for (size_t i = 0; i < env.texels.size(); ++i)
            for (int c = 0; c < 4; ++c) P->env_half[i * 4 + c] = float_to_half(env.texels[i][c]);

        // Lights (scene.rs:1315-1331; lib.rs:368-380 light order: directional first).
        std::vector<GpuLight> lights;
        for (uint32_t i = 0; i < S.n_lights; ++i) {
            const trt_dirlight_spec& l = S.lights[i];
            GpuLight g;
            std::memset(&g, 0, sizeof(g));
            V3 d = mk(l.dir[0], l.dir[1], l.dir[2]);
            float dl = std::sqrt(dot(d, d));
            d = mk(d.x / dl, d.y / dl, d.z / dl);
            float half = (l.angular_diameter_deg * 0.5f) * (PI_F / 180.0f);
            g.dir[0] = d.x; g.dir[1] = d.y; g.dir[2] = d.z;
            g.dir[3] = std::min(std::cos(half), 1.0f - std::numeric_limits<float>::epsilon() / 2.0f);
            for (int k = 0; k < 3; ++k) g.color[k] = l.color[k] * l.intensity;
            g.ext[3] = l.cast_shadow ? 1.0f : 0.0f;
            g.x[1] = l.specular_scale;
            lights.push_back(g);
        }

        // Heaps (heap.rs): tables in Table's order, words in Stream's.
        auto lut = energy_lut();
        std::vector<uint64_t> tbytes = {
            (uint64_t)lt.nodes.size() * 16, (uint64_t)mats.size() * 288, (uint64_t)lights.size() * 80, 0,
            (uint64_t)emitters.size() * 16, 0, (uint64_t)objects.size() * 16, (uint64_t)insts.size() * 160, 0,
            (uint64_t)lut.size() * 16, 0, (uint64_t)getris.size() * 64};
        uint64_t tsize = 0;
        std::vector<uint64_t> tat = place(tbytes, tsize);
        P->tables.assign(tsize / 4, 0u);
        auto put_t = [&](int k, const void* src, uint64_t bytes) {
            if (bytes) std::memcpy(reinterpret_cast<char*>(P->tables.data()) + tat[k], src, bytes);
        };
        put_t(0, lt.nodes.data(), tbytes[0]);
        put_t(1, mats.data(), tbytes[1]);
        put_t(2, lights.data(), tbytes[2]);
        put_t(4, emitters.data(), tbytes[4]);
        put_t(6, objects.data(), tbytes[6]);
        put_t(7, insts.data(), tbytes[7]);
        put_t(9, lut.data(), tbytes[9]);
        put_t(11, getris.data(), tbytes[11]);
        std::vector<uint64_t> wbytes = {(uint64_t)env_cdf.size() * 4, 0, 0, (uint64_t)rows.size() * 16, (uint64_t)indices.size() * 4};
        uint64_t wsize = 0;
        std::vector<uint64_t> wat = place(wbytes, wsize);
        P->words.assign(wsize / 4, 0u);
        std::memcpy(reinterpret_cast<char*>(P->words.data()) + wat[0], env_cdf.data(), wbytes[0]);
        if (wbytes[3]) std::memcpy(reinterpret_cast<char*>(P->words.data()) + wat[3], rows.data(), wbytes[3]);
        if (wbytes[4]) std::memcpy(reinterpret_cast<char*>(P->words.data()) + wat[4], indices.data(), wbytes[4]);

        // Params (lib.rs:713-758, gpu.rs:1971-1976, lib.rs:1005-1010).
        uint32_t* p = P->params;
        auto setf = [&](uint32_t w, float v) { p[w] = bu(v); };
        const trt_camera_spec& c = S.camera;
        for (int k = 0; k < 3; ++k) {
            setf(0 + k, c.position[k]); setf(4 + k, c.forward[k]); setf(8 + k, c.right[k]); setf(12 + k, c.up[k]);
        }
        setf(3, c.tan_half_fov);
        setf(7, (float)c.width / (float)c.height);
        setf(11, c.lens_radius);
        setf(15, c.focus_distance > 0.0f ? c.focus_distance : 1.0f);
        p[16] = c.width; p[17] = c.height; p[18] = 0; p[19] = S.seed;
        p[20] = (uint32_t)lights.size(); p[21] = (uint32_t)etris.size(); p[22] = S.preset.max_bounces; p[23] = S.preset.rr_depth;
        setf(24, has_env ? 1.0f : 0.0f); setf(25, (float)env.w); setf(26, (float)env.h); setf(27, -1.0f);
        setf(28, S.preset.clamp_indirect); setf(29, total); setf(30, S.preset.energy_compensation); setf(31, 0.0f);
        setf(32, sky_color.x); setf(33, sky_color.y); setf(34, sky_color.z); setf(35, 0.0f);
        p[36] = (uint32_t)lights.size(); p[37] = env_sampled ? 1u : 0u; p[38] = 0; p[39] = (uint32_t)lights.size();
        p[70] = top_first; p[71] = (uint32_t)unit_boxes.size();  // motion.zw (bits)
        setf(76, total);                                         // emit_power.x
        for (int k = 0; k < 4; ++k) p[84 + k] = bu(ltree_param[k]);
        p[89] = 0; p[90] = (uint32_t)insts.size();                 // procs: -, 0 objects, first record
        for (int k = 0; k < 12; ++k) p[124 + k] = (uint32_t)(tat[k] / 16);
        for (int k = 0; k < 5; ++k) p[136 + k] = (uint32_t)(wat[k] / 4);

        P->info.n_units = (uint32_t)unit_boxes.size();
        P->info.top_first = top_first;
        P->info.n_nodes = (uint32_t)P->nodes.size();
        P->info.n_tris = tri_total;
        P->info.n_vertices = (uint32_t)(P->vertices.size() / 3);
        P->info.n_emitters = (uint32_t)etris.size();
        P->info.light_tree_nodes = (uint32_t)lt.nodes.size();
        P->info.env_sampled = env_sampled ? 1u : 0u;
        P->info.emitter_total = total;
        P->info.env_nee_floor = env_nee_floor;
        if (have_tree) { P->lt_order = lt.order; P->lt_code = lt.code; }
        *out = P.release();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

void trt_prep_free(trt_prepared* p) { delete p; }

int trt_prep_env(const float* texels, uint32_t w, uint32_t h, uint16_t* env_half, float* cdf, float* brightest) {
    if (!texels || !w || !h) {
        g_error = "trt_prep_env: no texels";
        return 1;
    }
    EnvMap env;
    env.w = w;
    env.h = h;
    env.texels.resize((size_t)w * h);
    std::memcpy(env.texels.data(), texels, (size_t)w * h * 16);
    if (env_half)
        for (size_t i = 0; i < env.texels.size(); ++i)
            for (int c = 0; c < 4; ++c) env_half[i * 4 + c] = float_to_half(env.texels[i][c]);
    if (cdf) {
        std::vector<float> v = build_env_cdf(env);
        std::memcpy(cdf, v.data(), v.size() * 4);
    }
    if (brightest) {
        float b = 0.0f;
        for (const auto& t : env.texels) b = std::max(b, 0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2]);
        *brightest = b;
    }
    return 0;
}

void trt_prep_buffers(const trt_prepared* p, trt_prepared_buffers* o) {
    o->vertices = reinterpret_cast<const float*>(p->vertices.data());
    o->vertices_bytes = p->vertices.size() * 16;
    o->leaves = reinterpret_cast<const float*>(p->leaves.data());
    o->leaves_bytes = p->leaves.size() * 16;
    o->nodes = reinterpret_cast<const uint32_t*>(p->nodes.data());
    o->nodes_bytes = p->nodes.size() * 32;
    o->tables = p->tables.data();
    o->tables_bytes = p->tables.size() * 4;
    o->words = p->words.data();
    o->words_bytes = p->words.size() * 4;
    o->env_half = p->env_half.data();
    o->env_w = p->env_w;
    o->env_h = p->env_h;
}

void trt_prep_params(const trt_prepared* p, uint32_t out[156]) { std::memcpy(out, p->params, sizeof(p->params)); }

void trt_prep_get_info(const trt_prepared* p, trt_prep_info* out) { *out = p->info; }

uint32_t trt_prep_light_tree(const trt_prepared* p, uint32_t* order, uint32_t* codes, uint32_t cap) {
    uint32_t n = (uint32_t)p->lt_order.size();
    for (uint32_t i = 0; i < n && i < cap; ++i) {
        if (order) order[i] = p->lt_order[i];
        if (codes) codes[i] = p->lt_code[i];
    }
    return n;
}

uint32_t trt_prep_bvh(const float* tris, uint32_t n_tris, uint32_t max_depth, uint32_t* nodes, uint32_t nodes_cap,
                      uint32_t* order, uint32_t* depth) {
    try {
        std::vector<std::array<V3, 3>> t(n_tris);
        for (uint32_t i = 0; i < n_tris; ++i)
            for (int c = 0; c < 3; ++c) t[i][c] = mk(tris[i * 9 + c * 3], tris[i * 9 + c * 3 + 1], tris[i * 9 + c * 3 + 2]);
        Bvh b = build_tris(t, max_depth);
        if (b.nodes.size() > nodes_cap) { g_error = "node buffer too small"; return 0; }
        std::memcpy(nodes, b.nodes.data(), b.nodes.size() * 32);
        if (order) std::memcpy(order, b.order.data(), b.order.size() * 4);
        if (depth) *depth = (uint32_t)b.depth;
        return (uint32_t)b.nodes.size();
    } catch (const std::exception& e) {
        g_error = e.what();
        return 0;
    }
}

int trt_prep_unit_records(uint32_t n, const float* worlds, const uint32_t* info, const uint32_t* roots,
                          const uint32_t* cast_shadow, uint32_t* out) {
    if (n && (!worlds || !info || !roots || !cast_shadow || !out)) return 1;
    for (uint32_t i = 0; i < n; ++i) {
        Mat34 w;
        std::memcpy(w.m, worlds + 12ull * i, sizeof(w.m));
        GpuInstance g = instance_gpu(w, info[4ull * i], info[4ull * i + 1], info[4ull * i + 2], info[4ull * i + 3], 0u);
        unit_record(g, roots[i], cast_shadow[i] != 0);
        std::memcpy(out + 40ull * i, &g, sizeof(g));
    }
    return 0;
}

int trt_prep_units_top(uint32_t n, const float* worlds, const float* local_boxes, uint32_t* nodes, uint32_t* depth) {
    if (n == 0 || n > MAX_UNITS || !worlds || !local_boxes || !nodes) return 1;
    std::vector<Box> boxes(n);
    for (uint32_t i = 0; i < n; ++i) {
        Mat34 w;
        std::memcpy(w.m, worlds + 12ull * i, sizeof(w.m));
        const float* b = local_boxes + 6ull * i;
        boxes[i] = unit_box(w, mk(b[0], b[1], b[2]), mk(b[3], b[4], b[5]));
    }
    std::vector<GpuNode> top;
    std::vector<uint32_t> order;
    build_sah(boxes, TOP_DEPTH - 1, top, order);
    for (GpuNode& nd : top)
        if (nd.count > 0) nd.left_or_first = order[nd.left_or_first];
    long d = check_tree(top.data(), top.size(), TOP_DEPTH, 1, n);
    if (d < 0 || top.size() != 2ull * n - 1) return 1;
    if (depth) *depth = (uint32_t)d;
    std::memcpy(nodes, top.data(), top.size() * sizeof(GpuNode));
    return 0;
}

int trt_prep_check_tree(const uint32_t* nodes, uint32_t n_nodes, uint32_t max_depth, uint32_t max_leaf,
                        uint32_t n_items, uint32_t* depth) {
    long d = check_tree(reinterpret_cast<const GpuNode*>(nodes), n_nodes, max_depth, max_leaf, n_items);
    if (d < 0) return 1;
    if (depth) *depth = (uint32_t)d;
    return 0;
}

void trt_prep_specular_albedo(double mu, double alpha, uint32_t nr, uint32_t nphi, double out[2]) {
    specular_albedo(mu, alpha, nr, nphi, out);
}

}  // extern "C"
