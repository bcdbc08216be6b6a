// Test infrastructure, not product code: the CPU oracle of the path-trace pass (oracle.h says what it is for).
//
// Every function below restates the reference function it names, statement for statement, with the file:line it
// follows (paths inside the ThreeRT project). Arithmetic is IEEE f32 in source order: the build passes
// -ffp-contract=off, so no multiply-add is fused, and sqrt / division are correctly rounded. Transcendentals (cos, sin,
// acos, atan2, pow) are libm's; the reference leaves their precision to the GPU driver.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// ------------------------------------------------------------------------------------------------------------------
// Scalars and vectors (WGSL semantics as the kernel uses them)

constexpr float PI = 3.14159265358979f;        // pathtrace.wgsl:25
constexpr float INF = 3.0e38f;                  // pathtrace.wgsl:26
constexpr uint32_t MISS = 0xffffffffu;
constexpr uint32_t NO_INST = 0xffffffffu;       // pathtrace.wgsl:637
constexpr uint32_t TRACE_CLOSEST = 0, TRACE_SHADOW = 1, TRACE_ANY = 2;  // pathtrace.wgsl:28-30
constexpr uint32_t UNIT_SHADOW = 1, UNIT_SHIFTED = 2;                    // trace_units.wgsl:33-34
constexpr uint32_t INST_MIRRORED = 4;           // pathtrace.wgsl:279
constexpr uint32_t ROW_MATERIAL = 0xffffffu;    // pathtrace.wgsl:301
constexpr uint32_t NO_EMITTER = 0xffffffffu;    // pathtrace.wgsl:304
constexpr int32_t MAT_EMITTER_CARD = 2;         // pathtrace.wgsl:47
constexpr uint32_t EMITTER_GUIDE = 65536u;      // pathtrace.wgsl:457
constexpr uint32_t LT_LEAF = 0x80000000u;       // pathtrace.wgsl:494
constexpr uint32_t LT_PATH_BITS = 26u;          // pathtrace.wgsl:495
constexpr uint32_t EMITTER_MOVES = 0x80000000u; // pathtrace.wgsl:208
constexpr uint32_t EMITTER_CARD = 1u;           // pathtrace.wgsl:322
constexpr uint32_t EMIT_RIS_M = 6u;             // pathtrace.wgsl:42
constexpr float MIRROR_ROUGHNESS = 0.3f;        // pathtrace.wgsl:1245
constexpr uint32_t ENERGY_N = 32u;              // pathtrace.wgsl:1446
// sample.wgsl:114-124: a vertex's decisions.
constexpr uint32_t D_CAMERA = 0, D_BSDF = 1, D_RR = 2, D_SUN = 4, D_SUN_VIS = 5, D_EMIT = 7, D_EMIT_VIS = 8, D_ENV = 9,
                   D_ENV_VIS = 10;

inline float bf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t bu(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float fmax_(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

struct V3 { float x, y, z; };
inline V3 v3(float a) { return {a, a, a}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
// normalize(v): v over its length, a division per component.
inline V3 normalize(V3 a) { float l = std::sqrt(dot(a, a)); return {a.x / l, a.y / l, a.z / l}; }
inline V3 vmin(V3 a, V3 b) { return {fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)}; }
inline bool any_gt0(V3 a) { return a.x > 0.0f || a.y > 0.0f || a.z > 0.0f; }
inline bool all_le0(V3 a) { return a.x <= 0.0f && a.y <= 0.0f && a.z <= 0.0f; }
// mix(a, b, t) = a (1 - t) + b t (the WGSL builtin's definition).
inline V3 mix3(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
// reflect(e1, e2) = e1 - 2 dot(e2, e1) e2.
inline V3 reflect(V3 i, V3 n) { return i - (2.0f * dot(n, i)) * n; }
// pathtrace.wgsl:1981 luminance.
inline float luminance(V3 c) { return dot(c, V3{0.2126f, 0.7152f, 0.0722f}); }
// pathtrace.wgsl:1976 non_finite: by the bits.
inline bool non_finite3(V3 v) {
    return (bu(v.x) & 0x7fffffffu) >= 0x7f800000u || (bu(v.y) & 0x7fffffffu) >= 0x7f800000u ||
           (bu(v.z) & 0x7fffffffu) >= 0x7f800000u;
}
inline uint32_t reverse_bits(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
    x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
    return (x >> 16) | (x << 16);
}
// IEEE binary16 -> binary32 (unpack2x16float, the environment's RGBA16F texels).
inline float half_to_float(uint16_t h) {
    uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    if (e == 0) {
        if (m == 0) return bf(s);
        float f = (float)m * (1.0f / 16777216.0f);  // m * 2^-24
        return (s != 0) ? -f : f;
    }
    if (e == 31) return bf(s | 0x7f800000u | (m << 13));
    return bf(s | ((e + 112u) << 23) | (m << 13));
}

// ------------------------------------------------------------------------------------------------------------------
// Sampler: sample.wgsl (CPU mirror renderer/src/sample.rs:4-83)

// The direction numbers of Sobol dimensions 1-3 (Joe & Kuo), bit-reversed: sample.rs:4-31 computes them by the
// primitive-polynomial recurrence; sample.wgsl:5-64 unrolls their first 16.
struct SobolTable {
    uint32_t d[3][32];
    SobolTable() {
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
            for (int i = 0; i < 32; ++i) d[k][i] = reverse_bits(m[i] << (31 - i));
        }
    }
};
const SobolTable& sobol_table() { static SobolTable t; return t; }

// sample.wgsl:5-64 sobol_d1..d3: bit 31 - i of the (bit-reversed) index selects direction i.
inline uint32_t sobol_dim(uint32_t x, int dim) {
    const uint32_t* t = sobol_table().d[dim - 1];
    uint32_t r = 0;
    for (int i = 0; i < 16; ++i)
        if (x & (0x80000000u >> i)) r ^= t[i];
    return r;
}
// sample.wgsl:67-75
inline uint32_t owen_rev(uint32_t n, uint32_t seed) {
    n ^= n * 0x3d20adeau;
    n += seed;
    n *= (seed >> 16) | 1u;
    n ^= n * 0x05526c56u;
    n ^= n * 0x53a22864u;
    return n;
}
// sample.wgsl:77-85
inline uint32_t hash_hp(uint32_t i) {
    i ^= i >> 16;
    i *= 0x21f0aaadu;
    i ^= i >> 15;
    i *= 0xd35a2d97u;
    i ^= i >> 15;
    return i ^ 0xe6fe3bebu;
}
// sample.wgsl:88-101
inline float sobol_owen(uint32_t rev_index, uint32_t dim, uint32_t seed) {
    uint32_t r = dim == 0 ? reverse_bits(rev_index) : sobol_dim(rev_index, (int)dim);
    r = reverse_bits(owen_rev(r, seed));
    return (float)r * (1.0f / 4294967808.0f);
}

// The per-path sampler state (sample.wgsl:104-106 RNG_INDEX, RNG_SEED, RNG_PATH; pathtrace.wgsl:418 cur_depth).
struct Rng {
    uint32_t index = 0, seed = 0, path = 0, depth = 0;
    // sample.wgsl:110 rng_dim
    uint32_t dim(uint32_t slot) const { return (path << 28) ^ (depth << 20) ^ slot; }
    // sample.wgsl:144-145
    uint32_t seed_of(uint32_t d) const { return seed ^ hash_hp(d); }
    uint32_t index_of(uint32_t salt) const { return owen_rev(reverse_bits(index), salt) & 0xffff0000u; }
    // sample.wgsl:147-169 (offline: rng_white is false, Sobol everywhere).
    float rng1(uint32_t d) const {
        uint32_t s = seed_of(d);
        return sobol_owen(index_of(s ^ 0xbff95bfeu), 0, s ^ 0x635c77bdu);
    }
    void rng2(uint32_t d, float o[2]) const {
        uint32_t s = seed_of(d), i = index_of(s ^ 0xf8ade99au);
        o[0] = sobol_owen(i, 0, s ^ 0xe0aaaf76u);
        o[1] = sobol_owen(i, 1, s ^ 0x94964d4eu);
    }
    void rng3(uint32_t d, float o[3]) const {
        uint32_t s = seed_of(d), i = index_of(s ^ 0xcaa726acu);
        o[0] = sobol_owen(i, 0, s ^ 0x9e78e391u);
        o[1] = sobol_owen(i, 1, s ^ 0x67c33241u);
        o[2] = sobol_owen(i, 2, s ^ 0x78c395c5u);
    }
    void rng4(uint32_t d, float o[4]) const {
        uint32_t s = seed_of(d), i = index_of(s ^ 0xc2c1a055u);
        o[0] = sobol_owen(i, 0, s ^ 0x39468210u);
        o[1] = sobol_owen(i, 1, s ^ 0xe9d8a845u);
        o[2] = sobol_owen(i, 2, s ^ 0x5f32b482u);
        o[3] = sobol_owen(i, 3, s ^ 0x1524cc56u);
    }
    // sample.wgsl:173-177 rng_start
    void start(uint32_t px, uint32_t py, uint32_t idx, uint32_t sd, uint32_t p) {
        seed = hash_hp(px ^ hash_hp(py ^ hash_hp(sd)));
        index = idx;
        path = p;
    }
};
// sample.wgsl:111 rng_sub
inline uint32_t rng_sub(uint32_t d, uint32_t k) { return hash_hp(d ^ hash_hp(k + 0x9e3779b9u)) | 0x80000000u; }

// ------------------------------------------------------------------------------------------------------------------
// Records (pathtrace.wgsl:96-268; gpu.rs:127-186 Params; scene.rs:229-233, 480-501)

// Params, word offsets of its vec4s (gpu.rs:127-186, 39 vec4s).
enum : uint32_t {
    P_CAM_POS = 0, P_CAM_FWD = 4, P_CAM_RIGHT = 8, P_CAM_UP = 12, P_SIZE = 16, P_COUNTS = 20, P_ENV = 24, P_MISC = 28,
    P_SKY = 32, P_COUNTS2 = 36, P_MOTION = 68, P_LIGHT_LOD = 72, P_LTREE = 84, P_TABLE_FIRST = 124, P_WORD_FIRST = 136,
    P_WORDS = 156
};

struct Node { V3 bmin; uint32_t left_or_first; V3 bmax; uint32_t count; };
struct Instance { float m[3][4]; float n[3][4]; uint32_t info[4]; };
struct Hit { float t; uint32_t tri; float u, v; uint32_t inst, part; };

struct Scene {
    const orc_scene* s;
    const uint32_t* P;
    // Table section starts (heap.rs:36-62 Table's order in Params::table_first).
    uint32_t t_materials, t_lights, t_emitters, t_objects, t_instances, t_energy, t_emitter_tris;
    uint32_t w_rows, w_indices;

    float pf(uint32_t w) const { return bf(P[w]); }
    uint32_t pu(uint32_t w) const { return P[w]; }
    V3 pv(uint32_t w) const { return {pf(w), pf(w + 1), pf(w + 2)}; }

    const uint32_t* tvec(uint32_t i) const { return s->tables + 4ull * i; }
    float tf(uint32_t i, int c) const { return bf(s->tables[4ull * i + c]); }
    V3 tv(uint32_t i) const { return {tf(i, 0), tf(i, 1), tf(i, 2)}; }

    Node node(uint32_t i) const {
        const uint32_t* n = s->nodes + 8ull * i;
        return {{bf(n[0]), bf(n[1]), bf(n[2])}, n[3], {bf(n[4]), bf(n[5]), bf(n[6])}, n[7]};
    }
    // pathtrace.wgsl:262 instance_at (GpuInstance, 10 vec4s: scene.rs:229-233)
    Instance instance(uint32_t i) const {
        Instance r;
        const uint32_t* b = tvec(t_instances + i * 10u);
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 4; ++c) {
                r.m[k][c] = bf(b[k * 4 + c]);
                r.n[k][c] = bf(b[12 + k * 4 + c]);
            }
        for (int c = 0; c < 4; ++c) r.info[c] = b[24 + c];
        return r;
    }
    // pathtrace.wgsl:224 emitter_at
    void emitter(uint32_t i, float e[4]) const {
        for (int c = 0; c < 4; ++c) e[c] = tf(t_emitters + i, c);
    }
    float emitter_c(uint32_t i, int c) const { return tf(t_emitters + i, c); }
    // pathtrace.wgsl:207-214 emitter_tri_at (EmitterTri, 4 vec4s)
    struct ETri { V3 v0; uint32_t tri; V3 e1; uint32_t inst; V3 e2; uint32_t code; uint32_t part; uint32_t flags; };
    ETri etri(uint32_t i) const {
        const uint32_t* b = tvec(t_emitter_tris + i * 4u);
        return {{bf(b[0]), bf(b[1]), bf(b[2])}, b[3], {bf(b[4]), bf(b[5]), bf(b[6])}, b[7],
                {bf(b[8]), bf(b[9]), bf(b[10])}, b[11], b[12], b[13]};
    }
    // pathtrace.wgsl:305 row_word
    uint32_t row_word(uint32_t first, uint32_t section, uint32_t k) const {
        return s->words[w_rows + (first + section) * 4u + k];
    }
    float leaf_w(uint32_t ti, uint32_t k) const { return s->leaves[(ti * 3ull + k) * 4 + 3]; }
    // pathtrace.wgsl:187 leaf_id
    uint32_t leaf_id(uint32_t ti, uint32_t k) const { return bu(leaf_w(ti, k)); }
    V3 leaf_v(uint32_t ti, uint32_t k) const {
        const float* l = s->leaves + (ti * 3ull + k) * 4;
        return {l[0], l[1], l[2]};
    }

    explicit Scene(const orc_scene* sc, const uint32_t* params) : s(sc), P(params) {
        t_materials = P[P_TABLE_FIRST + 1];
        t_lights = P[P_TABLE_FIRST + 2];
        t_emitters = P[P_TABLE_FIRST + 4];
        t_objects = P[P_TABLE_FIRST + 6];
        t_instances = P[P_TABLE_FIRST + 7];
        t_energy = P[P_TABLE_FIRST + 9];
        t_emitter_tris = P[P_TABLE_FIRST + 11];
        w_rows = P[P_WORD_FIRST + 3];
        w_indices = P[P_WORD_FIRST + 4];
    }
};

// ------------------------------------------------------------------------------------------------------------------
// Traversal (pathtrace.wgsl:732-770, trace_units.wgsl:44-135)

struct Counters { uint64_t closest = 0, shadow = 0, nodes = 0, tris = 0, units = 0; };

// pathtrace.wgsl:732-739 ray_aabb
inline float ray_aabb(V3 o, V3 inv_d, V3 bmin, V3 bmax, float tmax) {
    V3 t0 = (bmin - o) * inv_d;
    V3 t1 = (bmax - o) * inv_d;
    V3 tmin_v = vmin(t0, t1);
    V3 tmax_v = vmax(t0, t1);
    float tn = fmax_(fmax_(tmin_v.x, tmin_v.y), fmax_(tmin_v.z, 0.0f));
    float tf = fmin_(fmin_(tmax_v.x, tmax_v.y), fmin_(tmax_v.z, tmax));
    return tn <= tf ? tn : INF;
}

// pathtrace.wgsl:742-761 intersect_tri: (t, u, v), t = INF for none.
inline void intersect_tri(const Scene& S, V3 o, V3 d, uint32_t i, float tmax, float out[3]) {
    V3 v0 = S.leaf_v(i, 0), e1 = S.leaf_v(i, 1), e2 = S.leaf_v(i, 2);
    out[0] = INF; out[1] = 0.0f; out[2] = 0.0f;
    V3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (std::fabs(det) < 1e-12f) return;
    float inv = 1.0f / det;
    V3 tv = o - v0;
    float u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return;
    V3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return;
    float t = dot(e2, qv) * inv;
    if (t <= 0.0f || t >= tmax) return;
    out[0] = t; out[1] = u; out[2] = v;
}

// pathtrace.wgsl:661 proc_dir: world -> a record's space by its normal rows.
inline V3 proc_dir(const Instance& r, V3 d) {
    return V3{r.n[0][0], r.n[0][1], r.n[0][2]} * d.x + V3{r.n[1][0], r.n[1][1], r.n[1][2]} * d.y +
           V3{r.n[2][0], r.n[2][1], r.n[2][2]} * d.z;
}
inline V3 safe_inv(V3 d) {
    // 1 / select(d, 1e-20, |d| < 1e-20), per component (pathtrace.wgsl:768, trace_units.wgsl:96)
    V3 s = {std::fabs(d.x) < 1e-20f ? 1e-20f : d.x, std::fabs(d.y) < 1e-20f ? 1e-20f : d.y,
            std::fabs(d.z) < 1e-20f ? 1e-20f : d.z};
    return V3{1.0f / s.x, 1.0f / s.y, 1.0f / s.z};
}

// trace_units.wgsl:44-135, the one loop over both levels with the module's 64-entry stack.
Hit trace_units(const Scene& S, V3 o, V3 d, V3 inv_d, Hit hit, uint32_t mode, Counters& C) {
    if (S.pu(P_MOTION + 3) == 0) return hit;
    uint32_t top = S.pu(P_MOTION + 2);
    Node whole = S.node(top);
    C.nodes++;
    if (ray_aabb(o, inv_d, whole.bmin, whole.bmax, hit.t) == INF) return hit;
    uint32_t stack[64];
    uint32_t sp = 0, node = top, rec = NO_INST;
    V3 ro = o, rd = d, rinv = inv_d;
    uint32_t off = top, first = 0, base = 0;
    for (;;) {
        Node n = S.node(node);
        C.nodes++;
        if (n.count == 0) {
            uint32_t l = off + n.left_or_first, r = l + 1;
            Node nl = S.node(l), nr = S.node(r);
            float tl = ray_aabb(ro, rinv, nl.bmin, nl.bmax, hit.t);
            float tr = ray_aabb(ro, rinv, nr.bmin, nr.bmax, hit.t);
            if (tl != INF || tr != INF) {
                uint32_t nearn = l, farn = r;
                if (tr < tl) { nearn = r; farn = l; std::swap(tl, tr); }
                node = nearn;
                if (tr != INF && sp < 64) stack[sp++] = farn;
                continue;
            }
        } else if (rec == NO_INST) {
            Instance u = S.instance(n.left_or_first);
            C.units++;
            uint32_t ubits = bu(u.n[1][3]);
            if (mode != TRACE_SHADOW || (ubits & UNIT_SHADOW) != 0) {
                rec = n.left_or_first;
                ro = o - V3{u.m[0][3], u.m[1][3], u.m[2][3]};
                if ((ubits & UNIT_SHIFTED) == 0) {
                    ro = proc_dir(u, ro);
                    rd = proc_dir(u, d);
                    rinv = safe_inv(rd);
                }
                off = bu(u.n[0][3]);
                first = u.info[0];
                base = sp;
                node = off;
                continue;
            }
        } else {
            for (uint32_t k = 0; k < n.count; ++k) {
                uint32_t ti = first + n.left_or_first + k;
                float x[3];
                C.tris++;
                intersect_tri(S, ro, rd, ti, hit.t, x);
                if (x[0] < hit.t) {
                    uint32_t part = S.leaf_id(ti, 0);
                    hit = Hit{x[0], ti, x[1], x[2], rec, part};
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

// pathtrace.wgsl:765-770 trace
Hit trace(const Scene& S, V3 o, V3 d, float tmax_in, uint32_t mode, Counters& C) {
    Hit hit{tmax_in, MISS, 0.0f, 0.0f, NO_INST, 0u};
    if (mode == TRACE_CLOSEST) C.closest++; else C.shadow++;
    return trace_units(S, o, d, safe_inv(d), hit, mode, C);
}

// Every unit's triangles without the trees (units.rs:1393-1423 `check`'s brute force): the top tree's leaves name
// the units; each unit's triangles are its mesh tree's leaves' ranges.
Hit trace_brute(const Scene& S, V3 o, V3 d, float tmax_in, uint32_t mode) {
    Hit hit{tmax_in, MISS, 0.0f, 0.0f, NO_INST, 0u};
    if (S.pu(P_MOTION + 3) == 0) return hit;
    uint32_t top = S.pu(P_MOTION + 2);
    // The top tree's leaves, in node order.
    std::vector<uint32_t> todo{top};
    std::vector<uint32_t> units;
    while (!todo.empty()) {
        uint32_t i = todo.back(); todo.pop_back();
        Node n = S.node(i);
        if (n.count == 0) { todo.push_back(top + n.left_or_first); todo.push_back(top + n.left_or_first + 1); }
        else units.push_back(n.left_or_first);
    }
    for (uint32_t rec : units) {
        Instance u = S.instance(rec);
        uint32_t ubits = bu(u.n[1][3]);
        if (mode == TRACE_SHADOW && (ubits & UNIT_SHADOW) == 0) continue;
        V3 ro = o - V3{u.m[0][3], u.m[1][3], u.m[2][3]}, rd = d;
        if ((ubits & UNIT_SHIFTED) == 0) { ro = proc_dir(u, ro); rd = proc_dir(u, d); }
        uint32_t root = bu(u.n[0][3]);
        std::vector<uint32_t> st{root};
        while (!st.empty()) {
            uint32_t i = st.back(); st.pop_back();
            Node n = S.node(i);
            if (n.count == 0) { st.push_back(root + n.left_or_first); st.push_back(root + n.left_or_first + 1); continue; }
            for (uint32_t k = 0; k < n.count; ++k) {
                uint32_t ti = u.info[0] + n.left_or_first + k;
                float x[3];
                intersect_tri(S, ro, rd, ti, hit.t, x);
                if (x[0] < hit.t) {
                    hit = Hit{x[0], ti, x[1], x[2], rec, S.leaf_id(ti, 0)};
                    if (mode != TRACE_CLOSEST) return hit;
                }
            }
        }
    }
    return hit;
}

// ------------------------------------------------------------------------------------------------------------------
// Shading

struct Attr { float n0[4], n1[4], n2[4], uv[4], x[4]; };  // records.wgsl:188 TriAttr
struct TriData { Attr a; V3 v0, e1, e2; };

// pathtrace.wgsl:314-317 tri_indices, 327-355 tri_data (F_INST; no particles, no deforming meshes).
TriData tri_data(const Scene& S, uint32_t ti, uint32_t inst, uint32_t part) {
    uint32_t base = 0;
    if (inst != NO_INST) base = S.instance(inst).info[2];
    const uint32_t* ix = S.s->words + S.w_indices + ti * 3u;
    uint32_t i0 = (ix[0] + base) * 3u, i1 = (ix[1] + base) * 3u, i2 = (ix[2] + base) * 3u;
    const float* p0 = S.s->vertices + 4ull * i0;
    const float* p1 = S.s->vertices + 4ull * i1;
    const float* p2 = S.s->vertices + 4ull * i2;
    const float* n0 = S.s->vertices + 4ull * (i0 + 1);
    const float* n1 = S.s->vertices + 4ull * (i1 + 1);
    const float* n2 = S.s->vertices + 4ull * (i2 + 1);
    TriData t;
    V3 P0{p0[0], p0[1], p0[2]}, P1{p1[0], p1[1], p1[2]}, P2{p2[0], p2[1], p2[2]};
    t.v0 = P0;
    t.e1 = P1 - P0;
    t.e2 = P2 - P0;
    float a_n0[4] = {n0[0], n0[1], n0[2], p0[3]};
    float a_n1[4] = {n1[0], n1[1], n1[2], n0[3]};
    float a_n2[4] = {n2[0], n2[1], n2[2], p1[3]};
    float a_uv[4] = {n1[3], p2[3], n2[3], bf(part)};
    float a_x[4] = {0.0f, bf(0u), 0.0f, 0.0f};
    std::memcpy(t.a.n0, a_n0, 16); std::memcpy(t.a.n1, a_n1, 16); std::memcpy(t.a.n2, a_n2, 16);
    std::memcpy(t.a.uv, a_uv, 16); std::memcpy(t.a.x, a_x, 16);
    return t;
}
// pathtrace.wgsl:276 inst_vec
inline V3 inst_vec(const Instance& r, V3 v) {
    return {dot(V3{r.m[0][0], r.m[0][1], r.m[0][2]}, v), dot(V3{r.m[1][0], r.m[1][1], r.m[1][2]}, v),
            dot(V3{r.m[2][0], r.m[2][1], r.m[2][2]}, v)};
}
// pathtrace.wgsl:280 inst_sign
inline float inst_sign(const Instance& r) { return (bu(r.n[1][3]) & INST_MIRRORED) != 0 ? -1.0f : 1.0f; }
// pathtrace.wgsl:281-283 inst_normal
inline void inst_normal(const Instance& r, float n[4]) {
    V3 v{n[0], n[1], n[2]};
    V3 o = normalize(V3{dot(V3{r.n[0][0], r.n[0][1], r.n[0][2]}, v), dot(V3{r.n[1][0], r.n[1][1], r.n[1][2]}, v),
                        dot(V3{r.n[2][0], r.n[2][1], r.n[2][2]}, v)});
    n[0] = o.x; n[1] = o.y; n[2] = o.z;
}
// pathtrace.wgsl:411-418 inst_attr (with inst_x, 286-288)
inline void inst_attr(const Instance& r, Attr& a) {
    inst_normal(r, a.n0);
    inst_normal(r, a.n1);
    inst_normal(r, a.n2);
    a.x[1] = bf(r.info[1] + bu(a.x[1]));
}
// pathtrace.wgsl:310-313 material_of
inline uint32_t material_of(const Scene& S, const Attr& a, uint32_t inst) {
    if (inst == NO_INST) return 0;
    return S.row_word(S.instance(inst).info[3], bu(a.uv[3]), 0) & ROW_MATERIAL;
}
// GpuMaterial (scene.rs:480-491), 18 vec4s: base_color 0, emissive 1, params 2, tex0 3, tex1 4, ...
struct Material { V3 base; float opacity; V3 emissive; float metallic, roughness, specular; int32_t flags; };
inline Material material_at(const Scene& S, uint32_t mi) {
    uint32_t b = S.t_materials + mi * 18u;
    Material m;
    m.base = S.tv(b); m.opacity = S.tf(b, 3);
    m.emissive = S.tv(b + 1);
    m.metallic = S.tf(b + 2, 0); m.roughness = S.tf(b + 2, 1); m.specular = S.tf(b + 2, 2);
    m.flags = (int32_t)S.tvec(b + 4)[2];
    return m;
}
// pathtrace.wgsl:1204 obj_power: objects[object * OBJECT_STRIDE].w, OBJECT_STRIDE 3 without F_TINT (1201).
inline float obj_power(const Scene& S, const Attr& a) { return S.tf(S.t_objects + bu(a.x[1]) * 3u, 3); }
// pathtrace.wgsl:1309-1314 emission (no texture)
inline V3 emission(const Material& m) { return m.emissive; }

struct Surface { V3 p, ng, n, base; float metallic, roughness, specular; V3 emissive; bool front, card; };

// pathtrace.wgsl:1317-1428 surface (triangles; FEAT = F_INST)
Surface surface(const Scene& S, V3 o, V3 d, const Hit& h) {
    TriData td = tri_data(S, h.tri, h.inst, h.part);
    V3 e1 = td.e1, e2 = td.e2;
    Attr a = td.a;
    float side = 1.0f;
    if (h.inst != NO_INST) {
        Instance r = S.instance(h.inst);
        e1 = inst_vec(r, e1);
        e2 = inst_vec(r, e2);
        inst_attr(r, a);
        side = inst_sign(r);
    }
    float w = 1.0f - h.u - h.v;
    V3 ng = normalize(cross(e1, e2)) * side;
    V3 n = normalize(V3{a.n0[0], a.n0[1], a.n0[2]} * w + V3{a.n1[0], a.n1[1], a.n1[2]} * h.u +
                     V3{a.n2[0], a.n2[1], a.n2[2]} * h.v);
    uint32_t mi = material_of(S, a, h.inst);
    Material m = material_at(S, mi);
    bool front = dot(ng, d) < 0.0f;
    if (!front) ng = -ng;
    if (dot(n, ng) < 0.0f) n = -n;
    Surface s;
    s.p = o + d * h.t;
    s.front = front;
    s.card = m.flags == MAT_EMITTER_CARD;
    s.emissive = emission(m) * obj_power(S, a);
    s.base = m.base;
    s.roughness = clampf(m.roughness, 0.02f, 1.0f);
    s.metallic = clampf(m.metallic, 0.0f, 1.0f);
    s.specular = m.specular;
    s.ng = ng;
    s.n = n;
    return s;
}

// pathtrace.wgsl:1447-1461 energy_node, energy_lookup
inline void energy_node(const Scene& S, uint32_t i, float o[2]) {
    uint32_t v = S.t_energy + (i >> 1);
    if ((i & 1u) == 1u) { o[0] = S.tf(v, 2); o[1] = S.tf(v, 3); } else { o[0] = S.tf(v, 0); o[1] = S.tf(v, 1); }
}
inline void energy_lookup(const Scene& S, float roughness, float nov, float out[2]) {
    float x = std::sqrt(clampf(nov, 0.0f, 1.0f)) * (float)(ENERGY_N - 1u);
    float y = clampf(roughness, 0.0f, 1.0f) * (float)(ENERGY_N - 1u);
    uint32_t x0 = std::min((uint32_t)x, ENERGY_N - 2u);
    uint32_t y0 = std::min((uint32_t)y, ENERGY_N - 2u);
    uint32_t i = y0 * ENERGY_N + x0;
    float fx = x - (float)x0, fy = y - (float)y0;
    float a[2], b[2], c[2], d[2];
    energy_node(S, i, a); energy_node(S, i + 1, b); energy_node(S, i + ENERGY_N, c); energy_node(S, i + ENERGY_N + 1, d);
    for (int k = 0; k < 2; ++k) out[k] = mixf(mixf(a[k], b[k], fx), mixf(c[k], d[k], fx), fy);
}

struct Lobes { V3 diffuse, f0, f90, w, e_spec, kd; float a2, p_spec, p_coat, p_trans; };

// pathtrace.wgsl:1478-1482 spec_terms + 1642-1700 lobes (no glass, no coat)
Lobes lobes(const Scene& S, const Surface& s, float nov) {
    Lobes l;
    float t = 0.0f * (1.0f - s.metallic);  // s.transmission is 0 without F_GLASS
    l.diffuse = s.base * (1.0f - s.metallic) * (1.0f - t);
    float f0 = 0.08f * s.specular;
    l.f0 = mix3(v3(f0), s.base, s.metallic);
    float e[2];
    energy_lookup(S, s.roughness, nov, e);
    float comp = S.pf(P_MISC + 2);
    float f90 = clampf(dot(l.f0, v3(50.0f / 3.0f)), 0.0f, 1.0f);
    V3 w = v3(1.0f) + l.f0 * (comp * (1.0f / fmax_(e[0] + e[1], 1e-3f) - 1.0f));
    l.f90 = v3(f90);
    l.w = w;
    l.e_spec = (l.f0 * e[0] + v3(f90 * e[1])) * w;
    l.kd = v3(1.0f) - l.e_spec;
    float r = s.roughness;
    l.a2 = r * r * r * r;
    float ws = dot(l.e_spec, V3{0.3f, 0.6f, 0.1f});
    float wd = dot(l.diffuse * l.kd, V3{0.3f, 0.6f, 0.1f});
    l.p_spec = clampf(ws / fmax_(ws + wd, 1e-6f), 0.05f, 1.0f);
    if (wd <= 0.0f) l.p_spec = 1.0f;
    float e_coat = 0.0f, under = 1.0f - e_coat, wt = 0.0f;
    float total = (ws + wd) * under + e_coat + wt;
    l.p_coat = e_coat / fmax_(total, 1e-6f);
    l.p_trans = wt / fmax_(total, 1e-6f);
    return l;
}

// pathtrace.wgsl:1714-1717 d_ggx
inline float d_ggx(float a2, float noh) {
    float d = (noh * a2 - noh) * noh + 1.0f;
    return a2 / (PI * d * d);
}
// pathtrace.wgsl:1720-1722
inline float vis_smith_joint_approx(float a2, float nov, float nol) {
    return 0.5f / fmax_(mixf(2.0f * nol * nov, nol + nov, std::sqrt(a2)), 1e-7f);
}
// pathtrace.wgsl:1726-1730
inline V3 f_schlick(V3 f0, V3 f90, float voh) {
    float c = 1.0f - voh;
    float c2 = c * c;
    return f0 + (f90 - f0) * (c2 * c2 * c);
}
// pathtrace.wgsl:1733-1760 eval_bsdf_k (no two-sided glass, no coat)
V3 eval_bsdf_k(const Surface& s, const Lobes& lb, V3 v, V3 l, float k) {
    float nol = dot(s.n, l);
    float nov = fmax_(dot(s.n, v), 1e-4f);
    if (nol <= 0.0f || dot(s.ng, l) <= 0.0f) return v3(0.0f);
    V3 h = normalize(v + l);
    float noh = fmax_(dot(s.n, h), 0.0f);
    float voh = fmax_(dot(v, h), 0.0f);
    float dv = d_ggx(lb.a2, noh) * vis_smith_joint_approx(lb.a2, nov, nol);
    V3 spec = dv * f_schlick(lb.f0, lb.f90, voh) * lb.w * k;
    V3 diff = lb.diffuse * (1.0f / PI) * lb.kd;
    return (diff + spec) * nol;
}
inline V3 eval_bsdf(const Surface& s, const Lobes& lb, V3 v, V3 l) { return eval_bsdf_k(s, lb, v, l, 1.0f); }
// pathtrace.wgsl:1768-1770 g1
inline float g1(float a2, float nov) { return 2.0f * nov / (nov + std::sqrt(a2 + (1.0f - a2) * nov * nov)); }
// pathtrace.wgsl:1772-1792 pdf_bsdf
float pdf_bsdf(const Surface& s, const Lobes& lb, V3 v, V3 l) {
    float nol = dot(s.n, l);
    float pg = 0.0f;
    if (nol <= 0.0f) return pg;
    float nov = fmax_(dot(s.n, v), 1e-4f);
    V3 h = normalize(v + l);
    float noh = fmax_(dot(s.n, h), 0.0f);
    float voh = fmax_(dot(v, h), 1e-6f);
    float dv = g1(lb.a2, nov) * voh * d_ggx(lb.a2, noh) / nov;
    float ps = dv / (4.0f * voh);
    float pd = nol / PI;
    float pc = 0.0f;
    return pg + lb.p_coat * pc + (1.0f - lb.p_coat - lb.p_trans) * (lb.p_spec * ps + (1.0f - lb.p_spec) * pd);
}
// pathtrace.wgsl:1967-1970 power_heuristic
inline float power_heuristic(float a, float b) {
    float a2 = a * a;
    return a2 / fmax_(a2 + b * b, 1e-20f);
}
// pathtrace.wgsl:1800-1803 light_mis (A_CUTOUT_PATHS off: the plain heuristic)
inline float light_mis(float pdf_l, const Surface& s, const Lobes& lb, V3 v, V3 l) {
    return power_heuristic(pdf_l, pdf_bsdf(s, lb, v, l));
}
// pathtrace.wgsl:1824-1831 basis: the columns t, bt, n.
struct Mat3 { V3 c0, c1, c2; };
inline Mat3 basis(V3 n) {
    float sgn = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sgn + n.z);
    float b = n.x * n.y * a;
    V3 t{1.0f + sgn * n.x * n.x * a, sgn * b, -sgn * n.x};
    V3 bt{b, sgn + n.y * n.y * a, -n.y};
    return {t, bt, n};
}
inline V3 mul(const Mat3& m, V3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
inline V3 mul_t(const Mat3& m, V3 v) { return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }
// pathtrace.wgsl:1834-1852 sample_vndf (Heitz 2018)
V3 sample_vndf(V3 v, const Mat3& tbn, float alpha, float u1, float u2) {
    V3 vl = mul_t(tbn, v);
    V3 vh = normalize(V3{alpha * vl.x, alpha * vl.y, vl.z});
    float lensq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lensq > 0.0f ? V3{-vh.y, vh.x, 0.0f} / std::sqrt(lensq) : V3{1.0f, 0.0f, 0.0f};
    V3 t2 = cross(vh, t1);
    float r = std::sqrt(u1);
    float phi = 2.0f * PI * u2;
    float p1 = r * std::cos(phi);
    float p2 = r * std::sin(phi);
    float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * std::sqrt(1.0f - p1 * p1) + s * p2;
    V3 nh = p1 * t1 + p2 * t2 + std::sqrt(fmax_(0.0f, 1.0f - p1 * p1 - p2 * p2)) * vh;
    V3 hl = normalize(V3{alpha * nh.x, alpha * nh.y, fmax_(0.0f, nh.z)});
    return mul(tbn, hl);
}

// ------------------------------------------------------------------------------------------------------------------
// Environment (pathtrace.wgsl:1889-1965)

// pathtrace.wgsl:1892-1896 env_uv
inline void env_uv(V3 d, float& u, float& v) {
    u = std::atan2(d.x, -d.z) / (2.0f * PI) + 0.5f;
    v = std::acos(clampf(d.y, -1.0f, 1.0f)) / PI;
}
inline float env_cdf_at(const Scene& S, uint32_t i) { return bf(S.s->words[i]); }

// textureSampleLevel(env_tex, samp, uv, 0) with the reference's sampler (gpu.rs:2690-2696: linear, repeat in u and
// v), filtered in f32 from the f16 texels: texel centres at (i + 0.5) / size.
V3 env_texel(const Scene& S, uint32_t x, uint32_t y) {
    const uint16_t* t = S.s->env_half + 4ull * (y * S.s->env_w + x);
    return {half_to_float(t[0]), half_to_float(t[1]), half_to_float(t[2])};
}
V3 env_bilinear(const Scene& S, float u, float v) {
    int w = (int)S.s->env_w, h = (int)S.s->env_h;
    float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
    float fx0 = std::floor(x), fy0 = std::floor(y);
    float fx = x - fx0, fy = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0;
    auto wrap = [](int i, int n) { int r = i % n; return r < 0 ? r + n : r; };
    int xa = wrap(x0, w), xb = wrap(x0 + 1, w), ya = wrap(y0, h), yb = wrap(y0 + 1, h);
    V3 a = env_texel(S, xa, ya), b = env_texel(S, xb, ya), c = env_texel(S, xa, yb), d = env_texel(S, xb, yb);
    return mix3(mix3(a, b, fx), mix3(c, d, fx), fy);
}
// pathtrace.wgsl:1898-1901 env_radiance
V3 env_radiance(const Scene& S, V3 d) {
    if (S.pf(P_ENV) < 0.5f) return S.pv(P_SKY);
    float u, v;
    env_uv(d, u, v);
    return env_bilinear(S, u, v);
}
// pathtrace.wgsl:1903-1916 env_pdf
float env_pdf(const Scene& S, V3 d) {
    if (S.pf(P_ENV) < 0.5f) return 1.0f / (4.0f * PI);
    uint32_t w = (uint32_t)S.pf(P_ENV + 1), h = (uint32_t)S.pf(P_ENV + 2);
    float u, v;
    env_uv(d, u, v);
    uint32_t x = std::min((uint32_t)(u * (float)w), w - 1u);
    uint32_t y = std::min((uint32_t)(v * (float)h), h - 1u);
    float row_p = env_cdf_at(S, y) - (y > 0u ? env_cdf_at(S, y - 1u) : 0.0f);
    uint32_t base = h + y * w;
    float col_p = env_cdf_at(S, base + x) - (x > 0u ? env_cdf_at(S, base + x - 1u) : 0.0f);
    float sin_t = std::sin(((float)y + 0.5f) / (float)h * PI);
    return row_p * col_p * (float)w * (float)h / (2.0f * PI * PI * fmax_(sin_t, 1e-4f));
}
// pathtrace.wgsl:1918-1926 lower_bound
uint32_t lower_bound(const Scene& S, uint32_t start, uint32_t count, float x) {
    uint32_t lo = 0, hi = count;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (env_cdf_at(S, start + mid) < x) lo = mid + 1u; else hi = mid;
    }
    return std::min(lo, count - 1u);
}
// pathtrace.wgsl:1928-1944 sample_env
V3 sample_env(const Scene& S, const Rng& R, uint32_t rd) {
    float u4[4];
    R.rng4(rd, u4);
    if (S.pf(P_ENV) < 0.5f) {
        float z = 1.0f - 2.0f * u4[0];
        float r = std::sqrt(fmax_(0.0f, 1.0f - z * z));
        float phi = 2.0f * PI * u4[1];
        return {r * std::cos(phi), z, r * std::sin(phi)};
    }
    uint32_t w = (uint32_t)S.pf(P_ENV + 1), h = (uint32_t)S.pf(P_ENV + 2);
    uint32_t y = lower_bound(S, 0u, h, u4[0]);
    uint32_t x = lower_bound(S, h + y * w, w, u4[1]);
    float u = ((float)x + u4[2]) / (float)w;
    float v = ((float)y + u4[3]) / (float)h;
    float theta = v * PI;
    float phi = (u - 0.5f) * 2.0f * PI;
    return {std::sin(theta) * std::sin(phi), std::cos(theta), -std::sin(theta) * std::cos(phi)};
}
// pathtrace.wgsl:1985-1987 offset_origin
inline V3 offset_origin(V3 p, V3 n) {
    return p + n * (1e-4f * fmax_(1.0f, fmax_(std::fabs(p.x), fmax_(std::fabs(p.y), std::fabs(p.z)))));
}
// pathtrace.wgsl:2010-2020 sun_disks
V3 sun_disks(const Scene& S, V3 d, float pdf) {
    V3 c = v3(0.0f);
    for (uint32_t i = 0; i < S.pu(P_COUNTS2); ++i) {
        uint32_t b = S.t_lights + i * 5u;
        V3 dir = S.tv(b + 1);
        float cosw = S.tf(b + 1, 3);
        if (dot(d, -dir) >= cosw) {
            float omega = 2.0f * PI * (1.0f - cosw);
            c = c + (S.tv(b + 2) / omega) * power_heuristic(pdf, 1.0f / omega);
        }
    }
    return c;
}
// pathtrace.wgsl:1991-2006 sky_mis (no background, no aerial perspective)
V3 sky_mis(const Scene& S, V3 d, float pdf) {
    float wgt = 1.0f;
    if (pdf > 0.0f && S.pu(P_COUNTS2 + 1) != 0u) wgt = power_heuristic(pdf, env_pdf(S, d));
    V3 c = env_radiance(S, d) * wgt;
    if (pdf > 0.0f) c = c + sun_disks(S, d, pdf);
    return c;
}

// ------------------------------------------------------------------------------------------------------------------
// Emitters (pathtrace.wgsl:457-626)

// pathtrace.wgsl:459-461 emitter_guide
inline uint32_t emitter_guide(const Scene& S, uint32_t k) {
    return bu(S.emitter_c(S.pu(P_COUNTS + 1) + k / 4u, (int)(k % 4u)));
}
// pathtrace.wgsl:465 emitter_totals
inline void emitter_totals(const Scene& S, float t[4]) { S.emitter(S.pu(P_COUNTS + 1) + EMITTER_GUIDE / 4u + 1u, t); }
// pathtrace.wgsl:468-471 emitters_on
inline bool emitters_on(const Scene& S) {
    if (S.pu(P_COUNTS + 1) == 0u) return false;
    float t[4];
    emitter_totals(S, t);
    return t[0] > 0.0f;
}
// pathtrace.wgsl:476-485 emitter_pick_u
void emitter_pick_u(const Scene& S, float u, float e[4]) {
    uint32_t k = std::min((uint32_t)(u * (float)EMITTER_GUIDE), EMITTER_GUIDE - 1u);
    uint32_t lo = emitter_guide(S, k), hi = emitter_guide(S, k + 1u);
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (S.emitter_c(mid, 1) < u) lo = mid + 1u; else hi = mid;
    }
    S.emitter(std::min(lo, S.pu(P_COUNTS + 1) - 1u), e);
}
// pathtrace.wgsl:505-525 lt_imp (A_FAR_EMITTERS off)
inline void unpack2x16(uint32_t w, float& a, float& b) {
    a = half_to_float((uint16_t)(w & 0xffffu));
    b = half_to_float((uint16_t)(w >> 16));
}
float lt_imp(const float nd[4], V3 x, V3 n) {
    float cx, cy, cz, cr;
    unpack2x16(bu(nd[0]), cx, cy);
    unpack2x16(bu(nd[1]), cz, cr);
    V3 dv = V3{cx, cy, cz} - x;
    float d2 = dot(dv, dv);
    float r2 = cr * cr;
    float cb = 1.0f;
    if (d2 > r2 && dot(n, n) > 0.0f) {
        float inv = 1.0f / std::sqrt(d2);
        float cos_t = dot(n, dv) * inv;
        float sin_b = cr * inv;
        float cos_b = std::sqrt(fmax_(1.0f - sin_b * sin_b, 0.0f));
        if (cos_t < cos_b) cb = fmax_(cos_t * cos_b + std::sqrt(fmax_(1.0f - cos_t * cos_t, 0.0f)) * sin_b, 0.0f);
    }
    return nd[2] * cb / fmax_(d2, r2);
}
inline void lt_node(const Scene& S, uint32_t i, float o[4]) {
    for (int c = 0; c < 4; ++c) o[c] = S.tf(i, c);  // the light tree is the tables' first section
}
// pathtrace.wgsl:528-541 emitter_pick_range
void emitter_pick_range(const Scene& S, uint32_t lo, uint32_t hi, float r, float e[4]) {
    float p0 = lo > 0u ? S.emitter_c(std::max(lo, 1u) - 1u, 1) : 0.0f;
    float p1 = S.emitter_c(hi - 1u, 1);
    float u = fmin_(p0 + r * (p1 - p0), p1);
    uint32_t k = std::min((uint32_t)(u * (float)EMITTER_GUIDE), EMITTER_GUIDE - 1u);
    uint32_t l = emitter_guide(S, k), h = emitter_guide(S, k + 1u);
    while (l < h) {
        uint32_t mid = (l + h) / 2u;
        if (S.emitter_c(mid, 1) < u) l = mid + 1u; else h = mid;
    }
    S.emitter(std::min(std::max(l, lo), hi - 1u), e);
}
struct EPick { float e[4]; float p, w; };
// pathtrace.wgsl:547-585 emitter_draw
EPick emitter_draw(const Scene& S, const Rng& R, V3 x, V3 n, uint32_t rd) {
    EPick out{{0, 0, 0, 0}, 0.0f, 0.0f};
    float r3[3];
    R.rng3(rd, r3);
    float tot[4];
    emitter_totals(S, tot);
    if (!(tot[0] > 0.0f)) return out;
    if (!(S.pf(P_LTREE + 3) > 0.5f)) {
        emitter_pick_u(S, r3[0], out.e);
        out.p = out.e[2] / tot[0];
        out.w = out.e[2];
        return out;
    }
    if (r3[0] < tot[1]) {
        emitter_pick_range(S, S.pu(P_LTREE + 1), S.pu(P_COUNTS + 1), r3[1], out.e);
        out.p = out.e[2] / tot[0];
        out.w = out.e[2];
        return out;
    }
    float p = 1.0f - tot[1];
    float u = r3[1];
    float root[4];
    lt_node(S, 0u, root);
    uint32_t w = bu(root[3]);
    for (uint32_t k = 0; k <= LT_PATH_BITS && (w & LT_LEAF) == 0u; ++k) {
        float l[4], r[4];
        lt_node(S, w, l);
        lt_node(S, w + 1u, r);
        float il = lt_imp(l, x, n), ir = lt_imp(r, x, n);
        if (!(il + ir > 0.0f)) return out;
        float pl = il / (il + ir);
        if (u < pl) { w = bu(l[3]); p *= pl; u = u / pl; }
        else { w = bu(r[3]); p *= 1.0f - pl; u = (u - pl) / (1.0f - pl); }
        u = clampf(u, 0.0f, 0.99999994f);
    }
    if ((w & LT_LEAF) == 0u) return out;
    uint32_t lo = w & 0x1fffffffu, hi = lo + ((w >> 29) & 3u) + 1u;
    float wsum = 0.0f;
    for (uint32_t j = lo; j < hi; ++j) wsum += S.emitter_c(j, 2);
    float t = r3[2] * wsum;
    S.emitter(hi - 1u, out.e);
    for (uint32_t j = lo; j < hi; ++j) {
        float c[4];
        S.emitter(j, c);
        if (t < c[2]) { std::memcpy(out.e, c, 16); break; }
        t -= c[2];
    }
    out.p = p * out.e[2] / wsum;
    out.w = out.e[2];
    return out;
}
// pathtrace.wgsl:590-626 emitter_pmf
float emitter_pmf(const Scene& S, uint32_t ei, const Scene::ETri& em, V3 x, V3 n) {
    float tot[4];
    emitter_totals(S, tot);
    if (!(tot[0] > 0.0f)) return 0.0f;
    uint32_t code = em.code & ~EMITTER_MOVES;
    if ((code >> LT_PATH_BITS) == 0u) return S.emitter_c(code, 2) / tot[0];
    uint32_t depth = (code >> LT_PATH_BITS) - 1u;
    float p = 1.0f - tot[1];
    float root[4];
    lt_node(S, 0u, root);
    uint32_t w = bu(root[3]);
    for (uint32_t k = 0; k < depth; ++k) {
        float l[4], r[4];
        lt_node(S, w, l);
        lt_node(S, w + 1u, r);
        float il = lt_imp(l, x, n), ir = lt_imp(r, x, n);
        if (!(il + ir > 0.0f)) return 0.0f;
        uint32_t right = (code >> k) & 1u;
        p *= (right == 1u ? ir : il) / (il + ir);
        w = bu(right == 1u ? r[3] : l[3]);
    }
    uint32_t lo = w & 0x1fffffffu, hi = lo + ((w >> 29) & 3u) + 1u;
    float wsum = 0.0f, we = 0.0f;
    for (uint32_t j = lo; j < hi; ++j) {
        float c[4];
        S.emitter(j, c);
        wsum += c[2];
        if (bu(c[0]) == ei) we = c[2];
    }
    return p * we / wsum;
}
// pathtrace.wgsl:2023-2028 emitter_attrs, 2269-2280 emitter_radiance (no texture, no material function)
V3 emitter_radiance(const Scene& S, const Scene::ETri& em) {
    Attr a = tri_data(S, em.tri, em.inst, em.part).a;
    if (em.inst != NO_INST) a.x[1] = bf(S.instance(em.inst).info[1] + bu(a.x[1]));
    Material m = material_at(S, material_of(S, a, em.inst));
    float pw = obj_power(S, a);
    return emission(m) * pw;
}
// pathtrace.wgsl:2050-2065 emit_mis (software traversal: hit_rank is the leaf's id, 2040)
float emit_mis(const Scene& S, const Hit& hit, V3 d, float pdf, V3 mis_x, V3 mis_n) {
    if (!emitters_on(S)) return 1.0f;
    uint32_t rows = S.instance(hit.inst).info[3];
    uint32_t first = S.row_word(rows, hit.part, 2u);
    if (first == NO_EMITTER) return 1.0f;
    uint32_t entry = first + S.leaf_id(hit.tri, 1u);
    Scene::ETri em = S.etri(entry);
    V3 cr = cross(em.e1, em.e2);
    float area = 0.5f * length(cr);
    float cos_l = std::fabs(dot(normalize(cr), d));
    float sel = emitter_pmf(S, entry, em, mis_x, mis_n);
    if (!(sel > 0.0f)) return 1.0f;
    return power_heuristic(pdf, sel / fmax_(area, 1e-12f) * hit.t * hit.t / fmax_(cos_l, 1e-6f));
}

struct ES { V3 le, l; float dist, pdf_w, w; };
// pathtrace.wgsl:2283-2340 sample_emitter_ris (no light LOD)
ES sample_emitter_ris(const Scene& S, const Rng& R, V3 x, V3 n, uint32_t m, const Surface& sf, const Lobes& lb, V3 v,
                      uint32_t rd) {
    ES r{v3(0.0f), V3{0.0f, 1.0f, 0.0f}, 0.0f, 0.0f, 0.0f};
    float wsum = 0.0f, pick_b[2] = {0.0f, 0.0f}, pick_ph = 0.0f, pick_pdf = 0.0f;
    uint32_t pick_i = 0;
    for (uint32_t k = 0; k < m; ++k) {
        uint32_t dk = rng_sub(rd, k);
        EPick pk = emitter_draw(S, R, x, n, dk);
        float bb[3];
        R.rng3(rng_sub(dk, 1u), bb);
        float b1 = bb[0], b2 = bb[1];
        if (pk.p <= 0.0f) continue;
        if (b1 + b2 > 1.0f) { b1 = 1.0f - b1; b2 = 1.0f - b2; }
        Scene::ETri em = S.etri(bu(pk.e[0]));
        V3 lp = em.v0 + em.e1 * b1 + em.e2 * b2;
        V3 cr = cross(em.e1, em.e2);
        float a2 = length(cr);
        if (!(a2 > 0.0f)) continue;
        V3 ln = cr / a2;
        V3 dl = lp - x;
        float d2 = fmax_(dot(dl, dl), 1e-8f);
        V3 l = dl * (1.0f / std::sqrt(d2));
        float g = std::fabs(dot(ln, l)) * (dot(n, n) == 0.0f ? 1.0f : fmax_(dot(n, l), 0.0f)) / d2;
        if (m > 1u) g = std::fabs(dot(ln, l)) * luminance(eval_bsdf(sf, lb, v, l)) / d2;
        float ph = pk.w / (pk.e[3] * 1.0f) * g;  // emitter_lod: 1 without light LOD (2087-2092)
        float pdf_a = pk.p / (0.5f * a2);
        float w = ph / pdf_a;
        if (!(w > 0.0f)) continue;
        wsum += w;
        if (bb[2] * wsum < w) {
            pick_b[0] = b1; pick_b[1] = b2;
            pick_ph = ph;
            pick_i = bu(pk.e[0]);
            pick_pdf = pdf_a;
        }
    }
    if (pick_ph <= 0.0f) return r;
    Scene::ETri em = S.etri(pick_i);
    V3 lp = em.v0 + em.e1 * pick_b[0] + em.e2 * pick_b[1];
    V3 ln = normalize(cross(em.e1, em.e2));
    V3 dl = lp - x;
    float d2 = dot(dl, dl);
    float dist = std::sqrt(d2);
    V3 l = dl / dist;
    float cos_l = dot(ln, -l);
    if ((em.flags & EMITTER_CARD) == 0u) cos_l = std::fabs(cos_l);
    if (cos_l <= 0.0f) return r;
    r.le = emitter_radiance(S, em);
    r.l = l;
    r.dist = dist;
    r.pdf_w = pick_pdf * d2 / cos_l;
    r.w = (wsum / (float)m) / pick_ph * cos_l / d2;
    return r;
}
// pathtrace.wgsl:2344-2374 sample_emitter
ES sample_emitter(const Scene& S, const Rng& R, V3 x, V3 n, uint32_t rd) {
    ES r{v3(0.0f), V3{0.0f, 1.0f, 0.0f}, 0.0f, 0.0f, 0.0f};
    EPick pk = emitter_draw(S, R, x, n, rd);
    if (pk.p <= 0.0f) return r;
    Scene::ETri em = S.etri(bu(pk.e[0]));
    float bb[2];
    R.rng2(rng_sub(rd, 1u), bb);
    float b1 = bb[0], b2 = bb[1];
    if (b1 + b2 > 1.0f) { b1 = 1.0f - b1; b2 = 1.0f - b2; }
    V3 lp = em.v0 + em.e1 * b1 + em.e2 * b2;
    V3 cr = cross(em.e1, em.e2);
    float area = 0.5f * length(cr);
    V3 ln = cr / (2.0f * area);
    V3 dl = lp - x;
    float d2 = dot(dl, dl);
    float dist = std::sqrt(d2);
    V3 l = dl / dist;
    float cos_l = dot(ln, -l);
    if ((em.flags & EMITTER_CARD) == 0u) cos_l = std::fabs(cos_l);
    if (cos_l <= 0.0f) return r;
    r.le = emitter_radiance(S, em);
    r.l = l;
    r.dist = dist;
    r.pdf_w = pk.p / area * d2 / cos_l;
    r.w = 1.0f / r.pdf_w;
    return r;
}

// ------------------------------------------------------------------------------------------------------------------
// Direct light (pathtrace.wgsl:2420-2546)

struct PathState {
    V3 mis_x{0, 0, 0}, mis_n{0, 0, 0};
    bool mirror_path = false;
};

// pathtrace.wgsl:2411-2412 env_sampled
inline bool env_sampled(const Scene& S) {
    return S.pu(P_COUNTS2 + 1) != 0u && (S.pf(P_ENV) > 0.5f || luminance(S.pv(P_SKY)) > 0.0f);
}
// pathtrace.wgsl:2415-2428 env_light
V3 env_light(const Scene& S, const Rng& R, const Surface& s, const Lobes& lb, V3 v, V3 o, Counters& C) {
    V3 l = sample_env(S, R, R.dim(D_ENV));
    V3 f = eval_bsdf(s, lb, v, l);
    if (any_gt0(f)) {
        float pdf_e = env_pdf(S, l);
        if (pdf_e > 0.0f) {
            // sky_tr -> shadow_tr(o, l, INF, true): a shadow caster stops it (no glass, no media)
            bool vis = trace(S, o, l, INF, TRACE_SHADOW, C).tri == MISS;
            if (vis) return env_radiance(S, l) * f * light_mis(pdf_e, s, lb, v, l) / pdf_e * 1.0f;
        }
    }
    return v3(0.0f);
}
// pathtrace.wgsl:2444-2546 direct_light (light_pick off; no local lights in a scene without them)
V3 direct_light(const Scene& S, const Rng& R, const Surface& s, const Lobes& lb, V3 v, PathState& st, Counters& C) {
    V3 sum = v3(0.0f);
    V3 o = offset_origin(s.p, s.ng);
    for (uint32_t i = 0; i < S.pu(P_COUNTS2); ++i) {
        uint32_t b = S.t_lights + i * 5u;
        float cos_max = S.tf(b + 1, 3);
        V3 to_light = -S.tv(b + 1);
        float u[2];
        R.rng2(rng_sub(R.dim(D_SUN), i), u);
        float cos_t = 1.0f - u[0] * (1.0f - cos_max);
        float sin_t = std::sqrt(fmax_(0.0f, 1.0f - cos_t * cos_t));
        float phi = 2.0f * PI * u[1];
        Mat3 tb = basis(to_light);
        V3 l = mul(tb, V3{sin_t * std::cos(phi), sin_t * std::sin(phi), cos_t});
        V3 color = S.tv(b + 2);
        if (all_le0(color)) continue;
        V3 f = eval_bsdf_k(s, lb, v, l, S.tf(b + 4, 1));
        if (any_gt0(f)) {
            bool shadows = S.tf(b + 3, 3) >= 0.5f;
            // light_vis -> shadow_tr(o, l, INF, false)
            bool vis = !shadows || trace(S, o, l, INF, TRACE_SHADOW, C).tri == MISS;
            if (vis) {
                float pdf_l = 1.0f / (2.0f * PI * (1.0f - cos_max));
                float wgt = light_mis(pdf_l, s, lb, v, l);
                sum = sum + color * f * wgt * 1.0f;
            }
        }
    }
    // (local lights: counts.x - counts2.x of them; the configs have none.)
    V3 ne = s.n;
    st.mis_x = o;
    st.mis_n = ne;
    uint32_t emitters = emitters_on(S) ? S.pu(P_COUNTS + 1) : 0u;
    if (emitters > 0u) {
        ES es;
        bool lt_on = S.pf(P_LTREE + 3) > 0.5f;
        bool seen_directly = R.depth == 0u || (R.depth == 1u && st.mirror_path);
        if (lt_on) es = sample_emitter_ris(S, R, o, ne, R.depth == 0u ? (uint32_t)S.pf(P_LTREE + 3) : 1u, s, lb, v, R.dim(D_EMIT));
        else if (seen_directly) es = sample_emitter_ris(S, R, o, ne, R.depth == 0u ? EMIT_RIS_M : EMIT_RIS_M / 2u, s, lb, v, R.dim(D_EMIT));
        else if (S.pf(P_LIGHT_LOD + 3) > 0.0f) es = sample_emitter_ris(S, R, o, ne, 2u, s, lb, v, R.dim(D_EMIT));
        else es = sample_emitter(S, R, o, ne, R.dim(D_EMIT));
        if (es.pdf_w > 0.0f) {
            V3 f = eval_bsdf(s, lb, v, es.l);
            if (any_gt0(f)) {
                // emitter_tr: any surface stops it (TRACE_ANY), to 0.999 of the distance
                bool vis = trace(S, o, es.l, es.dist * 0.999f, TRACE_ANY, C).tri == MISS;
                if (vis) {
                    float wgt = light_mis(es.pdf_w, s, lb, v, es.l) * 1.0f;
                    sum = sum + es.le * f * wgt * es.w;
                }
            }
        }
    }
    if (env_sampled(S)) sum = sum + env_light(S, R, s, lb, v, o, C);
    return sum;
}

// pathtrace.wgsl:4002-4026 camera_ray (offline: the sample's own jitter)
void camera_ray(const Scene& S, uint32_t gx, uint32_t gy, const float cam[4], V3& o, V3& d) {
    float w = (float)S.pu(P_SIZE), h = (float)S.pu(P_SIZE + 1);
    float ndcx = ((float)gx + cam[0]) / w * 2.0f - 1.0f;
    float ndcy = 1.0f - ((float)gy + cam[1]) / h * 2.0f;
    V3 fwd = S.pv(P_CAM_FWD), right = S.pv(P_CAM_RIGHT), up = S.pv(P_CAM_UP);
    float tanf_ = S.pf(P_CAM_POS + 3), aspect = S.pf(P_CAM_FWD + 3);
    d = normalize(fwd + right * (ndcx * tanf_ * aspect) + up * (ndcy * tanf_));
    o = S.pv(P_CAM_POS);
    if (S.pf(P_CAM_RIGHT + 3) > 0.0f) {
        V3 focus = o + d * (S.pf(P_CAM_UP + 3) / dot(d, fwd));
        float r = std::sqrt(cam[2]) * S.pf(P_CAM_RIGHT + 3);
        float phi = 2.0f * PI * cam[3];
        o = o + right * (r * std::cos(phi)) + up * (r * std::sin(phi));
        d = normalize(focus - o);
    }
}

// pathtrace.wgsl:4105-4558 main, offline (LIVE false), FEAT = F_INST: one path of pixel (gx, gy), sample `sample`.
void path(const Scene& S, uint32_t gx, uint32_t gy, uint32_t sample, float* px, Counters& C) {
    Rng R;
    R.start(gx, gy, sample, S.pu(P_SIZE + 3), 0u);
    R.depth = 0;
    float cam[4];
    R.rng4(R.dim(D_CAMERA), cam);
    V3 o, d;
    camera_ray(S, gx, gy, cam, o, d);
    V3 radiance = v3(0.0f), thr = v3(1.0f), albedo = v3(0.0f), normal = v3(0.0f);
    float first_t = 0.0f, last_pdf = 0.0f;
    bool specular_bounce = true, behind_glass = false, bent = false, straight = true;
    float clamp_v = S.pf(P_MISC);
    PathState st;
    uint32_t last = S.pu(P_COUNTS + 2);
    for (uint32_t depth = 0; depth <= last; ++depth) {
        R.depth = depth;
        Hit hit = trace(S, o, d, INF, TRACE_CLOSEST, C);
        if (hit.tri == MISS) {
            V3 c = thr * sky_mis(S, d, (depth > 0u && !bent) ? last_pdf : 0.0f);
            if (depth > 1u && !straight) {
                float lum = luminance(c);
                if (lum > clamp_v) c = c * (clamp_v / lum);
            }
            radiance = radiance + c;
            break;
        }
        Surface s = surface(S, o, d, hit);
        if (depth == 0u) {
            first_t = hit.t;
            albedo = s.card ? s.emissive / fmax_(fmax_(s.emissive.x, fmax_(s.emissive.y, s.emissive.z)), 1e-6f) : s.base;
            normal = s.n;
        }
        if (any_gt0(s.emissive) && (s.front || !s.card)) {
            float wgt = 1.0f;
            if (depth > 0u && !specular_bounce && !behind_glass) wgt = emit_mis(S, hit, d, last_pdf, st.mis_x, st.mis_n);
            V3 c = thr * s.emissive * wgt;
            if (depth > 1u && !straight) {
                float lum = luminance(c);
                if (lum > clamp_v) c = c * (clamp_v / lum);
            }
            radiance = radiance + c;
        }
        if (s.card) break;
        if (depth == last) break;
        V3 v = -d;
        float nov = fmax_(dot(s.n, v), 1e-4f);
        Lobes lb = lobes(S, s, nov);
        V3 dl = thr * direct_light(S, R, s, lb, v, st, C);
        if (depth > 0u && !straight) {
            float lum = luminance(dl);
            if (lum > clamp_v) dl = dl * (clamp_v / lum);
        }
        radiance = radiance + dl;
        // sample_bsdf (1848-1887, no coat, no glass)
        Mat3 tbn = basis(s.n);
        float r4[4];
        R.rng4(R.dim(D_BSDF), r4);
        bool sampled_spec = r4[1] < lb.p_spec;
        V3 l;
        if (sampled_spec) {
            V3 h = sample_vndf(v, tbn, s.roughness * s.roughness, r4[2], r4[3]);
            l = reflect(-v, h);
        } else {
            float rr = std::sqrt(r4[2]);
            float phi = 2.0f * PI * r4[3];
            l = mul(tbn, V3{rr * std::cos(phi), rr * std::sin(phi), std::sqrt(fmax_(0.0f, 1.0f - rr * rr))});
        }
        float pdf = pdf_bsdf(s, lb, v, l);
        V3 wgt = eval_bsdf(s, lb, v, l) / fmax_(pdf, 1e-20f);
        if (pdf <= 0.0f || all_le0(wgt)) break;
        thr = thr * wgt;
        last_pdf = pdf;
        specular_bounce = false;
        behind_glass = false;
        bent = false;
        straight = false;
        st.mirror_path = (depth == 0u || st.mirror_path) && s.roughness < MIRROR_ROUGHNESS && sampled_spec;
        if (depth >= S.pu(P_COUNTS + 3)) {
            float q = fmin_(fmax_(thr.x, fmax_(thr.y, thr.z)), 0.95f);
            if (R.rng1(R.dim(D_RR)) > q) break;
            thr = thr / q;
        }
        o = offset_origin(s.p, dot(l, s.ng) < 0.0f ? -s.ng : s.ng);
        d = l;
    }
    (void)first_t;
    if (non_finite3(radiance)) radiance = v3(0.0f);
    if (non_finite3(albedo)) albedo = v3(0.0f);
    if (non_finite3(normal)) normal = V3{0.0f, 1.0f, 0.0f};
    px[0] += radiance.x; px[1] += radiance.y; px[2] += radiance.z; px[3] += 1.0f;
    float lum = luminance(radiance);
    px[4] += albedo.x; px[5] += albedo.y; px[6] += albedo.z; px[7] += lum;
    px[8] += normal.x; px[9] += normal.y; px[10] += normal.z; px[11] += lum * lum;
}

template <class F>
void parallel_for(uint64_t n, int threads, F&& f) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint64_t> next{0};
    const uint64_t chunk = 64;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t]() {
            for (;;) {
                uint64_t a = next.fetch_add(chunk);
                if (a >= n) break;
                uint64_t b = std::min(n, a + chunk);
                f(t, a, b);
            }
        });
    for (auto& th : pool) th.join();
}

void add_stats(orc_stats* st, const std::vector<Counters>& cs) {
    if (!st) return;
    std::memset(st, 0, sizeof(*st));
    for (const Counters& c : cs) {
        st->closest_rays += c.closest;
        st->shadow_rays += c.shadow;
        st->node_visits += c.nodes;
        st->tri_tests += c.tris;
        st->unit_entries += c.units;
    }
}

int render_list(const orc_scene* s, const uint32_t* params, uint32_t first_sample, uint32_t spp,
                const uint32_t* pixels, uint64_t n_pixels, float* accum, int threads, orc_stats* stats) {
    Scene S(s, params);
    uint32_t w = S.pu(P_SIZE), h = S.pu(P_SIZE + 1);
    uint64_t n = pixels ? n_pixels : (uint64_t)w * h;
    int nt = threads <= 0 ? (int)std::max(1u, std::thread::hardware_concurrency()) : threads;
    std::vector<Counters> cs(nt);
    parallel_for(n, nt, [&](int t, uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) {
            uint64_t pix = pixels ? pixels[i] : i;
            uint32_t gx = (uint32_t)(pix % w), gy = (uint32_t)(pix / w);
            for (uint32_t k = 0; k < spp; ++k) path(S, gx, gy, first_sample + k, accum + 20 * pix, cs[t]);
        }
    });
    add_stats(stats, cs);
    return 0;
}

}  // namespace

extern "C" {

int orc_render(const orc_scene* s, const uint32_t* params, uint32_t first_sample, uint32_t spp, float* accum,
               int threads, orc_stats* stats) {
    return render_list(s, params, first_sample, spp, nullptr, 0, accum, threads, stats);
}

int orc_render_pixels(const orc_scene* s, const uint32_t* params, uint32_t first_sample, uint32_t spp,
                      const uint32_t* pixels, uint64_t n_pixels, float* accum, int threads, orc_stats* stats) {
    return render_list(s, params, first_sample, spp, pixels, n_pixels, accum, threads, stats);
}

int orc_trace(const orc_scene* s, const uint32_t* params, const orc_ray* rays, uint64_t n, orc_hit* hits,
              int threads, orc_stats* stats) {
    Scene S(s, params);
    int nt = threads <= 0 ? (int)std::max(1u, std::thread::hardware_concurrency()) : threads;
    std::vector<Counters> cs(nt);
    parallel_for(n, nt, [&](int t, uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) {
            const orc_ray& r = rays[i];
            Hit h = trace(S, V3{r.o[0], r.o[1], r.o[2]}, V3{r.d[0], r.d[1], r.d[2]}, r.tmax, r.mode, cs[t]);
            hits[i] = orc_hit{h.t, h.tri, h.u, h.v, h.inst, h.part};
        }
    });
    add_stats(stats, cs);
    return 0;
}

int orc_trace_brute(const orc_scene* s, const uint32_t* params, const orc_ray* rays, uint64_t n, orc_hit* hits,
                    int threads) {
    Scene S(s, params);
    parallel_for(n, threads, [&](int, uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) {
            const orc_ray& r = rays[i];
            Hit h = trace_brute(S, V3{r.o[0], r.o[1], r.o[2]}, V3{r.d[0], r.d[1], r.d[2]}, r.tmax, r.mode);
            hits[i] = orc_hit{h.t, h.tri, h.u, h.v, h.inst, h.part};
        }
    });
    return 0;
}

int orc_intersect(const orc_scene* s, const uint32_t* params, const orc_ray* rays, const orc_hit* which, uint64_t n,
                  float* t_out) {
    Scene S(s, params);
    for (uint64_t i = 0; i < n; ++i) {
        const orc_ray& r = rays[i];
        t_out[i] = INF;
        if (which[i].tri == MISS || which[i].inst == NO_INST) continue;
        Instance u = S.instance(which[i].inst);
        V3 o{r.o[0], r.o[1], r.o[2]}, d{r.d[0], r.d[1], r.d[2]};
        V3 ro = o - V3{u.m[0][3], u.m[1][3], u.m[2][3]}, rd = d;
        if ((bu(u.n[1][3]) & UNIT_SHIFTED) == 0) { ro = proc_dir(u, ro); rd = proc_dir(u, d); }
        float x[3];
        intersect_tri(S, ro, rd, which[i].tri, INF, x);
        t_out[i] = x[0];
    }
    return 0;
}

void orc_rng4(uint32_t pixel_seed, uint32_t index, uint32_t dim, float out[4]) {
    Rng R;
    R.seed = pixel_seed;
    R.index = index;
    // sample.rs:79-83 rng4 takes the dimension id itself (no rng_dim).
    uint32_t s = pixel_seed ^ hash_hp(dim);
    uint32_t i = owen_rev(reverse_bits(index), s ^ 0xc2c1a055u) & 0xffff0000u;
    out[0] = sobol_owen(i, 0, s ^ 0x39468210u);
    out[1] = sobol_owen(i, 1, s ^ 0xe9d8a845u);
    out[2] = sobol_owen(i, 2, s ^ 0x5f32b482u);
    out[3] = sobol_owen(i, 3, s ^ 0x1524cc56u);
    (void)R;
}

void orc_sobol_directions(uint32_t out[96]) {
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 32; ++i) out[k * 32 + i] = sobol_table().d[k][i];
}

uint32_t orc_hash_hp(uint32_t x) { return hash_hp(x); }

int orc_hardware_threads(void) { return (int)std::max(1u, std::thread::hardware_concurrency()); }

}  // extern "C"
