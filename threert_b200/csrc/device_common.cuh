// Device-side vocabulary of the pass: vector math with the WGSL semantics the reference kernel relies on, the
// sampler (renderer/shaders/sample.wgsl), and typed reads of the reference's packed buffers (the bindings of
// renderer/shaders/pathtrace.wgsl:141-268, here plain global-memory pointers).
//
// Arithmetic is written in source order and this code is compiled with -fmad=false, so no multiply-add is fused;
// division and sqrt are IEEE (nvcc's defaults without --use_fast_math). Everything that is not a transcendental then
// rounds exactly as the C++ restatement does.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace trt {

constexpr float PI = 3.14159265358979f;        // pathtrace.wgsl:25
constexpr float INF = 3.0e38f;                  // pathtrace.wgsl:26
constexpr uint32_t MISS = 0xffffffffu;
constexpr uint32_t NO_INST = 0xffffffffu;       // pathtrace.wgsl:637
constexpr uint32_t TRACE_CLOSEST = 0, TRACE_SHADOW = 1, TRACE_ANY = 2;
constexpr uint32_t UNIT_SHADOW = 1, UNIT_SHIFTED = 2, INST_MIRRORED = 4;
constexpr uint32_t ROW_MATERIAL = 0xffffffu, NO_EMITTER = 0xffffffffu;
constexpr int32_t MAT_EMITTER_CARD = 2;
constexpr uint32_t EMITTER_GUIDE = 65536u, LT_LEAF = 0x80000000u, LT_PATH_BITS = 26u;
constexpr uint32_t EMITTER_MOVES = 0x80000000u, EMITTER_CARD = 1u, EMIT_RIS_M = 6u;
constexpr float MIRROR_ROUGHNESS = 0.3f;
constexpr uint32_t ENERGY_N = 32u;
constexpr uint32_t D_CAMERA = 0, D_BSDF = 1, D_RR = 2, D_SUN = 4, D_EMIT = 7, D_ENV = 9;

// Params word offsets (renderer/src/gpu.rs:127-186).
enum : uint32_t {
    P_CAM_POS = 0, P_CAM_FWD = 4, P_CAM_RIGHT = 8, P_CAM_UP = 12, P_SIZE = 16, P_COUNTS = 20, P_ENV = 24, P_MISC = 28,
    P_SKY = 32, P_COUNTS2 = 36, P_MOTION = 68, P_LIGHT_LOD = 72, P_LTREE = 84, P_TABLE_FIRST = 124, P_WORD_FIRST = 136,
    P_WORDS = 156
};
struct Params { uint32_t w[P_WORDS]; };

__host__ __device__ __forceinline__ float bf(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}
__host__ __device__ __forceinline__ uint32_t bu(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    return u;
#endif
}

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float a) { return {a, a, a}; }
__device__ __forceinline__ V3 mk3(float a, float b, float c) { return {a, b, c}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) {
    float l = sqrtf(dot(a, a));
    return {a.x / l, a.y / l, a.z / l};
}
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ bool any_gt0(V3 a) { return a.x > 0.0f || a.y > 0.0f || a.z > 0.0f; }
__device__ __forceinline__ bool all_le0(V3 a) { return a.x <= 0.0f && a.y <= 0.0f && a.z <= 0.0f; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 mix3(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 reflect(V3 i, V3 n) { return i - (2.0f * dot(n, i)) * n; }
__device__ __forceinline__ float luminance(V3 c) { return dot(c, V3{0.2126f, 0.7152f, 0.0722f}); }
__device__ __forceinline__ bool non_finite3(V3 v) {
    return (bu(v.x) & 0x7fffffffu) >= 0x7f800000u || (bu(v.y) & 0x7fffffffu) >= 0x7f800000u ||
           (bu(v.z) & 0x7fffffffu) >= 0x7f800000u;
}
__device__ __forceinline__ V3 xyz(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
// An IEEE binary16 value (the low 16 bits of h) as f32: the conversion is exact, one cvt instruction.
__device__ __forceinline__ float half_to_float(uint32_t h) { return __half2float(__ushort_as_half((unsigned short)h)); }

// ---- sampler (sample.wgsl) ---------------------------------------------------------------------------------------

// Sobol dimensions 1-3 of a 16-bit bit-reversed index: the XOR of the direction numbers of its set bits (sample.wgsl
// sobol_d1..d3), by bytes. g_sobol_bytes[d][0][b] is the XOR of directions 0-7 selected by bits 7..0 of b (the index's
// bits 31..24), [d][1][b] of directions 8-15 (bits 23..16): the same XOR in two loads. Filled at start-up from the
// Joe-Kuo recurrence (sobol_directions in pathtrace.cu).
__device__ uint32_t g_sobol_bytes[3][2][256];

__device__ __forceinline__ uint32_t sobol_dim(uint32_t x, int dim) {
    return __ldg(&g_sobol_bytes[dim - 1][0][x >> 24]) ^ __ldg(&g_sobol_bytes[dim - 1][1][(x >> 16) & 255u]);
}
__device__ __forceinline__ uint32_t owen_rev(uint32_t n, uint32_t seed) {
    n ^= n * 0x3d20adeau;
    n += seed;
    n *= (seed >> 16) | 1u;
    n ^= n * 0x05526c56u;
    n ^= n * 0x53a22864u;
    return n;
}
__host__ __device__ __forceinline__ uint32_t hash_hp(uint32_t i) {
    i ^= i >> 16;
    i *= 0x21f0aaadu;
    i ^= i >> 15;
    i *= 0xd35a2d97u;
    i ^= i >> 15;
    return i ^ 0xe6fe3bebu;
}
__device__ __forceinline__ float sobol_owen(uint32_t rev_index, uint32_t dim, uint32_t seed) {
    uint32_t r = dim == 0 ? __brev(rev_index) : sobol_dim(rev_index, (int)dim);
    r = __brev(owen_rev(r, seed));
    return __uint2float_rn(r) * (1.0f / 4294967808.0f);
}
__device__ __forceinline__ uint32_t rng_sub(uint32_t d, uint32_t k) {
    return hash_hp(d ^ hash_hp(k + 0x9e3779b9u)) | 0x80000000u;
}

// A path's sampler: its pixel seed, its sample index, its vertex (RNG_PATH is 0 offline).
struct Rng {
    uint32_t index, seed, depth;
    __device__ uint32_t dim(uint32_t slot) const { return (depth << 20) ^ slot; }
    __device__ uint32_t seed_of(uint32_t d) const { return seed ^ hash_hp(d); }
    __device__ uint32_t index_of(uint32_t salt) const { return owen_rev(__brev(index), salt) & 0xffff0000u; }
    __device__ float rng1(uint32_t d) const {
        uint32_t s = seed_of(d);
        return sobol_owen(index_of(s ^ 0xbff95bfeu), 0, s ^ 0x635c77bdu);
    }
    __device__ void rng2(uint32_t d, float o[2]) const {
        uint32_t s = seed_of(d), i = index_of(s ^ 0xf8ade99au);
        o[0] = sobol_owen(i, 0, s ^ 0xe0aaaf76u);
        o[1] = sobol_owen(i, 1, s ^ 0x94964d4eu);
    }
    __device__ void rng3(uint32_t d, float o[3]) const {
        uint32_t s = seed_of(d), i = index_of(s ^ 0xcaa726acu);
        o[0] = sobol_owen(i, 0, s ^ 0x9e78e391u);
        o[1] = sobol_owen(i, 1, s ^ 0x67c33241u);
        o[2] = sobol_owen(i, 2, s ^ 0x78c395c5u);
    }
    __device__ void rng4(uint32_t d, float o[4]) const {
        uint32_t s = seed_of(d), i = index_of(s ^ 0xc2c1a055u);
        o[0] = sobol_owen(i, 0, s ^ 0x39468210u);
        o[1] = sobol_owen(i, 1, s ^ 0xe9d8a845u);
        o[2] = sobol_owen(i, 2, s ^ 0x5f32b482u);
        o[3] = sobol_owen(i, 3, s ^ 0x1524cc56u);
    }
};
__device__ __forceinline__ uint32_t pixel_seed(uint32_t px, uint32_t py, uint32_t sd) {
    return hash_hp(px ^ hash_hp(py ^ hash_hp(sd)));
}

// ---- the scene as the device holds it ------------------------------------------------------------------------------

struct DScene {
    const float4* vertices;   // 3 vec4s a vertex
    const float4* leaves;     // 3 vec4s a triangle
    const uint4* nodes;       // GpuNode: 2 uint4s (bmin, left_or_first), (bmax, count)
    const uint4* tables;
    const uint32_t* words;
    const ushort4* env;       // RGBA16F texels
    uint32_t env_w, env_h;
    uint64_t n_nodes, n_tris, n_table_vec4, n_words;
};

// Table / word section starts read out of Params once per thread.
struct Sections {
    uint32_t t_materials, t_lights, t_emitters, t_objects, t_instances, t_energy, t_emitter_tris;
    uint32_t w_rows, w_indices;
    __device__ explicit Sections(const Params& P) {
        t_materials = P.w[P_TABLE_FIRST + 1];
        t_lights = P.w[P_TABLE_FIRST + 2];
        t_emitters = P.w[P_TABLE_FIRST + 4];
        t_objects = P.w[P_TABLE_FIRST + 6];
        t_instances = P.w[P_TABLE_FIRST + 7];
        t_energy = P.w[P_TABLE_FIRST + 9];
        t_emitter_tris = P.w[P_TABLE_FIRST + 11];
        w_rows = P.w[P_WORD_FIRST + 3];
        w_indices = P.w[P_WORD_FIRST + 4];
    }
};

__device__ __forceinline__ float pf(const Params& P, uint32_t w) { return bf(P.w[w]); }
__device__ __forceinline__ V3 pv(const Params& P, uint32_t w) { return {pf(P, w), pf(P, w + 1), pf(P, w + 2)}; }
__device__ __forceinline__ float4 tab(const DScene& S, uint32_t i) {
    uint4 u = __ldg(S.tables + i);
    return make_float4(bf(u.x), bf(u.y), bf(u.z), bf(u.w));
}
__device__ __forceinline__ uint4 tabu(const DScene& S, uint32_t i) { return __ldg(S.tables + i); }

struct Inst { float4 m0, m1, m2, n0, n1, n2; uint4 info; };
__device__ __forceinline__ Inst instance_at(const DScene& S, const Sections& X, uint32_t i) {
    uint32_t b = X.t_instances + i * 10u;
    Inst r;
    r.m0 = tab(S, b); r.m1 = tab(S, b + 1); r.m2 = tab(S, b + 2);
    r.n0 = tab(S, b + 3); r.n1 = tab(S, b + 4); r.n2 = tab(S, b + 5);
    r.info = tabu(S, b + 6);
    return r;
}

}  // namespace trt
