// Test infrastructure, not product code: the oracle of the per-frame deformation (oracle.h says what it is for).
//
// Restates, one element after another, renderer/shaders/skin.wgsl main (the skinning pass), renderer/shaders/
// leaf_gather.wgsl main (the leaves again from the vertices) and renderer/src/units.rs:251-275 refit (a tree's boxes
// from its last node back to its root). f32 arithmetic in source order (built with -ffp-contract=off); glam's
// Vec3A::min / max are SSE minps / maxps: the first operand where it is smaller (larger), else the second.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "oracle.h"

namespace {

struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };
inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross3(F3 a, F3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline F4 add4(F4 a, F4 b) { return F4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline F4 mul4(F4 a, float s) { return F4{a.x * s, a.y * s, a.z * s, a.w * s}; }
inline float dot4(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline F3 xyz(F4 a) { return f3(a.x, a.y, a.z); }
inline uint32_t bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float from_bits(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
// skin.wgsl finite: the exponent is not all ones.
inline bool finite1(float v) { return (bits(v) & 0x7f800000u) != 0x7f800000u; }
inline float gmin(float a, float b) { return a < b ? a : b; }
inline float gmax(float a, float b) { return a > b ? a : b; }
inline F4 load4(const float* p) { return F4{p[0], p[1], p[2], p[3]}; }

struct Job { uint32_t first_vertex, n_vertices, first_corner, palette, first_tri, n_tris, root, n_nodes; };

// skin.wgsl:56-61 unit
F3 unit(F3 v) {
    float l = std::sqrt(dot3(v, v));
    if (l > 0.0f && finite1(l)) return f3(v.x / l, v.y / l, v.z / l);
    return f3(0.0f, 0.0f, 0.0f);
}

F3 corner_pos(const Job& J, const float* vertices, const uint32_t* words, uint32_t w_indices, uint32_t t, uint32_t c) {
    const float* p = vertices + 12ull * (J.first_vertex + words[w_indices + t * 3u + c]);
    return f3(p[0], p[1], p[2]);
}

}  // namespace

extern "C" {

int orc_skin(const uint32_t* jobs, uint32_t n_jobs, const float* corners, const float* palette, float* vertices) {
    for (uint32_t m = 0; m < n_jobs; ++m) {
        Job J;
        std::memcpy(&J, jobs + 8ull * m, sizeof(J));
        for (uint32_t local = 0; local < J.n_vertices; ++local) {
            // skin.wgsl:66-90 place
            const float* c = corners + 16ull * (J.first_corner + local);
            F4 cp = load4(c), cn = load4(c + 4), ct = load4(c + 8), cw = load4(c + 12);
            uint32_t a = bits(cp.w), b = bits(cn.w), flags = bits(ct.w);
            uint32_t j0 = (J.palette + (a & 0xffffu)) * 3u, j1 = (J.palette + (a >> 16)) * 3u;
            uint32_t j2 = (J.palette + (b & 0xffffu)) * 3u, j3 = (J.palette + (b >> 16)) * 3u;
            auto row = [&](uint32_t j) { return load4(palette + 4ull * j); };
            F4 r0 = add4(add4(add4(mul4(row(j0), cw.x), mul4(row(j1), cw.y)), mul4(row(j2), cw.z)), mul4(row(j3), cw.w));
            F4 r1 = add4(add4(add4(mul4(row(j0 + 1), cw.x), mul4(row(j1 + 1), cw.y)), mul4(row(j2 + 1), cw.z)), mul4(row(j3 + 1), cw.w));
            F4 r2 = add4(add4(add4(mul4(row(j0 + 2), cw.x), mul4(row(j1 + 2), cw.y)), mul4(row(j2 + 2), cw.z)), mul4(row(j3 + 2), cw.w));
            F4 p = F4{cp.x, cp.y, cp.z, 1.0f};
            F3 R0 = xyz(r0), R1 = xyz(r1), R2 = xyz(r2), N = xyz(cn), T = xyz(ct);
            F3 c12 = cross3(R1, R2);
            F3 n = f3(dot3(c12, N), dot3(cross3(R2, R0), N), dot3(cross3(R0, R1), N));
            if (dot3(R0, c12) < 0.0f) n = f3(-n.x, -n.y, -n.z);
            F3 q = f3(dot4(r0, p), dot4(r1, p), dot4(r2, p));
            // skin.wgsl:100-113 main's writes
            if (!(finite1(q.x) && finite1(q.y) && finite1(q.z))) q = f3(0.0f, 0.0f, 0.0f);
            float* v = vertices + 12ull * (J.first_vertex + local);
            v[0] = q.x; v[1] = q.y; v[2] = q.z;
            if (flags & 1u) {
                F3 un = unit(n);
                v[4] = un.x; v[5] = un.y; v[6] = un.z;
            }
            if (flags & 2u) {
                F3 ut = unit(f3(dot3(R0, T), dot3(R1, T), dot3(R2, T)));
                v[8] = ut.x; v[9] = ut.y; v[10] = ut.z;
            }
        }
    }
    return 0;
}

int orc_leaf_gather(const uint32_t* jobs, uint32_t n_jobs, const float* vertices, const uint32_t* words,
                    uint32_t w_indices, float* leaves) {
    for (uint32_t m = 0; m < n_jobs; ++m) {
        Job J;
        std::memcpy(&J, jobs + 8ull * m, sizeof(J));
        for (uint32_t local = 0; local < J.n_tris; ++local) {
            // leaf_gather.wgsl:41-51
            uint32_t t = J.first_tri + local;
            F3 p0 = corner_pos(J, vertices, words, w_indices, t, 0);
            F3 p1 = corner_pos(J, vertices, words, w_indices, t, 1);
            F3 p2 = corner_pos(J, vertices, words, w_indices, t, 2);
            F3 e1 = sub(p1, p0), e2 = sub(p2, p0);
            float* l = leaves + 12ull * t;
            l[0] = p0.x; l[1] = p0.y; l[2] = p0.z;
            l[4] = e1.x; l[5] = e1.y; l[6] = e1.z;
            l[8] = e2.x; l[9] = e2.y; l[10] = e2.z; l[11] = 0.0f;
        }
    }
    return 0;
}

int orc_refit(const uint32_t* jobs, uint32_t n_jobs, const float* vertices, const uint32_t* words, uint32_t w_indices,
              uint32_t* nodes) {
    const float inf = from_bits(0x7f800000u), ninf = from_bits(0xff800000u);
    for (uint32_t m = 0; m < n_jobs; ++m) {
        Job J;
        std::memcpy(&J, jobs + 8ull * m, sizeof(J));
        // units.rs:251-275: from the last node back; children lie after their parents.
        for (uint32_t k = J.n_nodes; k-- > 0;) {
            uint32_t* n = nodes + 8ull * (J.root + k);
            F3 lo = f3(inf, inf, inf), hi = f3(ninf, ninf, ninf);
            if (n[7] > 0) {
                for (uint32_t i = n[3]; i < n[3] + n[7]; ++i)
                    for (uint32_t c = 0; c < 3; ++c) {
                        F3 v = corner_pos(J, vertices, words, w_indices, J.first_tri + i, c);
                        if (std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z)) {
                            lo = f3(gmin(lo.x, v.x), gmin(lo.y, v.y), gmin(lo.z, v.z));
                            hi = f3(gmax(hi.x, v.x), gmax(hi.y, v.y), gmax(hi.z, v.z));
                        }
                    }
                if (lo.x > hi.x) { lo = f3(0.0f, 0.0f, 0.0f); hi = lo; }
            } else {
                const uint32_t* a = nodes + 8ull * (J.root + n[3]);
                const uint32_t* b = a + 8;
                lo = f3(gmin(from_bits(a[0]), from_bits(b[0])), gmin(from_bits(a[1]), from_bits(b[1])),
                        gmin(from_bits(a[2]), from_bits(b[2])));
                hi = f3(gmax(from_bits(a[4]), from_bits(b[4])), gmax(from_bits(a[5]), from_bits(b[5])),
                        gmax(from_bits(a[6]), from_bits(b[6])));
            }
            n[0] = bits(lo.x); n[1] = bits(lo.y); n[2] = bits(lo.z);
            n[4] = bits(hi.x); n[5] = bits(hi.y); n[6] = bits(hi.z);
        }
    }
    return 0;
}

}  // extern "C"
