// Test infrastructure, not product code: the oracle of the denoiser fallback (oracle.h says what it is for).
//
// Restates renderer/src/denoise.rs `denoise` (the a-trous filter main.rs:548-557 runs with 4 iterations) over the
// Frame of each Pixel (gpu.rs:4219-4232), in f32 and in the reference's order, one pixel after another.
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle.h"

namespace {

struct F3 { float x, y, z; };
inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 mul(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float lum(F3 c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }
inline float fin(float v) { return std::isfinite(v) ? v : 0.0f; }
inline F3 max_eps(F3 a) { return f3(std::fmax(a.x, 1e-3f), std::fmax(a.y, 1e-3f), std::fmax(a.z, 1e-3f)); }
inline float pow64(float x) {
    for (int k = 0; k < 6; ++k) x = x * x;
    return x;
}

}  // namespace

extern "C" int orc_denoise(const float* accum, uint32_t w, uint32_t h, uint32_t iterations, float* rgb) {
    const size_t n = (size_t)w * h;
    std::vector<F3> albedo(n), normal(n), cur(n), next(n);
    std::vector<float> var(n), var_f(n), next_var(n);
    for (size_t i = 0; i < n; ++i) {
        const float* p = accum + 20 * i;
        float c = std::fmax(fin(p[3]), 1.0f);
        F3 color = f3(fin(p[0]) / c, fin(p[1]) / c, fin(p[2]) / c);
        albedo[i] = f3(fin(p[4]) / c, fin(p[5]) / c, fin(p[6]) / c);
        F3 nr = f3(fin(p[8]) / c, fin(p[9]) / c, fin(p[10]) / c);
        float mean = fin(p[7]) / c;
        float variance = std::fmax(fin(p[11]) / c - mean * mean, 0.0f) / c;
        float rcp = 1.0f / std::sqrt(dot(nr, nr));  // normalize_or_zero
        normal[i] = (std::isfinite(rcp) && rcp > 0.0f) ? mul(nr, rcp) : f3(0, 0, 0);
        F3 ae = max_eps(albedo[i]);
        cur[i] = f3(color.x / ae.x, color.y / ae.y, color.z / ae.z);
        float la = lum(ae);
        var[i] = variance / (la * la);
    }
    const float K[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    for (uint32_t it = 0; it < iterations; ++it) {
        int step = 1 << it;
        for (size_t i = 0; i < n; ++i) {
            int x = (int)(i % w), y = (int)(i / w);
            float s = 0.0f, ws = 0.0f;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int qx = x + dx, qy = y + dy;
                    if (qx < 0 || qy < 0 || qx >= (int)w || qy >= (int)h) continue;
                    float k = (dx == 0 ? 0.5f : 0.25f) * (dy == 0 ? 0.5f : 0.25f);
                    s += k * var[(size_t)qy * w + qx];
                    ws += k;
                }
            var_f[i] = s / ws;
        }
        for (size_t i = 0; i < n; ++i) {
            int x = (int)(i % w), y = (int)(i / w);
            F3 cp = cur[i];
            float lp = lum(cp);
            float sigma_l = 4.0f * std::sqrt(std::fmax(var_f[i], 0.0f)) + 1e-4f;
            F3 sum = f3(0, 0, 0);
            float wsum = 0.0f, vsum = 0.0f;
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx) {
                    int qx = x + dx * step, qy = y + dy * step;
                    if (qx < 0 || qy < 0 || qx >= (int)w || qy >= (int)h) continue;
                    size_t q = (size_t)qy * w + qx;
                    float k = K[dx < 0 ? -dx : dx] * K[dy < 0 ? -dy : dy];
                    F3 cq = cur[q];
                    float wl = std::exp(-std::fabs(lp - lum(cq)) / sigma_l);
                    float wn = pow64(std::fmax(dot(normal[i], normal[q]), 0.0f));
                    F3 da = sub(albedo[i], albedo[q]);
                    float wa = std::exp(-dot(da, da) / 0.01f);
                    float wt = k * wl * wn * wa;
                    sum = add(sum, mul(cq, wt));
                    vsum += wt * wt * var[q];
                    wsum += wt;
                }
            if (wsum > 0.0f) {
                next[i] = f3(sum.x / wsum, sum.y / wsum, sum.z / wsum);
                next_var[i] = vsum / (wsum * wsum);
            } else {
                next[i] = cp;
                next_var[i] = var[i];
            }
        }
        cur.swap(next);
        var.swap(next_var);
    }
    for (size_t i = 0; i < n; ++i) {
        F3 ae = max_eps(albedo[i]);
        rgb[3 * i] = cur[i].x * ae.x;
        rgb[3 * i + 1] = cur[i].y * ae.y;
        rgb[3 * i + 2] = cur[i].z * ae.z;
    }
    return 0;
}
