// The denoiser fallback: renderer/src/denoise.rs `denoise` (edge-avoiding a-trous wavelet filter, Dammertz et al.
// 2010, guided by first-hit albedo and normal, its luminance edge-stopping width from the variance filtered over 3 x 3
// pixels as in SVGF), run on the scene's accum on the device. main.rs:548-557 calls it with 4 iterations on the Frame
// (gpu.rs:4219-4232: each Pixel over its count, the normal normalised or zero). Included by pathtrace.cu.
//
// Arithmetic follows denoise.rs in f32 and in its order; `exp` is the device's expf (within a few ulps of libm), so
// results match the oracle's restatement to ~1e-5 relative, not bit for bit.
#pragma once

namespace trt {

constexpr float DN_EPS = 1e-3f;
// denoise.rs:16 K: the B3 spline's taps 3/8, 1/4, 1/16 by distance
__device__ __forceinline__ float dn_k(int a) { return a == 0 ? 0.375f : (a == 1 ? 0.25f : 0.0625f); }

struct DenoiseBufs {
    float4* cur[2];   // demodulated irradiance (xyz)
    float* var[2];    // its variance
    float* var_f;     // the variance filtered over 3 x 3
    float4* alb;      // first-hit albedo (the Frame's)
    float4* nrm;      // first-hit normal, normalised or zero
};

__device__ __forceinline__ float dn_fin(float v) { return (__float_as_uint(v) & 0x7f800000u) == 0x7f800000u ? 0.0f : v; }
__device__ __forceinline__ V3 dn_max_eps(V3 a) { return V3{fmaxf(a.x, DN_EPS), fmaxf(a.y, DN_EPS), fmaxf(a.z, DN_EPS)}; }

// gpu.rs:4219-4232 (the Frame of a Pixel) and denoise.rs:11-15 (demodulation, the variance in irradiance units).
__global__ void k_dn_prep(const float4* __restrict__ accum, uint32_t n, DenoiseBufs D) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 c = accum[5ull * i], a = accum[5ull * i + 1], nn = accum[5ull * i + 2];
    float cnt = fmaxf(dn_fin(c.w), 1.0f);
    V3 color = V3{dn_fin(c.x) / cnt, dn_fin(c.y) / cnt, dn_fin(c.z) / cnt};
    V3 albedo = V3{dn_fin(a.x) / cnt, dn_fin(a.y) / cnt, dn_fin(a.z) / cnt};
    V3 normal = V3{dn_fin(nn.x) / cnt, dn_fin(nn.y) / cnt, dn_fin(nn.z) / cnt};
    float mean = dn_fin(a.w) / cnt;
    float variance = fmaxf(dn_fin(nn.w) / cnt - mean * mean, 0.0f) / cnt;
    // glam normalize_or_zero: v / |v| where 1 / |v| is finite and positive
    float len = sqrtf(dot(normal, normal));
    float rcp = 1.0f / len;
    normal = (rcp > 0.0f && (__float_as_uint(rcp) & 0x7f800000u) != 0x7f800000u) ? normal * rcp : v3(0.0f);
    V3 ae = dn_max_eps(albedo);
    V3 demod = V3{color.x / ae.x, color.y / ae.y, color.z / ae.z};
    float la = dot(ae, V3{0.2126f, 0.7152f, 0.0722f});
    D.cur[0][i] = f4(demod, 0.0f);
    D.var[0][i] = variance / (la * la);
    D.alb[i] = f4(albedo, 0.0f);
    D.nrm[i] = f4(normal, 0.0f);
}

// denoise.rs:20-35: the variance over 3 x 3 pixels, weights 0.5 / 0.25 a tap along each axis, over the taps inside.
__global__ void k_dn_var3(const float* __restrict__ var, float* var_f, uint32_t w, uint32_t h) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    int x = (int)(i % w), y = (int)(i / w);
    float s = 0.0f, ws = 0.0f;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            int qx = x + dx, qy = y + dy;
            if (qx < 0 || qy < 0 || qx >= (int)w || qy >= (int)h) continue;
            float k = (dx == 0 ? 0.5f : 0.25f) * (dy == 0 ? 0.5f : 0.25f);
            s += k * var[(uint32_t)qy * w + (uint32_t)qx];
            ws += k;
        }
    var_f[i] = s / ws;
}

__device__ __forceinline__ float pow64(float x) {
    // x^64 by six squarings (what powi(64) comes to)
    x = x * x; x = x * x; x = x * x; x = x * x; x = x * x;
    return x * x;
}

// denoise.rs:36-68: one a-trous iteration at `step`, 5 x 5 taps of the B3 spline kernel.
__global__ void k_dn_atrous(DenoiseBufs D, uint32_t src, uint32_t w, uint32_t h, int step) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    int x = (int)(i % w), y = (int)(i / w);
    const float4* cur = D.cur[src];
    const float* var = D.var[src];
    V3 cp = xyz(cur[i]);
    float lp = luminance(cp);
    V3 np = xyz(D.nrm[i]), ap = xyz(D.alb[i]);
    float sigma_l = 4.0f * sqrtf(fmaxf(D.var_f[i], 0.0f)) + 1e-4f;
    V3 sum = v3(0.0f);
    float wsum = 0.0f, vsum = 0.0f;
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            int qx = x + dx * step, qy = y + dy * step;
            if (qx < 0 || qy < 0 || qx >= (int)w || qy >= (int)h) continue;
            uint32_t q = (uint32_t)qy * w + (uint32_t)qx;
            float k = dn_k(dx < 0 ? -dx : dx) * dn_k(dy < 0 ? -dy : dy);
            V3 cq = xyz(cur[q]);
            float wl = expf(-fabsf(lp - luminance(cq)) / sigma_l);
            float wn = pow64(fmaxf(dot(np, xyz(D.nrm[q])), 0.0f));
            V3 da = ap - xyz(D.alb[q]);
            float wa = expf(-dot(da, da) / 0.01f);
            float wt = k * wl * wn * wa;
            sum = sum + cq * wt;
            vsum += wt * wt * var[q];
            wsum += wt;
        }
    uint32_t dst = src ^ 1u;
    if (wsum > 0.0f) {
        D.cur[dst][i] = f4(sum / wsum, 0.0f);
        D.var[dst][i] = vsum / (wsum * wsum);
    } else {
        D.cur[dst][i] = f4(cp, 0.0f);
        D.var[dst][i] = var[i];
    }
}

// denoise.rs:72: the filtered irradiance times the albedo again, as RGB floats.
__global__ void k_dn_remod(DenoiseBufs D, uint32_t src, uint32_t n, float* rgb) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 c = xyz(D.cur[src][i]);
    V3 ae = dn_max_eps(xyz(D.alb[i]));
    rgb[3ull * i] = c.x * ae.x;
    rgb[3ull * i + 1] = c.y * ae.y;
    rgb[3ull * i + 2] = c.z * ae.z;
}

}  // namespace trt
