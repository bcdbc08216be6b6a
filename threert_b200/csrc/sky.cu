// The atmosphere's sky baked on the device: renderer/src/sky.rs's medium (Bruneton & Neyret 2008 / Hillaire 2020 as
// the reference states it), its tables (Luts::build_at, sky.rs:401-433) and its equirectangular bake
// (bake_atmosphere_with, sky.rs:722-819), then the environment's importance tables (lib.rs:916-941 build_env_cdf).
//
// The reference computes in f64 with a single-precision exponential of its own (exp4, sky.rs:93-105) and stores its
// tables in f32; so does this file, statement for statement, so that the bake matches a CPU restatement to float
// rounding. The work is laid out for the GPU instead of the reference's rayon loops:
//  - the sun's optical-depth table (257 x 128 entries): a thread an entry;
//  - each order of the scattered light (64 x 32 entries x 32 gathering directions): a warp an entry, a lane a
//    direction, the directions' sum taken by lane 0 in the reference's order;
//  - the bake: a thread a texel; the overcast blend's horizontal illuminance by fixed-order block sums in f64;
//  - the CDF: a block a row (the row's running sum is sequential in f32, as the reference's), one thread for the
//    marginal over rows.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "sky.h"

namespace trt_sky {

// sky.rs:27-70, 236, 362-372, 637, 706-710.
constexpr double R_GROUND = 6360.0, R_TOP = 6460.0;
constexpr double H_RAYLEIGH = 8.0, H_MIE = 1.2;
constexpr double MIE_SCATTERING = 3.996e-3, MIE_ABSORPTION = 0.444e-3;
constexpr double OZONE_CENTRE = 25.0, OZONE_HALF_WIDTH = 15.0;
constexpr double SOFT_GROUND = 5.0, R_BASE = R_GROUND - SOFT_GROUND;
constexpr double SUN_VEIL_COLUMN = 1.65, SUN_VEIL_ALTITUDE = 55.0;
constexpr double OPAQUE = 80.0;
constexpr double NIGHT = -0.3;
constexpr double PI = 3.14159265358979323846;
constexpr float PI_F = 3.14159265358979323846f;
constexpr int SUN_COLS = 257, SUN_ROWS = 128, SC_COLS = 64, SC_ROWS = 32;
constexpr int AZIMUTHS = 2, STEPS = 12, VIEW_STEPS = 16;
constexpr int DIRS = 32, DIRS_UP = 16;  // gathering directions (2 panels or 1) x 8 Gauss-Legendre nodes x 2 azimuths
constexpr float SKY_LIGHT_CUBE = 128.0f;
constexpr float OVERCAST_TRANSMITTANCE = 0.3f, OVERCAST_GLOW = 3.0f;
constexpr int SUN_ENTRIES = SUN_COLS * SUN_ROWS, SC_ENTRIES = SC_COLS * SC_ROWS;

// Gauss-Legendre, 8 points on [-1, 1], the positive half (sky.rs:118-123).
__constant__ double GL8_X[4] = {0.1834346424956498, 0.525532409916329, 0.7966664774136267, 0.9602898564975362};
__constant__ double GL8_W[4] = {0.362683783378362, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};

// Atmosphere::earth (sky.rs:170-185), scaled on the host.
struct Atm {
    double rayleigh[3], mie_scattering, mie_extinction, ozone[3], mie_g, ground_albedo[3];
};

struct D3 { double x, y, z; };

__device__ __forceinline__ D3 densities(double h) {
    return {exp(-h / H_RAYLEIGH), exp(-h / H_MIE), fmax(1.0 - fabs(h - OZONE_CENTRE) / OZONE_HALF_WIDTH, 0.0)};
}

// sky.rs:93-105: e^x in single precision (k ln 2 + r, e^r by its degree-7 Taylor polynomial, 2^k by its bits).
__device__ __forceinline__ double exp1f(double x) {
    float v = (float)x;
    v = v < -87.0f ? -87.0f : (v > 88.0f ? 88.0f : v);
    float k = floorf(v * 1.44269504088896340736f + 0.5f);
    float r = (v - k * 0.69314575f) - k * 1.4286068e-6f;
    float poly = 1.0f + r * (1.0f + r * (0.5f + r * (1.0f / 6.0f + r * (1.0f / 24.0f + r * (1.0f / 120.0f +
                 r * (1.0f / 720.0f + r * (1.0f / 5040.0f)))))));
    return (double)(poly * __int_as_float(((int)k + 127) << 23));
}

__device__ __forceinline__ double distance_out(double r, double mu, double to) {
    return -r * mu + sqrt(fmax(r * r * (mu * mu - 1.0) + to * to, 0.0));
}
__device__ __forceinline__ bool distance_to_ground(double r, double mu, double* d) {
    double disc = r * r * (mu * mu - 1.0) + R_GROUND * R_GROUND;
    if (!(mu < 0.0 && disc >= 0.0)) return false;
    *d = fmax(-r * mu - sqrt(disc), 0.0);
    return true;
}

// sky.rs:128-151: the columns to the top by 8-point Gauss-Legendre on 12 panels of u (t = d u^2).
__device__ D3 columns_exact(double r, double mu) {
    const int PANELS = 12;
    double d = distance_out(r, mu, R_TOP);
    D3 n = {0, 0, 0};
    for (int p = 0; p < PANELS; ++p) {
        double centre = ((double)p + 0.5) / (double)PANELS, half = 0.5 / (double)PANELS;
        for (int g = 0; g < 4; ++g) {
            for (int si = 0; si < 2; ++si) {
                double s = si == 0 ? -1.0 : 1.0;
                double u = centre + s * half * GL8_X[g];
                double t = d * u * u;
                D3 dens = densities(sqrt(r * r + t * t + 2.0 * r * mu * t) - R_GROUND);
                double k = GL8_W[g] * half * 2.0 * d * u;
                n.x += k * dens.x;
                n.y += k * dens.y;
                n.z += k * dens.z;
            }
        }
    }
    return n;
}

__device__ __forceinline__ D3 extinction(const Atm& a, double air, double haze, double ozone) {
    return {a.rayleigh[0] * air + a.mie_extinction * haze + a.ozone[0] * ozone,
            a.rayleigh[1] * air + a.mie_extinction * haze + a.ozone[1] * ozone,
            a.rayleigh[2] * air + a.mie_extinction * haze + a.ozone[2] * ozone};
}

// sky.rs:158-168 slant and 195-200 optical_depth: a ray that points down is the mirror of the one that points up
// from its lowest point; deeper than the soft ground it is opaque.
__device__ D3 optical_depth(const Atm& a, double r, double mu) {
    D3 n;
    double ground = 0.0;
    if (mu >= 0.0) {
        n = columns_exact(r, mu);
    } else {
        double p = r * sqrt(fmax(1.0 - mu * mu, 0.0));
        if (p <= R_BASE) return {OPAQUE, OPAQUE, OPAQUE};
        D3 level = columns_exact(p, 0.0), mirror = columns_exact(r, -mu);
        n = {fmax(2.0 * level.x - mirror.x, 0.0), fmax(2.0 * level.y - mirror.y, 0.0),
             fmax(2.0 * level.z - mirror.z, 0.0)};
        double dd = fmax((R_GROUND - p) / 2.0, 0.0);
        ground = dd * dd * dd * dd;
    }
    D3 e = extinction(a, n.x, n.y, n.z);
    return {fmin(e.x + ground, OPAQUE), fmin(e.y + ground, OPAQUE), fmin(e.z + ground, OPAQUE)};
}

// sky.rs:203-220 Atmosphere::sun_transmittance, times the sun's illuminance and the clouds' share (sky.rs:694-703).
__device__ float3 sun_illuminance(const Atm& a, float3 dir, float3 lux, float cover) {
    float len = sqrtf(dir.x * dir.x + dir.y * dir.y + dir.z * dir.z);
    float rcp = 1.0f / len;
    float y = (isfinite(rcp) && rcp > 0.0f) ? dir.y * rcp : 0.0f;
    double mu = fmin(fmax((double)y, -1.0), 1.0);
    D3 od = optical_depth(a, R_GROUND, mu);
    double level = R_GROUND / (R_GROUND + SUN_VEIL_ALTITUDE);
    double veil = SUN_VEIL_COLUMN / sqrt(1.0 - level * level * (1.0 - mu * mu));
    float t0 = (float)(exp(-od.x) * exp(-veil * (a.rayleigh[0] + a.mie_extinction)));
    float t1 = (float)(exp(-od.y) * exp(-veil * (a.rayleigh[1] + a.mie_extinction)));
    float t2 = (float)(exp(-od.z) * exp(-veil * (a.rayleigh[2] + a.mie_extinction)));
    float cloud = 1.0f - fminf(fmaxf(cover, 0.0f), 1.0f);
    return make_float3(lux.x * t0 * cloud, lux.y * t1 * cloud, lux.z * t2 * cloud);
}

// sky.rs:248-284: where a point is in the tables.
struct At { double sun, scatter, altitude; };
__device__ __forceinline__ At at_new(double mu_sun, double r) {
    double root = sqrt(fabs(mu_sun));
    double altitude = sqrt(fmin(fmax((r - R_GROUND) * (1.0 / (R_TOP - R_GROUND)), 0.0), 1.0));
    if (mu_sun >= 0.0) return {0.5 + 0.5 * root, 0.5 + 0.5 * root, altitude};
    double under = r * mu_sun * mu_sun / (1.0 + sqrt(fmax(1.0 - mu_sun * mu_sun, 0.0)));
    return {0.5 - 0.5 * sqrt(fmin(under / (r - R_BASE), 1.0)), 0.5 - 0.5 * root, altitude};
}
__device__ __forceinline__ double mu_of_scatter(double x) {
    double s = 2.0 * x - 1.0;
    return s * fabs(s);
}
__device__ __forceinline__ double mu_of_sun(double x, double r) {
    if (x >= 0.5) {
        double q = 2.0 * x - 1.0;
        return q * q;
    }
    double q = 1.0 - 2.0 * x;
    double p = r - (r - R_BASE) * (q * q);
    double pr = p / r;
    return -sqrt(fmax(1.0 - pr * pr, 0.0));
}
// Table::fill's radius of a row (sky.rs:295-300).
__device__ __forceinline__ double row_radius(int row, int rows) {
    double q = rows > 1 ? (double)row / (double)(rows - 1) : 0.0;
    return R_GROUND + q * q * (R_TOP - R_GROUND);
}

// sky.rs:306-325 Table::at: linear between entries, the weights and the blend in f32. `d`: 3 floats an entry.
__device__ __forceinline__ D3 table_at(const float* __restrict__ d, int columns, int rows, double column,
                                       double altitude) {
    double fu = column * (double)(columns - 1);
    int iu = min(fu > 0.0 ? (int)fu : 0, columns - 2);
    float wu = (float)(fu - (double)iu);
    auto row = [&](int v, float o[3]) {
        const float* p = d + 3 * (v * columns + iu);
        for (int c = 0; c < 3; ++c) o[c] = p[c] + (p[c + 3] - p[c]) * wu;
    };
    float lo[3], hi[3];
    if (rows == 1) {
        row(0, lo);
        return {(double)lo[0], (double)lo[1], (double)lo[2]};
    }
    double fv = altitude * (double)(rows - 1);
    int iv = min(fv > 0.0 ? (int)fv : 0, rows - 2);
    row(iv, lo);
    row(iv + 1, hi);
    float wv = (float)(fv - (double)iv);
    return {(double)(lo[0] + (hi[0] - lo[0]) * wv), (double)(lo[1] + (hi[1] - lo[1]) * wv),
            (double)(lo[2] + (hi[2] - lo[2]) * wv)};
}

// sky.rs:436-442 Luts::sun_transmittance: the table's optical depth as transmittance, none where it is opaque.
__device__ __forceinline__ D3 sun_transmittance_at(const float* __restrict__ sun, At at) {
    D3 t = table_at(sun, SUN_COLS, SUN_ROWS, at.sun, at.altitude);
    double lim = OPAQUE - 1.0;
    return {t.x < lim ? exp1f(-t.x) : 0.0, t.y < lim ? exp1f(-t.y) : 0.0, t.z < lim ? exp1f(-t.z) : 0.0};
}
// sky.rs:446-449 sunlit_ground.
__device__ __forceinline__ D3 sunlit_ground(const Atm& a, const float* __restrict__ sun, double mu_sun) {
    D3 t = sun_transmittance_at(sun, at_new(mu_sun, R_GROUND));
    double m = fmax(mu_sun, 0.0);
    return {a.ground_albedo[0] / PI * m * t.x, a.ground_albedo[1] / PI * m * t.y, a.ground_albedo[2] / PI * m * t.z};
}

// sky.rs:328-347 Ray.
struct Ray { double r, mu, mu_sun, nu, length; };
__device__ __forceinline__ Ray ray_new(double r, double mu, double mu_sun, double nu, bool* lands) {
    double g = 0.0;
    *lands = distance_to_ground(r, mu, &g);
    return {r, mu, mu_sun, nu, *lands ? g : distance_out(r, mu, R_TOP)};
}
__device__ __forceinline__ double mu_sun_at_ground(const Ray& ray) {
    return fmin(fmax((ray.r * ray.mu_sun + ray.length * ray.nu) / R_GROUND, -1.0), 1.0);
}

// sky.rs:494-530 Luts::march: Simpson's rule on `steps` intervals of u (t = length u^2), the view's optical depth a
// running Simpson integral (its odd nodes by the three-point half-panel rule). `emitted(at, air, haze)`.
struct Node { At at; double air, haze; D3 ext; double jacobian; };
template <class E>
__device__ __forceinline__ void march(const Atm& a, const Ray& ray, int steps, E emitted, D3* out_l, D3* out_through) {
    steps = max(steps, 2) & ~1;
    double h = 1.0 / (double)steps;
    auto node = [&](int i) {
        double u = (double)i * h;
        double t = ray.length * u * u;
        double r = sqrt(ray.r * ray.r + t * t + 2.0 * ray.r * ray.mu * t);
        double altitude = fmax(r - R_GROUND, 0.0);
        double e0 = exp1f(-altitude * (1.0 / H_RAYLEIGH)), e1 = exp1f(-altitude * (1.0 / H_MIE));
        double ozone = fmax(1.0 - fabs(altitude - OZONE_CENTRE) * (1.0 / OZONE_HALF_WIDTH), 0.0);
        double jacobian = 2.0 * ray.length * u;
        Node n;
        n.at = at_new(fmin(fmax((ray.r * ray.mu_sun + t * ray.nu) / r, -1.0), 1.0), r);
        n.air = e0;
        n.haze = e1;
        D3 x = extinction(a, e0, e1, ozone);
        n.ext = {x.x * jacobian, x.y * jacobian, x.z * jacobian};
        n.jacobian = jacobian;
        return n;
    };
    D3 out = {0, 0, 0}, depth = {0, 0, 0};
    auto add = [&](const Node& n, D3 tau, double simpson) {
        D3 e = emitted(n.at, n.air, n.haze);
        double w = simpson * h / 3.0 * n.jacobian;
        out.x += w * exp1f(-tau.x) * e.x;
        out.y += w * exp1f(-tau.y) * e.y;
        out.z += w * exp1f(-tau.z) * e.z;
    };
    Node n0 = node(0);
    for (int k = 0; k < steps; k += 2) {
        Node n1 = node(k + 1), n2 = node(k + 2);
        D3 middle = {depth.x + h / 12.0 * (5.0 * n0.ext.x + 8.0 * n1.ext.x - n2.ext.x),
                     depth.y + h / 12.0 * (5.0 * n0.ext.y + 8.0 * n1.ext.y - n2.ext.y),
                     depth.z + h / 12.0 * (5.0 * n0.ext.z + 8.0 * n1.ext.z - n2.ext.z)};
        depth = {depth.x + h / 3.0 * (n0.ext.x + 4.0 * n1.ext.x + n2.ext.x),
                 depth.y + h / 3.0 * (n0.ext.y + 4.0 * n1.ext.y + n2.ext.y),
                 depth.z + h / 3.0 * (n0.ext.z + 4.0 * n1.ext.z + n2.ext.z)};
        add(n1, middle, 4.0);
        add(n2, depth, k + 2 == steps ? 1.0 : 2.0);
        n0 = n2;
    }
    *out_l = out;
    *out_through = {exp1f(-depth.x), exp1f(-depth.y), exp1f(-depth.z)};
}

// sky.rs:457-466 Luts::directions: the j-th (mu, phi, weight) of the iterator (panel, node, sign, azimuth).
__device__ __forceinline__ void direction(double r, bool up, int j, double* mu, double* phi, double* weight) {
    int k = j % AZIMUTHS, s = (j / AZIMUTHS) % 2, g = (j / (2 * AZIMUTHS)) % 4, panel = j / (8 * AZIMUTHS);
    double lo, hi;
    if (up) {
        lo = 0.0;
        hi = 1.0;
    } else {
        double rg = R_GROUND / r;
        double horizon = -sqrt(fmax(1.0 - rg * rg, 0.0));
        lo = panel == 0 ? -1.0 : horizon;
        hi = panel == 0 ? horizon : 1.0;
    }
    double whole = up ? 1.0 : 2.0;
    double centre = 0.5 * (lo + hi), half = 0.5 * (hi - lo);
    double sign = s == 0 ? -1.0 : 1.0;
    *mu = centre + sign * half * GL8_X[g];
    *phi = ((double)k + 0.5) / (double)AZIMUTHS * PI;
    *weight = GL8_W[g] * half / whole / (double)AZIMUTHS;
}

// The source of an order's gather: order one (the sun's light scattered isotropically, the sunlit ground) or a
// table of the order before (sky.rs:405-417).
struct Source {
    const float* sun;
    const float* order;         // SC_ROWS x SC_COLS, or null: order one
    const float* order_ground;  // SC_COLS
    __device__ __forceinline__ D3 at(At p) const {
        if (!order) {
            const double iso = 1.0 / (4.0 * PI);
            D3 t = sun_transmittance_at(sun, p);
            return {t.x * iso, t.y * iso, t.z * iso};
        }
        return table_at(order, SC_COLS, SC_ROWS, p.scatter, p.altitude);
    }
    __device__ __forceinline__ D3 ground(const Atm& a, double mu_sun) const {
        if (!order) return sunlit_ground(a, sun, mu_sun);
        return table_at(order_ground, SC_COLS, 1, at_new(mu_sun, R_GROUND).scatter, 0.0);
    }
};

// One gathering direction's share of an entry (sky.rs:471-490 gather; sky.rs:493-513 gather_ground).
__device__ D3 gather_one(const Atm& a, const Source& src, double mu_sun, double r, int j, bool up) {
    double mu, phi, weight;
    direction(r, up, j, &mu, &phi, &weight);
    double sin_sun = sqrt(fmax(1.0 - mu_sun * mu_sun, 0.0));
    double nu = sqrt(fmax(1.0 - mu * mu, 0.0)) * cos(phi) * sin_sun + mu * mu_sun;
    bool lands;
    Ray ray = ray_new(up ? R_GROUND + 1e-3 : r, mu, mu_sun, nu, &lands);
    D3 l, through;
    march(a, ray, STEPS, [&](At at, double air, double haze) {
        D3 s = src.at(at);
        return D3{(a.rayleigh[0] * air + a.mie_scattering * haze) * s.x,
                  (a.rayleigh[1] * air + a.mie_scattering * haze) * s.y,
                  (a.rayleigh[2] * air + a.mie_scattering * haze) * s.z};
    }, &l, &through);
    if (up) {
        double w = weight * 2.0 * mu;
        return {w * l.x * a.ground_albedo[0], w * l.y * a.ground_albedo[1], w * l.z * a.ground_albedo[2]};
    }
    D3 below = {0, 0, 0};
    if (lands) below = src.ground(a, mu_sun_at_ground(ray));
    return {weight * (l.x + through.x * below.x), weight * (l.y + through.y * below.y),
            weight * (l.z + through.z * below.z)};
}

// The sun's optical-depth table (sky.rs:402): a thread an entry.
__global__ void k_sun_table(Atm a, float* __restrict__ sun) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= SUN_ENTRIES) return;
    double r = row_radius(i / SUN_COLS, SUN_ROWS);
    double mu = mu_of_sun((double)(i % SUN_COLS) / (double)(SUN_COLS - 1), r);
    D3 t = optical_depth(a, r, mu);
    sun[3 * i] = (float)t.x;
    sun[3 * i + 1] = (float)t.y;
    sun[3 * i + 2] = (float)t.z;
}

// One order of the scattered light: a warp an entry (blockIdx.x), a lane a direction; `up` entries are the ground's.
// Lane 0 adds the directions in the reference's order.
__global__ void k_gather(Atm a, Source src, float* __restrict__ next, int up) {
    int i = blockIdx.x, lane = threadIdx.x;
    int rows = up ? 1 : SC_ROWS;
    if (i >= SC_COLS * rows) return;
    double r = up ? R_GROUND : row_radius(i / SC_COLS, rows);
    double mu_sun = mu_of_scatter((double)(i % SC_COLS) / (double)(SC_COLS - 1));
    if (mu_sun < NIGHT) {
        if (lane < 3) next[3 * i + lane] = 0.0f;
        return;
    }
    if (!up) r = fmin(fmax(r, R_GROUND + 1e-3), R_TOP - 1e-3);
    int n = up ? DIRS_UP : DIRS;
    D3 v = {0, 0, 0};
    if (lane < n) v = gather_one(a, src, mu_sun, r, lane, up != 0);
    D3 sum = {0, 0, 0};
    for (int j = 0; j < n; ++j) {
        double x = __shfl_sync(0xffffffffu, v.x, j), y = __shfl_sync(0xffffffffu, v.y, j),
               z = __shfl_sync(0xffffffffu, v.z, j);
        sum.x += x;
        sum.y += y;
        sum.z += z;
    }
    if (lane == 0) {
        next[3 * i] = (float)sum.x;
        next[3 * i + 1] = (float)sum.y;
        next[3 * i + 2] = (float)sum.z;
    }
}

// sky.rs:418-427: the orders' sum; mode 0 starts it, 1 adds an order, 2 adds the last as a geometric series.
__global__ void k_series(float* __restrict__ sum, const float* __restrict__ before, const float* __restrict__ next,
                         int n, int mode) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mode == 0) {
        sum[i] = next[i];
        return;
    }
    float ratio = 0.0f;
    if (before[i] > 0.0f) ratio = fminf(fmaxf(next[i] / before[i], 0.0f), 0.9f);
    sum[i] += mode == 2 ? next[i] / (1.0f - ratio) : next[i];
}

// The bake's per-texel inputs.
struct Bake {
    float3 sun_dir, sun_lux, sun_p;
    float altitude_km, row, dip;
    uint32_t width, height;
    int planet;
    float3 glow_uniform, glow_horizon;
    float glow_height, cover;
};

__device__ __forceinline__ float3 glow_at(const Bake& b, float elevation) {
    if (b.glow_horizon.x == 0.0f && b.glow_horizon.y == 0.0f && b.glow_horizon.z == 0.0f) return b.glow_uniform;
    float k = expf(-fmaxf(elevation, 0.0f) / fmaxf(b.glow_height, 1e-3f));
    return make_float3(b.glow_uniform.x + b.glow_horizon.x * k, b.glow_uniform.y + b.glow_horizon.y * k,
                       b.glow_uniform.z + b.glow_horizon.z * k);
}

// sky.rs:548-602 Luts::sky: radiance per unit of the sun's illuminance (planet frame, Z up).
__device__ float3 sky_radiance(const Atm& a, const float* __restrict__ sun, const float* __restrict__ scattered,
                               const float* __restrict__ ground, float altitude_km, float3 dir, float3 sunv) {
    double r0 = R_GROUND + (double)fmaxf(altitude_km, 0.0f);
    double mu0 = fmin(fmax((double)dir.z, -1.0), 1.0);
    double mu_sun0 = fmin(fmax((double)sunv.z, -1.0), 1.0);
    double nu = fmin(fmax((double)(dir.x * sunv.x + dir.y * sunv.y + dir.z * sunv.z), -1.0), 1.0);
    double top = R_TOP - 1e-3;
    double r = r0, mu = mu0, mu_sun = mu_sun0;
    if (r0 > top) {
        double disc = r0 * r0 * (mu0 * mu0 - 1.0) + top * top;
        if (mu0 >= 0.0 || disc <= 0.0) return make_float3(0.0f, 0.0f, 0.0f);
        double t = -r0 * mu0 - sqrt(disc);
        r = sqrt(r0 * r0 + t * t + 2.0 * r0 * mu0 * t);
        mu = fmin(fmax((r0 * mu0 + t) / r, -1.0), 1.0);
        mu_sun = fmin(fmax((r0 * mu_sun0 + t * nu) / r, -1.0), 1.0);
    }
    bool lands;
    Ray ray = ray_new(r, mu, mu_sun, nu, &lands);
    double by_air = 3.0 / (16.0 * PI) * (1.0 + nu * nu);
    double g = a.mie_g;
    double by_haze = (1.0 - g * g) / (4.0 * PI * pow(fmax(1.0 + g * g - 2.0 * g * nu, 1e-9), 1.5)) * a.mie_scattering;
    D3 l, through;
    march(a, ray, VIEW_STEPS, [&](At at, double air, double haze) {
        D3 s = sun_transmittance_at(sun, at), f = table_at(scattered, SC_COLS, SC_ROWS, at.scatter, at.altitude);
        double a0 = a.rayleigh[0] * air, a1 = a.rayleigh[1] * air, a2 = a.rayleigh[2] * air;
        return D3{(a0 * by_air + haze * by_haze) * s.x + (a0 + haze * a.mie_scattering) * f.x,
                  (a1 * by_air + haze * by_haze) * s.y + (a1 + haze * a.mie_scattering) * f.y,
                  (a2 * by_air + haze * by_haze) * s.z + (a2 + haze * a.mie_scattering) * f.z};
    }, &l, &through);
    D3 below = {0, 0, 0};
    if (lands) {
        double ms = mu_sun_at_ground(ray);
        D3 direct = sunlit_ground(a, sun, ms), sc = table_at(ground, SC_COLS, 1, at_new(ms, R_GROUND).scatter, 0.0);
        below = {direct.x + sc.x, direct.y + sc.y, direct.z + sc.z};
    }
    return make_float3((float)(l.x + through.x * below.x), (float)(l.y + through.y * below.y),
                       (float)(l.z + through.z * below.z));
}

__device__ __forceinline__ float3 fnormalize(float3 v) {
    float r = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x * r, v.y * r, v.z * r);
}

// sky.rs:730-772: a texel of the bake (before the overcast blend): radiance x the sun's illuminance + glow, times
// the horizon's cover k, k in w.
__global__ void k_bake(Atm a, Bake b, const float* __restrict__ sun, const float* __restrict__ scattered,
                       const float* __restrict__ ground, float4* __restrict__ tex) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n = b.width * b.height;
    if (i >= n) return;
    float x = (float)(i % b.width) + 0.5f, y = (float)(i / b.width) + 0.5f;
    float theta = y / (float)b.height * PI_F;
    float phi = (x / (float)b.width - 0.5f) * 2.0f * PI_F;
    float st = sinf(theta), ct = cosf(theta), sp = sinf(phi), cp = cosf(phi);
    float3 d = make_float3(st * sp, ct, -st * cp);
    float4 out;
    if (b.planet) {
        float k = fminf(fmaxf((PI_F / 2.0f - theta + 0.5f * b.row - b.dip) / b.row, 0.0f), 1.0f);
        if (k <= 0.0f) {
            tex[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            return;
        }
        float e = fmaxf(PI_F / 2.0f - theta, b.dip + 1e-4f);
        float ce = cosf(e), se = sinf(e);
        float3 dir = make_float3(sp * ce + 0.0f * se, 0.0f * ce + 1.0f * se, -cp * ce + 0.0f * se);
        float3 l = sky_radiance(a, sun, scattered, ground, b.altitude_km, make_float3(dir.x, dir.z, dir.y), b.sun_p);
        float3 g = glow_at(b, e);
        out = make_float4((l.x * b.sun_lux.x + g.x) * k, (l.y * b.sun_lux.y + g.y) * k, (l.z * b.sun_lux.z + g.z) * k, k);
    } else {
        float side = fmaxf(fmaxf(fabsf(d.x), fabsf(d.z)), 1e-6f);
        float r = d.y / side * (0.5f * SKY_LIGHT_CUBE);
        if (r <= -0.5f) {
            tex[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            return;
        }
        float3 dir = d;
        float k = 1.0f;
        if (r < 0.5f) {
            dir = fnormalize(make_float3(d.x, side / SKY_LIGHT_CUBE, d.z));
            k = r + 0.5f;
        }
        float3 l = sky_radiance(a, sun, scattered, ground, b.altitude_km, make_float3(dir.x, dir.z, dir.y), b.sun_p);
        float3 g = glow_at(b, asinf(fminf(fmaxf(dir.y, -1.0f), 1.0f)));
        out = make_float4((l.x * b.sun_lux.x + g.x) * k, (l.y * b.sun_lux.y + g.y) * k, (l.z * b.sun_lux.z + g.z) * k, k);
    }
    tex[i] = out;
}

// The clear sky's horizontal illuminance (sky.rs:778-782) by blocks: each block sums its rows in a fixed order (f64).
constexpr int COVER_THREADS = 256;
__global__ void k_cover_partial(Bake b, const float4* __restrict__ tex, double* __restrict__ partial) {
    __shared__ double s[3][COVER_THREADS];
    float dt = PI_F / (float)b.height, dp = 2.0f * PI_F / (float)b.width;
    uint32_t n = b.width * b.height;
    uint32_t per = (n + gridDim.x - 1) / gridDim.x;
    uint32_t lo = blockIdx.x * per, hi = min(lo + per, n);
    double acc[3] = {0, 0, 0};
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        float theta = ((float)(i / b.width) + 0.5f) * dt;
        float k = fmaxf(cosf(theta), 0.0f) * sinf(theta) * dt * dp;
        float4 t = tex[i];
        acc[0] += (double)(t.x * k);
        acc[1] += (double)(t.y * k);
        acc[2] += (double)(t.z * k);
    }
    for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int w = COVER_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 3; ++c) s[c][threadIdx.x] += s[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) partial[3 * blockIdx.x + c] = s[c][0];
}

// The device's results (read back by the host).
struct Result {
    float sun[3];
    float horizon_v;
    float e_oc;
    uint32_t brightest_bits;
};

// sky.rs:783-796 and 802-817: the overcast dome's illuminance (from the block sums), the sun's illuminance at the
// ground, the planet's limb row. One thread.
__global__ void k_finish(Atm a, Bake b, const double* __restrict__ partial, int n_partial, Result* __restrict__ res) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float cover = fminf(fmaxf(b.cover, 0.0f), 1.0f);
    if (cover > 0.0f) {
        double es[3] = {0, 0, 0};
        for (int p = 0; p < n_partial; ++p)
            for (int c = 0; c < 3; ++c) es[c] += partial[3 * p + c];
        float dt = PI_F / (float)b.height, dp = 2.0f * PI_F / (float)b.width;
        float3 sd = fnormalize(b.sun_dir);
        float3 s0 = sun_illuminance(a, b.sun_dir, b.sun_lux, 0.0f);
        float up = fmaxf(sd.y, 0.0f);
        float3 e_sun = make_float3(s0.x * up, s0.y * up, s0.z * up);
        float3 e_glow = make_float3(0.0f, 0.0f, 0.0f);
        bool glow_zero = b.glow_uniform.x == 0.0f && b.glow_uniform.y == 0.0f && b.glow_uniform.z == 0.0f &&
                         b.glow_horizon.x == 0.0f && b.glow_horizon.y == 0.0f && b.glow_horizon.z == 0.0f;
        if (!glow_zero) {
            for (uint32_t y = 0; y < b.height; ++y) {
                float theta = ((float)y + 0.5f) * dt;
                float3 g = glow_at(b, fmaxf(PI_F / 2.0f - theta, -PI_F / 2.0f));
                float k = fmaxf(cosf(theta), 0.0f) * sinf(theta) * dt * dp * (float)b.width;
                e_glow = make_float3(e_glow.x + g.x * k, e_glow.y + g.y * k, e_glow.z + g.z * k);
            }
        }
        float tx = (float)es[0] - e_glow.x + e_sun.x, ty = (float)es[1] - e_glow.y + e_sun.y,
              tz = (float)es[2] - e_glow.z + e_sun.z;
        float lum = 0.2126f * tx + 0.7152f * ty + 0.0722f * tz;
        res->e_oc = fmaxf(lum, 0.0f) * OVERCAST_TRANSMITTANCE;
    } else {
        res->e_oc = 0.0f;
    }
    float hv = 0.0f;
    if (b.planet) {
        float rowc = ceilf((PI_F / 2.0f - b.dip) / b.row) - 1.0f;
        rowc = fminf(fmaxf(rowc, 0.0f), (float)b.height - 1.0f);
        hv = (rowc + 0.5f) / (float)b.height;
    }
    res->horizon_v = hv;
    float3 s = sun_illuminance(a, b.sun_dir, b.sun_lux, cover);
    res->sun[0] = s.x;
    res->sun[1] = s.y;
    res->sun[2] = s.z;
    res->brightest_bits = 0u;
}

// sky.rs:797-811: the overcast blend (with a cover), then the alpha (the planet's limb share, else 1).
__global__ void k_overcast(Bake b, const Result* __restrict__ res, float4* __restrict__ tex) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n = b.width * b.height;
    if (i >= n) return;
    float4 t = tex[i];
    float cover = fminf(fmaxf(b.cover, 0.0f), 1.0f);
    if (cover > 0.0f) {
        float dt = PI_F / (float)b.height;
        float e = PI_F / 2.0f - ((float)(i / b.width) + 0.5f) * dt;
        float eo = res->e_oc;
        float kk = (1.0f + 2.0f * sinf(fmaxf(e, 0.0f))) / 3.0f;
        float s = 9.0f / (7.0f * PI_F);
        float3 c = make_float3(eo * s * kk, eo * s * kk, eo * s * kk);
        float3 g = glow_at(b, fmaxf(e, -PI_F / 2.0f));
        float ox = (c.x + g.x * OVERCAST_GLOW) * t.w, oy = (c.y + g.y * OVERCAST_GLOW) * t.w,
              oz = (c.z + g.z * OVERCAST_GLOW) * t.w;
        t.x = t.x + (ox - t.x) * cover;
        t.y = t.y + (oy - t.y) * cover;
        t.z = t.z + (oz - t.z) * cover;
    }
    t.w = (b.planet && t.w > 0.0f) ? t.w : 1.0f;
    tex[i] = t;
}

// The environment's texels as RGBA16F (round to nearest even) and the brightest luminance (lib.rs:1013-1015).
__global__ void k_env_pack(const float4* __restrict__ tex, uint32_t n, ushort4* __restrict__ env,
                           Result* __restrict__ res) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float lum = 0.0f;
    if (i < n) {
        float4 t = tex[i];
        env[i] = make_ushort4(__half_as_ushort(__float2half_rn(t.x)), __half_as_ushort(__float2half_rn(t.y)),
                              __half_as_ushort(__float2half_rn(t.z)), __half_as_ushort(__float2half_rn(t.w)));
        lum = fmaxf(0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z, 0.0f);
    }
    for (int o = 16; o > 0; o >>= 1) lum = fmaxf(lum, __shfl_xor_sync(0xffffffffu, lum, o));
    if ((threadIdx.x & 31) == 0 && lum > 0.0f) atomicMax(&res->brightest_bits, __float_as_uint(lum));
}

// lib.rs:916-933: a row's conditional CDF over luminance x sin(theta), its running sum in f32 in texel order.
__global__ void k_env_rows(const float4* __restrict__ tex, uint32_t w, const float* __restrict__ sin_rows,
                           float* __restrict__ rows, float* __restrict__ cond) {
    extern __shared__ float sh[];
    uint32_t y = blockIdx.x;
    float sin_t = sin_rows[y];
    for (uint32_t x = threadIdx.x; x < w; x += blockDim.x) {
        float4 t = tex[(size_t)y * w + x];
        sh[x] = fmaxf(0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z, 0.0f) * sin_t + 1e-12f;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float acc = 0.0f;
        for (uint32_t x = 0; x < w; ++x) {
            acc += sh[x];
            sh[x] = acc;
        }
        rows[y] = acc;
    }
    __syncthreads();
    float total = rows[y];
    for (uint32_t x = threadIdx.x; x < w; x += blockDim.x) cond[(size_t)y * w + x] = sh[x] / total;
}

// lib.rs:934-940: the marginal over rows. One thread.
__global__ void k_env_marginal(const float* __restrict__ rows, uint32_t h, float* __restrict__ marg) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float total = 0.0f;
    for (uint32_t y = 0; y < h; ++y) total += rows[y];
    float acc = 0.0f;
    for (uint32_t y = 0; y < h; ++y) {
        acc += rows[y] / total;
        marg[y] = acc;
    }
}

}  // namespace trt_sky

using namespace trt_sky;

struct SkyState {
    int device = 0;
    // The tables: sun, two orders and their grounds, the sums (scattered, ground).
    float* tables = nullptr;
    float *sun = nullptr, *order[2] = {nullptr, nullptr}, *order_ground[2] = {nullptr, nullptr};
    float *scattered = nullptr, *ground = nullptr;
    bool have_tables = false;
    float key[6] = {0, 0, 0, 0, 0, 0};  // rayleigh, mie, g, ground albedo: what the tables depend on
    Atm atm{};
    Bake bake{};
    float4* tex = nullptr;
    uint32_t tex_cap = 0;
    double* partial = nullptr;
    Result* res = nullptr;
    float* rows = nullptr;
    float* sin_rows = nullptr;
    uint32_t rows_cap = 0;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
};

namespace {

constexpr int COVER_BLOCKS = 148;
constexpr size_t TABLE_FLOATS = 3 * (size_t)(SUN_ENTRIES + 4 * SC_ENTRIES + 4 * SC_COLS);

int sky_cuda(cudaError_t e, const char* what, std::string* err) {
    if (e == cudaSuccess) return TRT_OK;
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
    return TRT_ECUDA;
}
#define SKY_CUDA(call)                                      \
    do {                                                    \
        int rc_ = sky_cuda((call), #call, err);             \
        if (rc_ != TRT_OK) return rc_;                      \
    } while (0)

Atm make_atm(const trt_atmosphere& s) {
    const double RAY[3] = {5.802e-3, 13.558e-3, 33.1e-3}, OZ[3] = {0.650e-3, 1.881e-3, 0.085e-3};
    Atm a;
    double rs = (double)std::fmax(s.rayleigh_scale, 0.0f), ms = (double)std::fmax(s.mie_scale, 0.0f);
    for (int c = 0; c < 3; ++c) a.rayleigh[c] = RAY[c] * rs;
    a.mie_scattering = MIE_SCATTERING * ms;
    a.mie_extinction = MIE_SCATTERING * ms + MIE_ABSORPTION;
    for (int c = 0; c < 3; ++c) a.ozone[c] = OZ[c];
    a.mie_g = std::fmin(std::fmax((double)s.mie_g, -0.99), 0.99);
    for (int c = 0; c < 3; ++c) a.ground_albedo[c] = std::fmin(std::fmax((double)s.ground_albedo[c], 0.0), 1.0);
    return a;
}

// sky.rs:867-871: the planet's horizon elevation for a viewer altitude_km up.
float horizon_elevation(float altitude_km) {
    double r = R_GROUND, h = (double)std::fmax(altitude_km, 0.0f);
    return (float)std::asin(-std::sqrt(h * (2.0 * r + h)) / (r + h));
}

}  // namespace

int sky_bake(SkyState** stp, int device, cudaStream_t stream, const trt_atmosphere& a, float* texels_host,
             float* tables_host, trt_sky_result* out, std::string* err) {
    if (a.width < 2 || a.height < 2 || a.width > 16384 || a.height > 8192) {
        if (err) *err = "trt_sky_bake: the bake's size must be 2..16384 x 2..8192";
        return TRT_EINVAL;
    }
    SkyState* st = *stp;
    if (!st) {
        st = new SkyState;
        st->device = device;
        *stp = st;
        SKY_CUDA(cudaMalloc(&st->tables, TABLE_FLOATS * 4));
        st->sun = st->tables;
        st->order[0] = st->sun + 3 * SUN_ENTRIES;
        st->order[1] = st->order[0] + 3 * SC_ENTRIES;
        st->scattered = st->order[1] + 3 * SC_ENTRIES;
        st->order_ground[0] = st->scattered + 3 * SC_ENTRIES;
        st->order_ground[1] = st->order_ground[0] + 3 * SC_COLS;
        st->ground = st->order_ground[1] + 3 * SC_COLS;
        SKY_CUDA(cudaMalloc(&st->partial, COVER_BLOCKS * 3 * sizeof(double)));
        SKY_CUDA(cudaMalloc(&st->res, sizeof(Result)));
        for (auto& e : st->ev) SKY_CUDA(cudaEventCreate(&e));
    }
    uint32_t n = a.width * a.height;
    if (n > st->tex_cap) {
        if (st->tex) cudaFree(st->tex);
        st->tex = nullptr;
        st->tex_cap = 0;
        SKY_CUDA(cudaMalloc(&st->tex, (size_t)n * sizeof(float4)));
        st->tex_cap = n;
    }
    float key[6] = {a.rayleigh_scale, a.mie_scale, a.mie_g, a.ground_albedo[0], a.ground_albedo[1], a.ground_albedo[2]};
    bool tables = !st->have_tables || std::memcmp(key, st->key, sizeof(key)) != 0;
    Atm atm = make_atm(a);
    SKY_CUDA(cudaEventRecord(st->ev[0], stream));
    if (tables) {
        st->have_tables = false;
        k_sun_table<<<(SUN_ENTRIES + 127) / 128, 128, 0, stream>>>(atm, st->sun);
        // sky.rs:409-429: order two from the sun, then orders three and four from the order before, summed; the
        // last closed as a geometric series.
        Source first{st->sun, nullptr, nullptr};
        k_gather<<<SC_ENTRIES, 32, 0, stream>>>(atm, first, st->order[0], 0);
        k_gather<<<SC_COLS, 32, 0, stream>>>(atm, first, st->order_ground[0], 1);
        k_series<<<(3 * SC_ENTRIES + 255) / 256, 256, 0, stream>>>(st->scattered, nullptr, st->order[0], 3 * SC_ENTRIES, 0);
        k_series<<<1, 3 * SC_COLS, 0, stream>>>(st->ground, nullptr, st->order_ground[0], 3 * SC_COLS, 0);
        int cur = 0;
        for (int order = 3; order <= 4; ++order) {
            Source src{st->sun, st->order[cur], st->order_ground[cur]};
            k_gather<<<SC_ENTRIES, 32, 0, stream>>>(atm, src, st->order[cur ^ 1], 0);
            k_gather<<<SC_COLS, 32, 0, stream>>>(atm, src, st->order_ground[cur ^ 1], 1);
            int mode = order == 4 ? 2 : 1;
            k_series<<<(3 * SC_ENTRIES + 255) / 256, 256, 0, stream>>>(st->scattered, st->order[cur],
                                                                        st->order[cur ^ 1], 3 * SC_ENTRIES, mode);
            k_series<<<1, 3 * SC_COLS, 0, stream>>>(st->ground, st->order_ground[cur], st->order_ground[cur ^ 1],
                                                    3 * SC_COLS, mode);
            cur ^= 1;
        }
        SKY_CUDA(cudaGetLastError());
        std::memcpy(st->key, key, sizeof(key));
        st->have_tables = true;
    }
    SKY_CUDA(cudaEventRecord(st->ev[1], stream));
    Bake b;
    b.sun_dir = make_float3(a.sun_dir[0], a.sun_dir[1], a.sun_dir[2]);
    b.sun_lux = make_float3(a.sun_lux[0], a.sun_lux[1], a.sun_lux[2]);
    {
        // to_planet (x, z, y), normalised as glam does: times 1 / length.
        float px = a.sun_dir[0], py = a.sun_dir[2], pz = a.sun_dir[1];
        float r = 1.0f / std::sqrt(px * px + py * py + pz * pz);
        b.sun_p = make_float3(px * r, py * r, pz * r);
    }
    b.altitude_km = std::fmax(a.altitude_m / 1000.0f, 0.005f);
    b.row = PI_F / (float)a.height;
    b.dip = horizon_elevation(b.altitude_km);
    b.width = a.width;
    b.height = a.height;
    b.planet = a.planet ? 1 : 0;
    b.glow_uniform = make_float3(a.glow_uniform[0], a.glow_uniform[1], a.glow_uniform[2]);
    b.glow_horizon = make_float3(a.glow_horizon[0], a.glow_horizon[1], a.glow_horizon[2]);
    b.glow_height = a.glow_height;
    b.cover = a.cloud_cover;
    st->atm = atm;
    st->bake = b;
    k_bake<<<(n + 127) / 128, 128, 0, stream>>>(atm, b, st->sun, st->scattered, st->ground, st->tex);
    float cover = std::fmin(std::fmax(a.cloud_cover, 0.0f), 1.0f);
    if (cover > 0.0f) k_cover_partial<<<COVER_BLOCKS, COVER_THREADS, 0, stream>>>(b, st->tex, st->partial);
    k_finish<<<1, 32, 0, stream>>>(atm, b, st->partial, COVER_BLOCKS, st->res);
    k_overcast<<<(n + 255) / 256, 256, 0, stream>>>(b, st->res, st->tex);
    SKY_CUDA(cudaGetLastError());
    SKY_CUDA(cudaEventRecord(st->ev[2], stream));
    Result r;
    SKY_CUDA(cudaMemcpyAsync(&r, st->res, sizeof(Result), cudaMemcpyDeviceToHost, stream));
    if (texels_host)
        SKY_CUDA(cudaMemcpyAsync(texels_host, st->tex, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost, stream));
    if (tables_host) {
        float* o = tables_host;
        SKY_CUDA(cudaMemcpyAsync(o, st->sun, 3 * SUN_ENTRIES * 4, cudaMemcpyDeviceToHost, stream));
        SKY_CUDA(cudaMemcpyAsync(o + 3 * SUN_ENTRIES, st->scattered, 3 * SC_ENTRIES * 4, cudaMemcpyDeviceToHost, stream));
        SKY_CUDA(cudaMemcpyAsync(o + 3 * (SUN_ENTRIES + SC_ENTRIES), st->ground, 3 * SC_COLS * 4,
                                 cudaMemcpyDeviceToHost, stream));
    }
    SKY_CUDA(cudaStreamSynchronize(stream));
    if (out) {
        for (int c = 0; c < 3; ++c) out->sun_illuminance[c] = r.sun[c];
        out->horizon_v = r.horizon_v;
        out->brightest = 0.0f;
        float t_ms = 0.0f, b_ms = 0.0f;
        cudaEventElapsedTime(&t_ms, st->ev[0], st->ev[1]);
        cudaEventElapsedTime(&b_ms, st->ev[1], st->ev[2]);
        out->tables_ms = tables ? t_ms : 0.0f;
        out->bake_ms = b_ms;
    }
    return TRT_OK;
}

int sky_env(SkyState* st, cudaStream_t stream, const float* sin_rows_host, void* env, float* cdf, trt_sky_result* out,
            std::string* err) {
    if (!st || !st->tex) {
        if (err) *err = "sky_env: nothing baked";
        return TRT_EINVAL;
    }
    uint32_t w = st->bake.width, h = st->bake.height, n = w * h;
    if (h > st->rows_cap) {
        if (st->rows) cudaFree(st->rows);
        st->rows = nullptr;
        st->rows_cap = 0;
        SKY_CUDA(cudaMalloc(&st->rows, 2 * (size_t)h * 4));
        st->sin_rows = st->rows + h;
        st->rows_cap = h;
    }
    if (w * 4 > 48 * 1024) {
        if (err) *err = "sky_env: rows wider than 12288 texels";
        return TRT_EINVAL;
    }
    SKY_CUDA(cudaMemcpyAsync(st->sin_rows, sin_rows_host, (size_t)h * 4, cudaMemcpyHostToDevice, stream));
    SKY_CUDA(cudaEventRecord(st->ev[1], stream));
    SKY_CUDA(cudaMemsetAsync(&st->res->brightest_bits, 0, 4, stream));
    k_env_pack<<<(n + 255) / 256, 256, 0, stream>>>(st->tex, n, (ushort4*)env, st->res);
    k_env_rows<<<h, 256, w * 4, stream>>>(st->tex, w, st->sin_rows, st->rows, cdf + h);
    k_env_marginal<<<1, 32, 0, stream>>>(st->rows, h, cdf);
    SKY_CUDA(cudaGetLastError());
    SKY_CUDA(cudaEventRecord(st->ev[2], stream));
    Result r;
    SKY_CUDA(cudaMemcpyAsync(&r, st->res, sizeof(Result), cudaMemcpyDeviceToHost, stream));
    SKY_CUDA(cudaStreamSynchronize(stream));
    if (out) {
        uint32_t bits = r.brightest_bits;
        float f;
        std::memcpy(&f, &bits, 4);
        out->brightest = f;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, st->ev[1], st->ev[2]);
        out->bake_ms += ms;
    }
    return TRT_OK;
}

const float4* sky_texels(const SkyState* st) { return st ? st->tex : nullptr; }

void sky_free(SkyState* st) {
    if (!st) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(st->device);
    if (st->tables) cudaFree(st->tables);
    if (st->tex) cudaFree(st->tex);
    if (st->partial) cudaFree(st->partial);
    if (st->res) cudaFree(st->res);
    if (st->rows) cudaFree(st->rows);
    for (auto& e : st->ev)
        if (e) cudaEventDestroy(e);
    cudaSetDevice(prev);
    delete st;
}
