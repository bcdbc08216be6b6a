// Test infrastructure, not product code: the CPU oracle of the atmosphere's sky bake.
//
// A statement-for-statement restatement of renderer/src/sky.rs's physical sky (the medium, its optical-depth and
// multiple-scattering tables, the view march and the equirectangular bake), in double precision where the reference
// computes in f64 and in single where it computes in f32, so that the device bake (threert_b200/csrc/sky.cu) can be
// held to it. Pinned by the reference's own known answers (tests/test_sky.py): the sun-transmittance table of
// sky.rs:1317-1330, the closed-form columns of 1228-1251, the fast exponential's bounds of 1211-1225, the
// table-against-quadrature bound of 1254-1275 and the physical checks of 1344-1411.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// sky.rs:27-70: the planet, the medium's constants, the soft ground and the sun's veil (km, per km).
const double R_GROUND = 6360.0, R_TOP = 6460.0;
const double H_RAYLEIGH = 8.0, H_MIE = 1.2;
const double RAYLEIGH_SCATTERING[3] = {5.802e-3, 13.558e-3, 33.1e-3};
const double MIE_SCATTERING = 3.996e-3, MIE_ABSORPTION = 0.444e-3;
const double OZONE_ABSORPTION[3] = {0.650e-3, 1.881e-3, 0.085e-3};
const double OZONE_CENTRE = 25.0, OZONE_HALF_WIDTH = 15.0;
const double SOFT_GROUND = 5.0, R_BASE = R_GROUND - SOFT_GROUND;
const double SUN_VEIL_COLUMN = 1.65, SUN_VEIL_ALTITUDE = 55.0;
const double OPAQUE = 80.0;  // sky.rs:236
const double NIGHT = -0.3;   // sky.rs:372
const double PI = 3.14159265358979323846;
const float PI_F = 3.14159265358979323846f;
const int SUN_COLS = 257, SUN_ROWS = 128, SC_COLS = 64, SC_ROWS = 32;  // sky.rs:367-368
const int ORDERS = 3, AZIMUTHS = 2, STEPS = 12, VIEW_STEPS = 16;       // sky.rs:362 QUALITY
const float SKY_LIGHT_CUBE = 128.0f;                                    // sky.rs:637
const float OVERCAST_TRANSMITTANCE = 0.3f, OVERCAST_GLOW = 3.0f;        // sky.rs:706, 710

struct D3 { double v[3]; };
struct F3 { float x, y, z; };

F3 f3(float x, float y, float z) { return {x, y, z}; }
float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// glam Vec3::normalize: self * (1 / length).
F3 fnormalize(F3 a) {
    float r = 1.0f / std::sqrt(fdot(a, a));
    return {a.x * r, a.y * r, a.z * r};
}

// sky.rs:72-81, 170-185 Atmosphere::earth.
struct Atm {
    double rayleigh[3], mie_scattering, mie_extinction, ozone[3], mie_g, ground_albedo[3];
};

Atm earth(float rayleigh_scale, float mie_scale, float mie_g, const float ground[3]) {
    Atm a;
    double rs = (double)std::max(rayleigh_scale, 0.0f), ms = (double)std::max(mie_scale, 0.0f);
    for (int c = 0; c < 3; ++c) a.rayleigh[c] = RAYLEIGH_SCATTERING[c] * rs;
    a.mie_scattering = MIE_SCATTERING * ms;
    a.mie_extinction = MIE_SCATTERING * ms + MIE_ABSORPTION;
    for (int c = 0; c < 3; ++c) a.ozone[c] = OZONE_ABSORPTION[c];
    a.mie_g = std::min(std::max((double)mie_g, -0.99), 0.99);
    for (int c = 0; c < 3; ++c) a.ground_albedo[c] = std::min(std::max((double)ground[c], 0.0), 1.0);
    return a;
}

// sky.rs:55-58.
double ground_depth(double p) {
    double d = std::max((R_GROUND - p) / 2.0, 0.0);
    return d * d * d * d;
}

// sky.rs:84-86.
D3 densities(double h) {
    return {{std::exp(-h / H_RAYLEIGH), std::exp(-h / H_MIE),
             std::max(1.0 - std::fabs(h - OZONE_CENTRE) / OZONE_HALF_WIDTH, 0.0)}};
}

// sky.rs:93-105: e^x in single precision, by x = k ln 2 + r and a degree-7 Taylor polynomial of e^r.
void exp4(const double x[4], double out[4]) {
    for (int i = 0; i < 4; ++i) {
        float v = (float)x[i];
        v = v < -87.0f ? -87.0f : (v > 88.0f ? 88.0f : v);
        float k = std::floor(v * 1.44269504088896340736f + 0.5f);
        float r = (v - k * 0.69314575f) - k * 1.4286068e-6f;
        float poly = 1.0f + r * (1.0f + r * (0.5f + r * (1.0f / 6.0f + r * (1.0f / 24.0f + r * (1.0f / 120.0f +
                     r * (1.0f / 720.0f + r * (1.0f / 5040.0f)))))));
        uint32_t bits = ((uint32_t)((int32_t)k + 127)) << 23;
        float scale;
        std::memcpy(&scale, &bits, 4);
        out[i] = (double)(poly * scale);
    }
}

// sky.rs:107-115.
double distance_out(double r, double mu, double to) {
    return -r * mu + std::sqrt(std::max(r * r * (mu * mu - 1.0) + to * to, 0.0));
}
bool distance_to_ground(double r, double mu, double* d) {
    double disc = r * r * (mu * mu - 1.0) + R_GROUND * R_GROUND;
    if (!(mu < 0.0 && disc >= 0.0)) return false;
    *d = std::max(-r * mu - std::sqrt(disc), 0.0);
    return true;
}

// sky.rs:118-123 (Abramowitz & Stegun Table 25.4, the positive half).
const double GL8_X[4] = {0.1834346424956498, 0.525532409916329, 0.7966664774136267, 0.9602898564975362};
const double GL8_W[4] = {0.362683783378362, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};

// sky.rs:128-151.
D3 columns_exact(double r, double mu) {
    const int PANELS = 12;
    double d = distance_out(r, mu, R_TOP);
    D3 n = {{0, 0, 0}};
    for (int p = 0; p < PANELS; ++p) {
        double centre = ((double)p + 0.5) / (double)PANELS, half = 0.5 / (double)PANELS;
        for (int g = 0; g < 4; ++g) {
            for (double s : {-1.0, 1.0}) {
                double u = centre + s * half * GL8_X[g];
                double t = d * u * u;
                D3 dens = densities(std::sqrt(r * r + t * t + 2.0 * r * mu * t) - R_GROUND);
                double k = GL8_W[g] * half * 2.0 * d * u;
                for (int c = 0; c < 3; ++c) n.v[c] += k * dens.v[c];
            }
        }
    }
    return n;
}

// sky.rs:158-168: false where the ray is deeper than the soft ground.
bool slant(double r, double mu, D3* cols, double* ground) {
    if (mu >= 0.0) {
        *cols = columns_exact(r, mu);
        *ground = 0.0;
        return true;
    }
    double p = r * std::sqrt(std::max(1.0 - mu * mu, 0.0));
    if (p <= R_BASE) return false;
    D3 level = columns_exact(p, 0.0), mirror = columns_exact(r, -mu);
    for (int c = 0; c < 3; ++c) cols->v[c] = std::max(2.0 * level.v[c] - mirror.v[c], 0.0);
    *ground = ground_depth(p);
    return true;
}

// sky.rs:187-191.
D3 extinction(const Atm& a, D3 dens) {
    D3 e;
    for (int c = 0; c < 3; ++c)
        e.v[c] = a.rayleigh[c] * dens.v[0] + a.mie_extinction * dens.v[1] + a.ozone[c] * dens.v[2];
    return e;
}

// sky.rs:195-200.
D3 optical_depth(const Atm& a, double r, double mu) {
    D3 n;
    double ground;
    if (!slant(r, mu, &n, &ground)) return {{OPAQUE, OPAQUE, OPAQUE}};
    D3 e = extinction(a, n);
    for (int c = 0; c < 3; ++c) e.v[c] = std::min(e.v[c] + ground, OPAQUE);
    return e;
}

// sky.rs:203-220.
F3 sun_transmittance(const Atm& a, F3 dir) {
    // glam normalize_or_zero: the zero vector where 1 / length is not a finite positive number.
    float len = std::sqrt(fdot(dir, dir));
    float rcp = 1.0f / len;
    float y = (std::isfinite(rcp) && rcp > 0.0f) ? dir.y * rcp : 0.0f;
    double mu = std::min(std::max((double)y, -1.0), 1.0);
    D3 od = optical_depth(a, R_GROUND, mu);
    double level = R_GROUND / (R_GROUND + SUN_VEIL_ALTITUDE);
    double veil = SUN_VEIL_COLUMN / std::sqrt(1.0 - level * level * (1.0 - mu * mu));
    float out[3];
    for (int c = 0; c < 3; ++c)
        out[c] = (float)(std::exp(-od.v[c]) * std::exp(-veil * (a.rayleigh[c] + a.mie_extinction)));
    return {out[0], out[1], out[2]};
}

// sky.rs:224-235.
double phase_rayleigh(double nu) { return 3.0 / (16.0 * PI) * (1.0 + nu * nu); }
double phase_mie(const Atm& a, double nu) {
    double g = a.mie_g;
    return (1.0 - g * g) / (4.0 * PI * std::pow(std::max(1.0 + g * g - 2.0 * g * nu, 1e-9), 1.5));
}

// sky.rs:248-284 At.
struct At { double sun, scatter, altitude; };
At at_new(double mu_sun, double r) {
    double root = std::sqrt(std::fabs(mu_sun));
    double altitude = std::sqrt(std::min(std::max((r - R_GROUND) * (1.0 / (R_TOP - R_GROUND)), 0.0), 1.0));
    if (mu_sun >= 0.0) return {0.5 + 0.5 * root, 0.5 + 0.5 * root, altitude};
    double under = r * mu_sun * mu_sun / (1.0 + std::sqrt(std::max(1.0 - mu_sun * mu_sun, 0.0)));
    return {0.5 - 0.5 * std::sqrt(std::min(under / (r - R_BASE), 1.0)), 0.5 - 0.5 * root, altitude};
}
At at_ground(double mu_sun) { return at_new(mu_sun, R_GROUND); }
double mu_of_scatter(double x, double) {
    double s = 2.0 * x - 1.0;
    return s * std::fabs(s);
}
double mu_of_sun(double x, double r) {
    if (x >= 0.5) {
        double q = 2.0 * x - 1.0;
        return q * q;
    }
    double q = 1.0 - 2.0 * x;
    double p = r - (r - R_BASE) * (q * q);
    double pr = p / r;
    return -std::sqrt(std::max(1.0 - pr * pr, 0.0));
}

// sky.rs:286-326 Table.
struct Table {
    int columns = 0, rows = 0;
    std::vector<float> data;  // 3 a entry
    D3 at(double column, double altitude) const {
        double fu = column * (double)(columns - 1);
        int iu = std::min(fu > 0.0 ? (int)fu : 0, columns - 2);
        float wu = (float)(fu - (double)iu);
        auto row = [&](int v, float out[3]) {
            const float* p = &data[3 * ((size_t)v * columns + iu)];
            const float* q = p + 3;
            for (int c = 0; c < 3; ++c) out[c] = p[c] + (q[c] - p[c]) * wu;
        };
        D3 r;
        if (rows == 1) {
            float o[3];
            row(0, o);
            for (int c = 0; c < 3; ++c) r.v[c] = (double)o[c];
            return r;
        }
        double fv = altitude * (double)(rows - 1);
        int iv = std::min(fv > 0.0 ? (int)fv : 0, rows - 2);
        float lo[3], hi[3];
        row(iv, lo);
        row(iv + 1, hi);
        float wv = (float)(fv - (double)iv);
        for (int c = 0; c < 3; ++c) r.v[c] = (double)(lo[c] + (hi[c] - lo[c]) * wv);
        return r;
    }
};

template <class F>
Table fill(int columns, int rows, double (*mu_of)(double, double), F f) {
    Table t;
    t.columns = columns;
    t.rows = rows;
    t.data.assign((size_t)columns * rows * 3, 0.0f);
    int n = columns * rows;
    int threads = std::max(1, std::min((int)std::thread::hardware_concurrency(), 32));
    std::vector<std::thread> pool;
    for (int w = 0; w < threads; ++w) {
        pool.emplace_back([&, w] {
            for (int i = w; i < n; i += threads) {
                double q = rows > 1 ? (double)(i / columns) / (double)(rows - 1) : 0.0;
                double r = R_GROUND + q * q * (R_TOP - R_GROUND);
                D3 v = f(mu_of((double)(i % columns) / (double)(columns - 1), r), r);
                for (int c = 0; c < 3; ++c) t.data[3 * (size_t)i + c] = (float)v.v[c];
            }
        });
    }
    for (auto& th : pool) th.join();
    return t;
}

// sky.rs:328-347 Ray.
struct Ray { double r, mu, mu_sun, nu, length; };
Ray ray_new(double r, double mu, double mu_sun, double nu, bool* lands) {
    double g;
    *lands = distance_to_ground(r, mu, &g);
    return {r, mu, mu_sun, nu, *lands ? g : distance_out(r, mu, R_TOP)};
}
double mu_sun_at_ground(const Ray& ray) {
    return std::min(std::max((ray.r * ray.mu_sun + ray.length * ray.nu) / R_GROUND, -1.0), 1.0);
}

// sky.rs:494-530 Luts::march.
struct Node { At at; double air, haze; D3 ext; double jacobian; };
template <class E>
void march(const Atm& a, const Ray& ray, int steps, E emitted, D3* out_l, D3* out_through) {
    steps = std::max(steps, 2) & ~1;
    double h = 1.0 / (double)steps;
    auto node = [&](int i) {
        double u = (double)i * h;
        double t = ray.length * u * u;
        double r = std::sqrt(ray.r * ray.r + t * t + 2.0 * ray.r * ray.mu * t);
        double altitude = std::max(r - R_GROUND, 0.0);
        double x[4] = {-altitude * (1.0 / H_RAYLEIGH), -altitude * (1.0 / H_MIE), 0.0, 0.0}, e[4];
        exp4(x, e);
        double ozone = std::max(1.0 - std::fabs(altitude - OZONE_CENTRE) * (1.0 / OZONE_HALF_WIDTH), 0.0);
        double jacobian = 2.0 * ray.length * u;
        Node n;
        n.at = at_new(std::min(std::max((ray.r * ray.mu_sun + t * ray.nu) / r, -1.0), 1.0), r);
        n.air = e[0];
        n.haze = e[1];
        n.ext = extinction(a, {{e[0], e[1], ozone}});
        for (int c = 0; c < 3; ++c) n.ext.v[c] = n.ext.v[c] * jacobian;
        n.jacobian = jacobian;
        return n;
    };
    D3 out = {{0, 0, 0}}, depth = {{0, 0, 0}};
    auto add = [&](const Node& n, D3 tau, double simpson) {
        D3 e = emitted(n.at, n.air, n.haze);
        double x[4] = {-tau.v[0], -tau.v[1], -tau.v[2], 0.0}, view[4];
        exp4(x, view);
        for (int c = 0; c < 3; ++c) out.v[c] += simpson * h / 3.0 * n.jacobian * view[c] * e.v[c];
    };
    Node n0 = node(0);
    for (int k = 0; k < steps; k += 2) {
        Node n1 = node(k + 1), n2 = node(k + 2);
        D3 middle;
        for (int c = 0; c < 3; ++c)
            middle.v[c] = depth.v[c] + h / 12.0 * (5.0 * n0.ext.v[c] + 8.0 * n1.ext.v[c] - n2.ext.v[c]);
        for (int c = 0; c < 3; ++c) depth.v[c] = depth.v[c] + h / 3.0 * (n0.ext.v[c] + 4.0 * n1.ext.v[c] + n2.ext.v[c]);
        add(n1, middle, 4.0);
        add(n2, depth, k + 2 == steps ? 1.0 : 2.0);
        n0 = n2;
    }
    double x[4] = {-depth.v[0], -depth.v[1], -depth.v[2], 0.0}, th[4];
    exp4(x, th);
    *out_l = out;
    *out_through = {{th[0], th[1], th[2]}};
}

// sky.rs:457-466 Luts::directions: (mu, phi, weight) in the iterator's order.
struct Dir { double mu, phi, weight; };
std::vector<Dir> directions(double r, bool up, int azimuths) {
    double rg = R_GROUND / r;
    double horizon = -std::sqrt(std::max(1.0 - rg * rg, 0.0));
    double panels[2][2] = {{-1.0, horizon}, {horizon, 1.0}};
    if (up) {
        panels[0][0] = 0.0; panels[0][1] = 1.0;
        panels[1][0] = 0.0; panels[1][1] = 0.0;
    }
    double whole = up ? 1.0 : 2.0;
    std::vector<Dir> out;
    for (auto& pn : panels) {
        double lo = pn[0], hi = pn[1];
        if (!(hi > lo)) continue;
        double centre = 0.5 * (lo + hi), half = 0.5 * (hi - lo);
        for (int g = 0; g < 4; ++g)
            for (double sign : {-1.0, 1.0})
                for (int k = 0; k < azimuths; ++k)
                    out.push_back({centre + sign * half * GL8_X[g], ((double)k + 0.5) / (double)azimuths * PI,
                                   GL8_W[g] * half / whole / (double)azimuths});
    }
    return out;
}

// sky.rs:374-603 Luts.
struct Luts {
    Table sun, scattered, ground;
    int view_steps = VIEW_STEPS;

    // sky.rs:436-442.
    D3 sun_transmittance_at(At at) const {
        D3 t = sun.at(at.sun, at.altitude);
        double x[4] = {-t.v[0], -t.v[1], -t.v[2], 0.0}, e[4];
        exp4(x, e);
        D3 r;
        for (int c = 0; c < 3; ++c) r.v[c] = t.v[c] < OPAQUE - 1.0 ? e[c] : 0.0;
        return r;
    }
    // sky.rs:446-449.
    D3 sunlit_ground(const Atm& a, double mu_sun) const {
        D3 t = sun_transmittance_at(at_ground(mu_sun));
        D3 r;
        for (int c = 0; c < 3; ++c) r.v[c] = a.ground_albedo[c] / PI * std::max(mu_sun, 0.0) * t.v[c];
        return r;
    }

    // sky.rs:471-490 gather.
    template <class S, class G>
    Table gather(const Atm& a, S source, G ground_of) const {
        return fill(SC_COLS, SC_ROWS, mu_of_scatter, [&](double mu_sun, double r) -> D3 {
            if (mu_sun < NIGHT) return {{0, 0, 0}};
            r = std::min(std::max(r, R_GROUND + 1e-3), R_TOP - 1e-3);
            double sin_sun = std::sqrt(std::max(1.0 - mu_sun * mu_sun, 0.0));
            D3 sum = {{0, 0, 0}};
            for (const Dir& d : directions(r, false, AZIMUTHS)) {
                double nu = std::sqrt(std::max(1.0 - d.mu * d.mu, 0.0)) * std::cos(d.phi) * sin_sun + d.mu * mu_sun;
                bool lands;
                Ray ray = ray_new(r, d.mu, mu_sun, nu, &lands);
                D3 l, through;
                march(a, ray, STEPS, [&](At at, double air, double haze) {
                    D3 s = source(at), e;
                    for (int c = 0; c < 3; ++c) e.v[c] = (a.rayleigh[c] * air + a.mie_scattering * haze) * s.v[c];
                    return e;
                }, &l, &through);
                D3 below = {{0, 0, 0}};
                if (lands) below = ground_of(mu_sun_at_ground(ray));
                for (int c = 0; c < 3; ++c) sum.v[c] += d.weight * (l.v[c] + through.v[c] * below.v[c]);
            }
            return sum;
        });
    }

    // sky.rs:493-513 gather_ground.
    template <class S>
    Table gather_ground(const Atm& a, S source) const {
        return fill(SC_COLS, 1, mu_of_scatter, [&](double mu_sun, double) -> D3 {
            if (mu_sun < NIGHT) return {{0, 0, 0}};
            double sin_sun = std::sqrt(std::max(1.0 - mu_sun * mu_sun, 0.0));
            D3 sum = {{0, 0, 0}};
            for (const Dir& d : directions(R_GROUND, true, AZIMUTHS)) {
                double nu = std::sqrt(std::max(1.0 - d.mu * d.mu, 0.0)) * std::cos(d.phi) * sin_sun + d.mu * mu_sun;
                bool lands;
                Ray ray = ray_new(R_GROUND + 1e-3, d.mu, mu_sun, nu, &lands);
                D3 l, through;
                march(a, ray, STEPS, [&](At at, double air, double haze) {
                    D3 s = source(at), e;
                    for (int c = 0; c < 3; ++c) e.v[c] = (a.rayleigh[c] * air + a.mie_scattering * haze) * s.v[c];
                    return e;
                }, &l, &through);
                for (int c = 0; c < 3; ++c) sum.v[c] += d.weight * 2.0 * d.mu * l.v[c] * a.ground_albedo[c];
            }
            return sum;
        });
    }

    // sky.rs:401-433 build_at with QUALITY.
    void build(const Atm& a) {
        sun = fill(SUN_COLS, SUN_ROWS, mu_of_sun, [&](double mu_sun, double r) { return optical_depth(a, r, mu_sun); });
        const double isotropic = 1.0 / (4.0 * PI);
        auto first = [&](At at) {
            D3 t = sun_transmittance_at(at);
            for (int c = 0; c < 3; ++c) t.v[c] = t.v[c] * isotropic;
            return t;
        };
        auto first_ground = [&](double mu_sun) { return sunlit_ground(a, mu_sun); };
        Table order = gather(a, first, first_ground), order_ground = gather_ground(a, first);
        std::vector<float> sum = order.data, sum_ground = order_ground.data;
        int last_n = std::max(ORDERS, 2) + 1;
        for (int n = 3; n <= last_n; ++n) {
            auto source = [&](At at) { return order.at(at.scatter, at.altitude); };
            auto ground_of = [&](double mu_sun) { return order_ground.at(at_ground(mu_sun).scatter, 0.0); };
            Table next = gather(a, source, ground_of), next_ground = gather_ground(a, source);
            bool last = n == last_n;
            auto add = [&](std::vector<float>& s, const std::vector<float>& before, const std::vector<float>& nx) {
                for (size_t i = 0; i < s.size(); ++i) {
                    float ratio = 0.0f;
                    if (before[i] > 0.0f) ratio = std::min(std::max(nx[i] / before[i], 0.0f), 0.9f);
                    s[i] += last ? nx[i] / (1.0f - ratio) : nx[i];
                }
            };
            add(sum, order.data, next.data);
            add(sum_ground, order_ground.data, next_ground.data);
            order = next;
            order_ground = next_ground;
        }
        scattered = order;
        scattered.data = sum;
        ground = order_ground;
        ground.data = sum_ground;
    }

    // sky.rs:548-602 sky.
    F3 sky(const Atm& a, float altitude_km, F3 dir, F3 sunv) const {
        double r0 = R_GROUND + (double)std::max(altitude_km, 0.0f);
        double mu0 = std::min(std::max((double)dir.z, -1.0), 1.0);
        double mu_sun0 = std::min(std::max((double)sunv.z, -1.0), 1.0);
        double nu = std::min(std::max((double)fdot(dir, sunv), -1.0), 1.0);
        double top = R_TOP - 1e-3;
        double r, mu, mu_sun;
        if (r0 <= top) {
            r = r0; mu = mu0; mu_sun = mu_sun0;
        } else {
            double disc = r0 * r0 * (mu0 * mu0 - 1.0) + top * top;
            if (mu0 >= 0.0 || disc <= 0.0) return f3(0, 0, 0);
            double t = -r0 * mu0 - std::sqrt(disc);
            r = std::sqrt(r0 * r0 + t * t + 2.0 * r0 * mu0 * t);
            mu = std::min(std::max((r0 * mu0 + t) / r, -1.0), 1.0);
            mu_sun = std::min(std::max((r0 * mu_sun0 + t * nu) / r, -1.0), 1.0);
        }
        bool lands;
        Ray ray = ray_new(r, mu, mu_sun, nu, &lands);
        double by_air = phase_rayleigh(nu), by_haze = phase_mie(a, nu) * a.mie_scattering;
        D3 l, through;
        march(a, ray, view_steps, [&](At at, double air, double haze) {
            D3 s = sun_transmittance_at(at), further = scattered.at(at.scatter, at.altitude), e;
            for (int c = 0; c < 3; ++c) {
                double air_c = a.rayleigh[c] * air;
                e.v[c] = (air_c * by_air + haze * by_haze) * s.v[c] + (air_c + haze * a.mie_scattering) * further.v[c];
            }
            return e;
        }, &l, &through);
        D3 below = {{0, 0, 0}};
        if (lands) {
            double ms = mu_sun_at_ground(ray);
            D3 direct = sunlit_ground(a, ms), sc = ground.at(at_ground(ms).scatter, 0.0);
            for (int c = 0; c < 3; ++c) below.v[c] = direct.v[c] + sc.v[c];
        }
        float o[3];
        for (int c = 0; c < 3; ++c) o[c] = (float)(l.v[c] + through.v[c] * below.v[c]);
        return {o[0], o[1], o[2]};
    }
};

// sky.rs:867-871.
float horizon_elevation(float altitude_km) {
    double r = R_GROUND, h = (double)std::max(altitude_km, 0.0f);
    return (float)std::asin(-std::sqrt(h * (2.0 * r + h)) / (r + h));
}

// sky.rs:661-686 Glow.
struct Glow {
    F3 uniform, horizon;
    float height;
    bool horizon_zero() const { return horizon.x == 0.0f && horizon.y == 0.0f && horizon.z == 0.0f; }
    bool is_zero() const { return uniform.x == 0.0f && uniform.y == 0.0f && uniform.z == 0.0f && horizon_zero(); }
    F3 at(float elevation) const {
        if (horizon_zero()) return uniform;
        float k = std::exp(-std::max(elevation, 0.0f) / std::max(height, 1e-3f));
        return {uniform.x + horizon.x * k, uniform.y + horizon.y * k, uniform.z + horizon.z * k};
    }
};

// sky.rs:694-703, 714-716.
F3 sun_illuminance(const Atm& a, F3 sun_dir, F3 sun_lux, float cover) {
    F3 t = sun_transmittance(a, sun_dir);
    float cloud = 1.0f - std::min(std::max(cover, 0.0f), 1.0f);
    return {sun_lux.x * t.x * cloud, sun_lux.y * t.y * cloud, sun_lux.z * t.z * cloud};
}
F3 cie_overcast(F3 e_h, float e) {
    float k = (1.0f + 2.0f * std::sin(std::max(e, 0.0f))) / 3.0f;
    float s = 9.0f / (7.0f * PI_F);
    return {e_h.x * s * k, e_h.y * s * k, e_h.z * s * k};
}

struct Handle { Atm a; Luts luts; };

// sky.rs:722-819 bake_atmosphere_with.
void bake_with(const Handle& H, F3 sun_dir, F3 sun_lux, float altitude_m, uint32_t width, uint32_t height, Glow glow,
               float cover, bool planet, float* texels, float sun_out[3], float* horizon_v_out) {
    const Atm& a = H.a;
    auto to_planet = [](F3 d) { return f3(d.x, d.z, d.y); };
    F3 sun_p = fnormalize(to_planet(sun_dir));
    float altitude_km = std::max(altitude_m / 1000.0f, 0.005f);
    float row = PI_F / (float)height;
    float dip = horizon_elevation(altitude_km);
    size_t n = (size_t)width * height;
    int threads = std::max(1, std::min((int)std::thread::hardware_concurrency(), 32));
    std::vector<std::thread> pool;
    for (int w = 0; w < threads; ++w) {
        pool.emplace_back([&, w] {
            for (size_t i = w; i < n; i += threads) {
                float* t = texels + 4 * i;
                float x = (float)(uint32_t)(i % width) + 0.5f, y = (float)(uint32_t)(i / width) + 0.5f;
                float theta = y / (float)height * PI_F;
                float phi = (x / (float)width - 0.5f) * 2.0f * PI_F;
                F3 d = f3(std::sin(theta) * std::sin(phi), std::cos(theta), -std::sin(theta) * std::cos(phi));
                if (planet) {
                    float k = std::min(std::max((PI_F / 2.0f - theta + 0.5f * row - dip) / row, 0.0f), 1.0f);
                    if (k <= 0.0f) { t[0] = t[1] = t[2] = t[3] = 0.0f; continue; }
                    float e = std::max(PI_F / 2.0f - theta, dip + 1e-4f);
                    F3 flat = f3(std::sin(phi), 0.0f, -std::cos(phi));
                    float ce = std::cos(e), se = std::sin(e);
                    F3 dir = f3(flat.x * ce + 0.0f * se, flat.y * ce + 1.0f * se, flat.z * ce + 0.0f * se);
                    F3 l = H.luts.sky(a, altitude_km, to_planet(dir), sun_p);
                    F3 g = glow.at(e);
                    t[0] = (l.x * sun_lux.x + g.x) * k; t[1] = (l.y * sun_lux.y + g.y) * k;
                    t[2] = (l.z * sun_lux.z + g.z) * k; t[3] = k;
                    continue;
                }
                float side = std::max(std::max(std::fabs(d.x), std::fabs(d.z)), 1e-6f);
                float r = d.y / side * (0.5f * SKY_LIGHT_CUBE);
                if (r <= -0.5f) { t[0] = t[1] = t[2] = t[3] = 0.0f; continue; }
                F3 dir = d;
                float k = 1.0f;
                if (r < 0.5f) { dir = fnormalize(f3(d.x, side / SKY_LIGHT_CUBE, d.z)); k = r + 0.5f; }
                F3 l = H.luts.sky(a, altitude_km, to_planet(dir), sun_p);
                F3 g = glow.at(std::asin(std::min(std::max(dir.y, -1.0f), 1.0f)));
                t[0] = (l.x * sun_lux.x + g.x) * k; t[1] = (l.y * sun_lux.y + g.y) * k;
                t[2] = (l.z * sun_lux.z + g.z) * k; t[3] = k;
            }
        });
    }
    for (auto& th : pool) th.join();
    cover = std::min(std::max(cover, 0.0f), 1.0f);
    if (cover > 0.0f) {
        float dt = PI_F / (float)height, dp = 2.0f * PI_F / (float)width;
        F3 e_sky = f3(0, 0, 0);
        for (size_t i = 0; i < n; ++i) {
            float theta = ((float)(uint32_t)(i / width) + 0.5f) * dt;
            float k = std::max(std::cos(theta), 0.0f) * std::sin(theta) * dt * dp;
            e_sky = f3(e_sky.x + texels[4 * i] * k, e_sky.y + texels[4 * i + 1] * k, e_sky.z + texels[4 * i + 2] * k);
        }
        F3 sd = fnormalize(sun_dir);
        F3 s0 = sun_illuminance(a, sun_dir, sun_lux, 0.0f);
        float up = std::max(sd.y, 0.0f);
        F3 e_sun = f3(s0.x * up, s0.y * up, s0.z * up);
        F3 e_glow = f3(0, 0, 0);
        if (!glow.is_zero()) {
            for (uint32_t yy = 0; yy < height; ++yy) {
                float theta = ((float)yy + 0.5f) * dt;
                F3 g = glow.at(std::max(PI_F / 2.0f - theta, -PI_F / 2.0f));
                float k = std::max(std::cos(theta), 0.0f) * std::sin(theta) * dt * dp * (float)width;
                e_glow = f3(e_glow.x + g.x * k, e_glow.y + g.y * k, e_glow.z + g.z * k);
            }
        }
        F3 tot = f3(e_sky.x - e_glow.x + e_sun.x, e_sky.y - e_glow.y + e_sun.y, e_sky.z - e_glow.z + e_sun.z);
        float lum = 0.2126f * tot.x + 0.7152f * tot.y + 0.0722f * tot.z;
        float oc_e = std::max(lum, 0.0f) * OVERCAST_TRANSMITTANCE;
        F3 e_oc = f3(oc_e, oc_e, oc_e);
        for (size_t i = 0; i < n; ++i) {
            float* t = texels + 4 * i;
            float e = PI_F / 2.0f - ((float)(uint32_t)(i / width) + 0.5f) * dt;
            F3 c = cie_overcast(e_oc, e);
            F3 g = glow.at(std::max(e, -PI_F / 2.0f));
            F3 oc = f3((c.x + g.x * OVERCAST_GLOW) * t[3], (c.y + g.y * OVERCAST_GLOW) * t[3],
                       (c.z + g.z * OVERCAST_GLOW) * t[3]);
            t[0] = t[0] + (oc.x - t[0]) * cover;
            t[1] = t[1] + (oc.y - t[1]) * cover;
            t[2] = t[2] + (oc.z - t[2]) * cover;
        }
    }
    for (size_t i = 0; i < n; ++i) texels[4 * i + 3] = (planet && texels[4 * i + 3] > 0.0f) ? texels[4 * i + 3] : 1.0f;
    float hv = 0.0f;
    if (planet) {
        float rowc = std::ceil((PI_F / 2.0f - dip) / row) - 1.0f;
        rowc = std::min(std::max(rowc, 0.0f), (float)height - 1.0f);
        hv = (rowc + 0.5f) / (float)height;
    }
    *horizon_v_out = hv;
    F3 s = sun_illuminance(a, sun_dir, sun_lux, cover);
    sun_out[0] = s.x; sun_out[1] = s.y; sun_out[2] = s.z;
}

}  // namespace

extern "C" {

void orc_sky_exp4(const double* x, double* out) { exp4(x, out); }

void orc_sky_columns(double r, double mu, double* out) {
    D3 n = columns_exact(r, mu);
    for (int c = 0; c < 3; ++c) out[c] = n.v[c];
}

// Atmosphere::sun_transmittance of Atmosphere::earth(rayleigh, mie, g, ground).
void orc_sky_sun_transmittance(float rayleigh, float mie, float g, const float* ground, const float* dir, float* out) {
    Atm a = earth(rayleigh, mie, g, ground);
    F3 t = sun_transmittance(a, f3(dir[0], dir[1], dir[2]));
    out[0] = t.x; out[1] = t.y; out[2] = t.z;
}

float orc_sky_horizon_elevation(float altitude_km) { return horizon_elevation(altitude_km); }

// Luts::build of Atmosphere::earth(...): a handle for the calls below.
void* orc_sky_tables(float rayleigh, float mie, float g, const float* ground) {
    Handle* h = new Handle;
    h->a = earth(rayleigh, mie, g, ground);
    h->luts.build(h->a);
    return h;
}

void orc_sky_tables_free(void* h) { delete (Handle*)h; }

// The tables: sun 257 x 128 x 3, scattered 64 x 32 x 3, ground 64 x 3 (f32, entry-major).
void orc_sky_tables_get(void* hp, float* sun, float* scattered, float* ground) {
    const Handle* h = (const Handle*)hp;
    std::memcpy(sun, h->luts.sun.data.data(), h->luts.sun.data.size() * 4);
    std::memcpy(scattered, h->luts.scattered.data.data(), h->luts.scattered.data.size() * 4);
    std::memcpy(ground, h->luts.ground.data.data(), h->luts.ground.data.size() * 4);
}

// exp(-Atmosphere::optical_depth(r, mu)) and the table's Luts::sun_transmittance(At::new(mu, r)).
void orc_sky_transmittances(void* hp, double r, double mu, double* exact, double* table) {
    const Handle* h = (const Handle*)hp;
    D3 od = optical_depth(h->a, r, mu);
    D3 t = h->luts.sun_transmittance_at(at_new(mu, r));
    for (int c = 0; c < 3; ++c) {
        exact[c] = std::exp(-od.v[c]);
        table[c] = t.v[c];
    }
}

// Luts::sky (planet frame, Z up).
void orc_sky_radiance(void* hp, float altitude_km, const float* dir, const float* sun, float* out) {
    const Handle* h = (const Handle*)hp;
    F3 l = h->luts.sky(h->a, altitude_km, f3(dir[0], dir[1], dir[2]), f3(sun[0], sun[1], sun[2]));
    out[0] = l.x; out[1] = l.y; out[2] = l.z;
}

// bake_atmosphere_with: glow = (uniform rgb, horizon rgb, height); texels width * height * 4.
void orc_sky_bake(void* hp, const float* sun_dir, const float* sun_lux, float altitude_m, uint32_t width,
                  uint32_t height, const float* glow, float cover, int planet, float* texels, float* sun_illuminance,
                  float* horizon_v) {
    const Handle* h = (const Handle*)hp;
    Glow g{f3(glow[0], glow[1], glow[2]), f3(glow[3], glow[4], glow[5]), glow[6]};
    bake_with(*h, f3(sun_dir[0], sun_dir[1], sun_dir[2]), f3(sun_lux[0], sun_lux[1], sun_lux[2]), altitude_m, width,
              height, g, cover, planet != 0, texels, sun_illuminance, horizon_v);
}

}  // extern "C"
