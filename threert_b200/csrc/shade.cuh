// Surface, BSDF, environment and emitter sampling of the offline pass (renderer/shaders/pathtrace.wgsl with
// LIVE = false, APPROX = 0, FEAT = F_INST: no textures, glass, coat, media, fog or procedural geometry), as device
// functions the wavefront's shade kernel calls. Each function names the WGSL function and lines it computes.
// Their loops are not unrolled: the shade kernel's code is large and its warps wait on instruction fetch, and the
// smaller code shades the city 1.3 % faster.
#pragma once
#include "traverse.cuh"

namespace trt {

struct Attr { float4 n0, n1, n2, uv, x; };  // records.wgsl:188 TriAttr
struct TriData { Attr a; V3 v0, e1, e2; };

// pathtrace.wgsl:314-317 tri_indices + 327-355 tri_data
__device__ __forceinline__ TriData tri_data(const DScene& S, const Sections& X, uint32_t ti, uint32_t inst, uint32_t part,
                                            const Inst* rec) {
    uint32_t base = (inst != NO_INST) ? rec->info.z : 0u;
    const uint32_t* ix = S.words + X.w_indices + ti * 3u;
    uint32_t i0 = (__ldg(ix) + base) * 3u, i1 = (__ldg(ix + 1) + base) * 3u, i2 = (__ldg(ix + 2) + base) * 3u;
    float4 p0 = __ldg(S.vertices + i0), p1 = __ldg(S.vertices + i1), p2 = __ldg(S.vertices + i2);
    float4 n0 = __ldg(S.vertices + i0 + 1), n1 = __ldg(S.vertices + i1 + 1), n2 = __ldg(S.vertices + i2 + 1);
    TriData t;
    t.v0 = xyz(p0);
    t.e1 = xyz(p1) - xyz(p0);
    t.e2 = xyz(p2) - xyz(p0);
    t.a.n0 = make_float4(n0.x, n0.y, n0.z, p0.w);
    t.a.n1 = make_float4(n1.x, n1.y, n1.z, n0.w);
    t.a.n2 = make_float4(n2.x, n2.y, n2.z, p1.w);
    t.a.uv = make_float4(n1.w, p2.w, n2.w, bf(part));
    t.a.x = make_float4(0.0f, bf(0u), 0.0f, 0.0f);
    return t;
}
// pathtrace.wgsl:276 inst_vec
__device__ __forceinline__ V3 inst_vec(const Inst& r, V3 v) {
    return {dot(xyz(r.m0), v), dot(xyz(r.m1), v), dot(xyz(r.m2), v)};
}
// pathtrace.wgsl:281-283 inst_normal
__device__ __forceinline__ float4 inst_normal(const Inst& r, float4 n) {
    V3 v = xyz(n);
    V3 o = normalize(V3{dot(xyz(r.n0), v), dot(xyz(r.n1), v), dot(xyz(r.n2), v)});
    return f4(o, n.w);
}
__device__ __forceinline__ uint32_t material_of(const DScene& S, const Sections& X, const Attr& a, uint32_t inst,
                                                const Inst& r) {
    if (inst == NO_INST) return 0;
    return __ldg(S.words + X.w_rows + (r.info.w + bu(a.uv.w)) * 4u) & ROW_MATERIAL;
}
__device__ __forceinline__ float obj_power(const DScene& S, const Sections& X, uint32_t object) {
    return tab(S, X.t_objects + object * 3u).w;
}

struct Surface { V3 p, ng, n, base, emissive; float metallic, roughness, specular; bool front, card; };

// pathtrace.wgsl:1317-1428 surface
__device__ Surface surface(const DScene& S, const Sections& X, V3 o, V3 d, const Hit& h) {
    Inst r = instance_at(S, X, h.inst);
    TriData td = tri_data(S, X, h.tri, h.inst, h.part, &r);
    V3 e1 = inst_vec(r, td.e1), e2 = inst_vec(r, td.e2);
    Attr a = td.a;
    a.n0 = inst_normal(r, a.n0);
    a.n1 = inst_normal(r, a.n1);
    a.n2 = inst_normal(r, a.n2);
    uint32_t object = r.info.y + bu(a.x.y);
    float side = (bu(r.n1.w) & INST_MIRRORED) != 0 ? -1.0f : 1.0f;
    float w = 1.0f - h.u - h.v;
    V3 ng = normalize(cross(e1, e2)) * side;
    V3 n = normalize(xyz(a.n0) * w + xyz(a.n1) * h.u + xyz(a.n2) * h.v);
    uint32_t mi = material_of(S, X, a, h.inst, r);
    uint32_t mb = X.t_materials + mi * 18u;
    float4 base = tab(S, mb), em = tab(S, mb + 1), par = tab(S, mb + 2);
    int32_t flags = (int32_t)tabu(S, mb + 4).z;
    bool front = dot(ng, d) < 0.0f;
    if (!front) ng = -ng;
    if (dot(n, ng) < 0.0f) n = -n;
    Surface s;
    s.p = o + d * h.t;
    s.front = front;
    s.card = flags == MAT_EMITTER_CARD;
    s.emissive = xyz(em) * obj_power(S, X, object);
    s.base = xyz(base);
    s.roughness = clampf(par.y, 0.02f, 1.0f);
    s.metallic = clampf(par.x, 0.0f, 1.0f);
    s.specular = par.z;
    s.ng = ng;
    s.n = n;
    return s;
}

// pathtrace.wgsl:1447-1461 energy_lookup
__device__ __forceinline__ float2 energy_node(const DScene& S, const Sections& X, uint32_t i) {
    float4 v = tab(S, X.t_energy + (i >> 1));
    return (i & 1u) ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
}
__device__ __forceinline__ float2 energy_lookup(const DScene& S, const Sections& X, float roughness, float nov) {
    float x = sqrtf(clampf(nov, 0.0f, 1.0f)) * (float)(ENERGY_N - 1u);
    float y = clampf(roughness, 0.0f, 1.0f) * (float)(ENERGY_N - 1u);
    uint32_t x0 = min((uint32_t)x, ENERGY_N - 2u), y0 = min((uint32_t)y, ENERGY_N - 2u);
    uint32_t i = y0 * ENERGY_N + x0;
    float fx = x - (float)x0, fy = y - (float)y0;
    float2 a = energy_node(S, X, i), b = energy_node(S, X, i + 1), c = energy_node(S, X, i + ENERGY_N),
           d = energy_node(S, X, i + ENERGY_N + 1);
    return make_float2(mixf(mixf(a.x, b.x, fx), mixf(c.x, d.x, fx), fy), mixf(mixf(a.y, b.y, fx), mixf(c.y, d.y, fx), fy));
}

struct Lobes { V3 diffuse, f0, f90, w, e_spec, kd; float a2, p_spec; };

// pathtrace.wgsl:1478-1482 spec_terms + 1642-1700 lobes
__device__ Lobes lobes(const DScene& S, const Sections& X, const Params& P, const Surface& s, float nov) {
    Lobes l;
    float t = 0.0f * (1.0f - s.metallic);
    l.diffuse = s.base * (1.0f - s.metallic) * (1.0f - t);
    float f0 = 0.08f * s.specular;
    l.f0 = mix3(v3(f0), s.base, s.metallic);
    float2 e = energy_lookup(S, X, s.roughness, nov);
    float comp = pf(P, P_MISC + 2);
    float f90 = clampf(dot(l.f0, v3(50.0f / 3.0f)), 0.0f, 1.0f);
    V3 w = v3(1.0f) + l.f0 * (comp * (1.0f / fmaxf(e.x + e.y, 1e-3f) - 1.0f));
    l.f90 = v3(f90);
    l.w = w;
    l.e_spec = (l.f0 * e.x + v3(f90 * e.y)) * w;
    l.kd = v3(1.0f) - l.e_spec;
    float r = s.roughness;
    l.a2 = r * r * r * r;
    float ws = dot(l.e_spec, V3{0.3f, 0.6f, 0.1f});
    float wd = dot(l.diffuse * l.kd, V3{0.3f, 0.6f, 0.1f});
    l.p_spec = clampf(ws / fmaxf(ws + wd, 1e-6f), 0.05f, 1.0f);
    if (wd <= 0.0f) l.p_spec = 1.0f;
    return l;
}
__device__ __forceinline__ float d_ggx(float a2, float noh) {
    float d = (noh * a2 - noh) * noh + 1.0f;
    return a2 / (PI * d * d);
}
__device__ __forceinline__ float vis_smith_joint_approx(float a2, float nov, float nol) {
    return 0.5f / fmaxf(mixf(2.0f * nol * nov, nol + nov, sqrtf(a2)), 1e-7f);
}
__device__ __forceinline__ V3 f_schlick(V3 f0, V3 f90, float voh) {
    float c = 1.0f - voh;
    float c2 = c * c;
    return f0 + (f90 - f0) * (c2 * c2 * c);
}
// pathtrace.wgsl:1733-1760 eval_bsdf_k (BSDF x cos)
__device__ V3 eval_bsdf_k(const Surface& s, const Lobes& lb, V3 v, V3 l, float k) {
    float nol = dot(s.n, l);
    float nov = fmaxf(dot(s.n, v), 1e-4f);
    if (nol <= 0.0f || dot(s.ng, l) <= 0.0f) return v3(0.0f);
    V3 h = normalize(v + l);
    float noh = fmaxf(dot(s.n, h), 0.0f);
    float voh = fmaxf(dot(v, h), 0.0f);
    float dv = d_ggx(lb.a2, noh) * vis_smith_joint_approx(lb.a2, nov, nol);
    V3 spec = dv * f_schlick(lb.f0, lb.f90, voh) * lb.w * k;
    V3 diff = lb.diffuse * (1.0f / PI) * lb.kd;
    return (diff + spec) * nol;
}
__device__ __forceinline__ float g1(float a2, float nov) { return 2.0f * nov / (nov + sqrtf(a2 + (1.0f - a2) * nov * nov)); }
// pathtrace.wgsl:1772-1792 pdf_bsdf
__device__ float pdf_bsdf(const Surface& s, const Lobes& lb, V3 v, V3 l) {
    float nol = dot(s.n, l);
    float pg = 0.0f;
    if (nol <= 0.0f) return pg;
    float nov = fmaxf(dot(s.n, v), 1e-4f);
    V3 h = normalize(v + l);
    float noh = fmaxf(dot(s.n, h), 0.0f);
    float voh = fmaxf(dot(v, h), 1e-6f);
    float dv = g1(lb.a2, nov) * voh * d_ggx(lb.a2, noh) / nov;
    float ps = dv / (4.0f * voh);
    float pd = nol / PI;
    float p_coat = 0.0f, p_trans = 0.0f, pc = 0.0f;
    return pg + p_coat * pc + (1.0f - p_coat - p_trans) * (lb.p_spec * ps + (1.0f - lb.p_spec) * pd);
}
__device__ __forceinline__ float power_heuristic(float a, float b) {
    float a2 = a * a;
    return a2 / fmaxf(a2 + b * b, 1e-20f);
}
__device__ __forceinline__ float light_mis(float pdf_l, const Surface& s, const Lobes& lb, V3 v, V3 l) {
    return power_heuristic(pdf_l, pdf_bsdf(s, lb, v, l));
}
// pathtrace.wgsl:1824-1831 basis (columns t, bt, n)
struct Mat3 { V3 c0, c1, c2; };
__device__ __forceinline__ Mat3 basis(V3 n) {
    float sgn = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sgn + n.z);
    float b = n.x * n.y * a;
    return {V3{1.0f + sgn * n.x * n.x * a, sgn * b, -sgn * n.x}, V3{b, sgn + n.y * n.y * a, -n.y}, n};
}
__device__ __forceinline__ V3 mul(const Mat3& m, V3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
__device__ __forceinline__ V3 mul_t(const Mat3& m, V3 v) { return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }
// pathtrace.wgsl:1834-1852 sample_vndf
__device__ V3 sample_vndf(V3 v, const Mat3& tbn, float alpha, float u1, float u2) {
    V3 vl = mul_t(tbn, v);
    V3 vh = normalize(V3{alpha * vl.x, alpha * vl.y, vl.z});
    float lensq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lensq > 0.0f ? V3{-vh.y, vh.x, 0.0f} / sqrtf(lensq) : V3{1.0f, 0.0f, 0.0f};
    V3 t2 = cross(vh, t1);
    float r = sqrtf(u1);
    float phi = 2.0f * PI * u2;
    float p1 = r * cosf(phi);
    float p2 = r * sinf(phi);
    float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * sqrtf(1.0f - p1 * p1) + s * p2;
    V3 nh = p1 * t1 + p2 * t2 + sqrtf(fmaxf(0.0f, 1.0f - p1 * p1 - p2 * p2)) * vh;
    V3 hl = normalize(V3{alpha * nh.x, alpha * nh.y, fmaxf(0.0f, nh.z)});
    return mul(tbn, hl);
}

// ---- environment (pathtrace.wgsl:1889-1965) ----------------------------------------------------------------------

__device__ __forceinline__ void env_uv(V3 d, float& u, float& v) {
    u = atan2f(d.x, -d.z) / (2.0f * PI) + 0.5f;
    v = acosf(clampf(d.y, -1.0f, 1.0f)) / PI;
}
__device__ __forceinline__ float env_cdf_at(const DScene& S, uint32_t i) { return bf(__ldg(S.words + i)); }
__device__ __forceinline__ V3 env_texel(const DScene& S, uint32_t x, uint32_t y) {
    ushort4 t = __ldg(S.env + (size_t)y * S.env_w + x);
    return {half_to_float(t.x), half_to_float(t.y), half_to_float(t.z)};
}
// textureSampleLevel with a linear, repeating sampler, filtered in f32 from the f16 texels.
__device__ V3 env_bilinear(const DScene& S, float u, float v) {
    int w = (int)S.env_w, h = (int)S.env_h;
    float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
    float fx0 = floorf(x), fy0 = floorf(y);
    float fx = x - fx0, fy = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0;
    int xa = ((x0 % w) + w) % w, xb = (((x0 + 1) % w) + w) % w, ya = ((y0 % h) + h) % h, yb = (((y0 + 1) % h) + h) % h;
    V3 a = env_texel(S, xa, ya), b = env_texel(S, xb, ya), c = env_texel(S, xa, yb), d = env_texel(S, xb, yb);
    return mix3(mix3(a, b, fx), mix3(c, d, fx), fy);
}
__device__ V3 env_radiance(const DScene& S, const Params& P, V3 d) {
    if (pf(P, P_ENV) < 0.5f) return pv(P, P_SKY);
    float u, v;
    env_uv(d, u, v);
    return env_bilinear(S, u, v);
}
__device__ float env_pdf(const DScene& S, const Params& P, V3 d) {
    if (pf(P, P_ENV) < 0.5f) return 1.0f / (4.0f * PI);
    uint32_t w = (uint32_t)pf(P, P_ENV + 1), h = (uint32_t)pf(P, P_ENV + 2);
    float u, v;
    env_uv(d, u, v);
    uint32_t x = min((uint32_t)(u * (float)w), w - 1u);
    uint32_t y = min((uint32_t)(v * (float)h), h - 1u);
    float row_p = env_cdf_at(S, y) - (y > 0u ? env_cdf_at(S, y - 1u) : 0.0f);
    uint32_t base = h + y * w;
    float col_p = env_cdf_at(S, base + x) - (x > 0u ? env_cdf_at(S, base + x - 1u) : 0.0f);
    float sin_t = sinf(((float)y + 0.5f) / (float)h * PI);
    return row_p * col_p * (float)w * (float)h / (2.0f * PI * PI * fmaxf(sin_t, 1e-4f));
}
__device__ uint32_t lower_bound(const DScene& S, uint32_t start, uint32_t count, float x) {
    uint32_t lo = 0, hi = count;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (env_cdf_at(S, start + mid) < x) lo = mid + 1u; else hi = mid;
    }
    return min(lo, count - 1u);
}
__device__ V3 sample_env(const DScene& S, const Params& P, const Rng& R, uint32_t rd) {
    float u4[4];
    R.rng4(rd, u4);
    if (pf(P, P_ENV) < 0.5f) {
        float z = 1.0f - 2.0f * u4[0];
        float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        float phi = 2.0f * PI * u4[1];
        return {r * cosf(phi), z, r * sinf(phi)};
    }
    uint32_t w = (uint32_t)pf(P, P_ENV + 1), h = (uint32_t)pf(P, P_ENV + 2);
    uint32_t y = lower_bound(S, 0u, h, u4[0]);
    uint32_t x = lower_bound(S, h + y * w, w, u4[1]);
    float u = ((float)x + u4[2]) / (float)w;
    float v = ((float)y + u4[3]) / (float)h;
    float theta = v * PI;
    float phi = (u - 0.5f) * 2.0f * PI;
    return {sinf(theta) * sinf(phi), cosf(theta), -sinf(theta) * cosf(phi)};
}
__device__ __forceinline__ V3 offset_origin(V3 p, V3 n) {
    return p + n * (1e-4f * fmaxf(1.0f, fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z)))));
}
__device__ V3 sun_disks(const DScene& S, const Sections& X, const Params& P, V3 d, float pdf) {
    V3 c = v3(0.0f);
    #pragma unroll 1
    for (uint32_t i = 0; i < P.w[P_COUNTS2]; ++i) {
        uint32_t b = X.t_lights + i * 5u;
        float4 dir = tab(S, b + 1);
        if (dot(d, -xyz(dir)) >= dir.w) {
            float omega = 2.0f * PI * (1.0f - dir.w);
            c = c + (xyz(tab(S, b + 2)) / omega) * power_heuristic(pdf, 1.0f / omega);
        }
    }
    return c;
}
__device__ V3 sky_mis(const DScene& S, const Sections& X, const Params& P, V3 d, float pdf) {
    float wgt = 1.0f;
    if (pdf > 0.0f && P.w[P_COUNTS2 + 1] != 0u) wgt = power_heuristic(pdf, env_pdf(S, P, d));
    V3 c = env_radiance(S, P, d) * wgt;
    if (pdf > 0.0f) c = c + sun_disks(S, X, P, d, pdf);
    return c;
}

// ---- emitters (pathtrace.wgsl:457-626, 2040-2065, 2269-2374) --------------------------------------------------------

__device__ __forceinline__ float4 emitter_at(const DScene& S, const Sections& X, uint32_t i) { return tab(S, X.t_emitters + i); }
__device__ __forceinline__ uint32_t emitter_guide(const DScene& S, const Sections& X, const Params& P, uint32_t k) {
    uint4 v = tabu(S, X.t_emitters + P.w[P_COUNTS + 1] + k / 4u);
    uint32_t j = k % 4u;
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}
__device__ __forceinline__ float4 emitter_totals(const DScene& S, const Sections& X, const Params& P) {
    return emitter_at(S, X, P.w[P_COUNTS + 1] + EMITTER_GUIDE / 4u + 1u);
}
__device__ __forceinline__ bool emitters_on(const DScene& S, const Sections& X, const Params& P) {
    if (P.w[P_COUNTS + 1] == 0u) return false;
    return emitter_totals(S, X, P).x > 0.0f;
}
__device__ float4 emitter_pick_u(const DScene& S, const Sections& X, const Params& P, float u) {
    uint32_t k = min((uint32_t)(u * (float)EMITTER_GUIDE), EMITTER_GUIDE - 1u);
    uint32_t lo = emitter_guide(S, X, P, k), hi = emitter_guide(S, X, P, k + 1u);
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (emitter_at(S, X, mid).y < u) lo = mid + 1u; else hi = mid;
    }
    return emitter_at(S, X, min(lo, P.w[P_COUNTS + 1] - 1u));
}
__device__ float lt_imp(float4 nd, V3 x, V3 n) {
    uint32_t wa = bu(nd.x), wb = bu(nd.y);
    float cx = half_to_float(wa & 0xffffu), cy = half_to_float(wa >> 16), cz = half_to_float(wb & 0xffffu),
          cr = half_to_float(wb >> 16);
    V3 dv = V3{cx, cy, cz} - x;
    float d2 = dot(dv, dv);
    float r2 = cr * cr;
    float cb = 1.0f;
    if (d2 > r2 && dot(n, n) > 0.0f) {
        float inv = 1.0f / sqrtf(d2);
        float cos_t = dot(n, dv) * inv;
        float sin_b = cr * inv;
        float cos_b = sqrtf(fmaxf(1.0f - sin_b * sin_b, 0.0f));
        if (cos_t < cos_b) cb = fmaxf(cos_t * cos_b + sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f)) * sin_b, 0.0f);
    }
    return nd.z * cb / fmaxf(d2, r2);
}
__device__ float4 emitter_pick_range(const DScene& S, const Sections& X, const Params& P, uint32_t lo, uint32_t hi, float r) {
    float p0 = lo > 0u ? emitter_at(S, X, max(lo, 1u) - 1u).y : 0.0f;
    float p1 = emitter_at(S, X, hi - 1u).y;
    float u = fminf(p0 + r * (p1 - p0), p1);
    uint32_t k = min((uint32_t)(u * (float)EMITTER_GUIDE), EMITTER_GUIDE - 1u);
    uint32_t l = emitter_guide(S, X, P, k), h = emitter_guide(S, X, P, k + 1u);
    while (l < h) {
        uint32_t mid = (l + h) / 2u;
        if (emitter_at(S, X, mid).y < u) l = mid + 1u; else h = mid;
    }
    return emitter_at(S, X, min(max(l, lo), hi - 1u));
}
struct EPick { float4 e; float p, w; };
// pathtrace.wgsl:547-585 emitter_draw
__device__ EPick emitter_draw(const DScene& S, const Sections& X, const Params& P, const Rng& R, V3 x, V3 n, uint32_t rd) {
    EPick out{make_float4(0, 0, 0, 0), 0.0f, 0.0f};
    float r3[3];
    R.rng3(rd, r3);
    float4 tot = emitter_totals(S, X, P);
    if (!(tot.x > 0.0f)) return out;
    if (!(pf(P, P_LTREE + 3) > 0.5f)) {
        out.e = emitter_pick_u(S, X, P, r3[0]);
        out.p = out.e.z / tot.x;
        out.w = out.e.z;
        return out;
    }
    if (r3[0] < tot.y) {
        out.e = emitter_pick_range(S, X, P, P.w[P_LTREE + 1], P.w[P_COUNTS + 1], r3[1]);
        out.p = out.e.z / tot.x;
        out.w = out.e.z;
        return out;
    }
    float p = 1.0f - tot.y;
    float u = r3[1];
    uint32_t w = bu(tab(S, 0u).w);
    #pragma unroll 1
    for (uint32_t k = 0; k <= LT_PATH_BITS && (w & LT_LEAF) == 0u; ++k) {
        float4 l = tab(S, w), r = tab(S, w + 1u);
        float il = lt_imp(l, x, n), ir = lt_imp(r, x, n);
        if (!(il + ir > 0.0f)) return out;
        float pl = il / (il + ir);
        if (u < pl) { w = bu(l.w); p *= pl; u = u / pl; }
        else { w = bu(r.w); p *= 1.0f - pl; u = (u - pl) / (1.0f - pl); }
        u = clampf(u, 0.0f, 0.99999994f);
    }
    if ((w & LT_LEAF) == 0u) return out;
    uint32_t lo = w & 0x1fffffffu, hi = lo + ((w >> 29) & 3u) + 1u;
    float wsum = 0.0f;
    #pragma unroll 1
    for (uint32_t j = lo; j < hi; ++j) wsum += emitter_at(S, X, j).z;
    float t = r3[2] * wsum;
    out.e = emitter_at(S, X, hi - 1u);
    #pragma unroll 1
    for (uint32_t j = lo; j < hi; ++j) {
        float4 c = emitter_at(S, X, j);
        if (t < c.z) { out.e = c; break; }
        t -= c.z;
    }
    out.p = p * out.e.z / wsum;
    out.w = out.e.z;
    return out;
}
struct ETri { V3 v0; uint32_t tri; V3 e1; uint32_t inst; V3 e2; uint32_t code; uint32_t part, flags; };
__device__ __forceinline__ ETri etri_at(const DScene& S, const Sections& X, uint32_t i) {
    uint32_t b = X.t_emitter_tris + i * 4u;
    uint4 r0 = tabu(S, b), r1 = tabu(S, b + 1), r2 = tabu(S, b + 2), r3 = tabu(S, b + 3);
    return {{bf(r0.x), bf(r0.y), bf(r0.z)}, r0.w, {bf(r1.x), bf(r1.y), bf(r1.z)}, r1.w,
            {bf(r2.x), bf(r2.y), bf(r2.z)}, r2.w, r3.x, r3.y};
}
// pathtrace.wgsl:590-626 emitter_pmf
__device__ float emitter_pmf(const DScene& S, const Sections& X, const Params& P, uint32_t ei, const ETri& em, V3 x, V3 n) {
    float4 tot = emitter_totals(S, X, P);
    if (!(tot.x > 0.0f)) return 0.0f;
    uint32_t code = em.code & ~EMITTER_MOVES;
    if ((code >> LT_PATH_BITS) == 0u) return emitter_at(S, X, code).z / tot.x;
    uint32_t depth = (code >> LT_PATH_BITS) - 1u;
    float p = 1.0f - tot.y;
    uint32_t w = bu(tab(S, 0u).w);
    #pragma unroll 1
    for (uint32_t k = 0; k < depth; ++k) {
        float4 l = tab(S, w), r = tab(S, w + 1u);
        float il = lt_imp(l, x, n), ir = lt_imp(r, x, n);
        if (!(il + ir > 0.0f)) return 0.0f;
        uint32_t right = (code >> k) & 1u;
        p *= (right == 1u ? ir : il) / (il + ir);
        w = bu(right == 1u ? r.w : l.w);
    }
    uint32_t lo = w & 0x1fffffffu, hi = lo + ((w >> 29) & 3u) + 1u;
    float wsum = 0.0f, we = 0.0f;
    #pragma unroll 1
    for (uint32_t j = lo; j < hi; ++j) {
        float4 c = emitter_at(S, X, j);
        wsum += c.z;
        if (bu(c.x) == ei) we = c.z;
    }
    return p * we / wsum;
}
// pathtrace.wgsl:2023-2028 emitter_attrs + 2269-2280 emitter_radiance
__device__ V3 emitter_radiance(const DScene& S, const Sections& X, const ETri& em) {
    Inst r = instance_at(S, X, em.inst);
    Attr a = tri_data(S, X, em.tri, em.inst, em.part, &r).a;
    uint32_t object = r.info.y + bu(a.x.y);
    uint32_t mi = material_of(S, X, a, em.inst, r);
    float4 e = tab(S, X.t_materials + mi * 18u + 1u);
    return xyz(e) * obj_power(S, X, object);
}
// pathtrace.wgsl:2050-2065 emit_mis
__device__ float emit_mis(const DScene& S, const Sections& X, const Params& P, const Hit& hit, V3 d, float pdf, V3 mis_x,
                          V3 mis_n) {
    if (!emitters_on(S, X, P)) return 1.0f;
    uint32_t rows = tabu(S, X.t_instances + hit.inst * 10u + 6u).w;
    uint32_t first = __ldg(S.words + X.w_rows + (rows + hit.part) * 4u + 2u);
    if (first == NO_EMITTER) return 1.0f;
    uint32_t entry = first + bu(__ldg(S.leaves + 3ull * hit.tri + 1).w);
    ETri em = etri_at(S, X, entry);
    V3 cr = cross(em.e1, em.e2);
    float area = 0.5f * length(cr);
    float cos_l = fabsf(dot(normalize(cr), d));
    float sel = emitter_pmf(S, X, P, entry, em, mis_x, mis_n);
    if (!(sel > 0.0f)) return 1.0f;
    return power_heuristic(pdf, sel / fmaxf(area, 1e-12f) * hit.t * hit.t / fmaxf(cos_l, 1e-6f));
}
struct ES { V3 le, l; float dist, pdf_w, w; };
// pathtrace.wgsl:2283-2340 sample_emitter_ris
__device__ ES sample_emitter_ris(const DScene& S, const Sections& X, const Params& P, const Rng& R, V3 x, V3 n, uint32_t m,
                                 const Surface& sf, const Lobes& lb, V3 v, uint32_t rd) {
    ES r{v3(0.0f), V3{0.0f, 1.0f, 0.0f}, 0.0f, 0.0f, 0.0f};
    float wsum = 0.0f, pb0 = 0.0f, pb1 = 0.0f, pick_ph = 0.0f, pick_pdf = 0.0f;
    uint32_t pick_i = 0;
    #pragma unroll 1
    for (uint32_t k = 0; k < m; ++k) {
        uint32_t dk = rng_sub(rd, k);
        EPick pk = emitter_draw(S, X, P, R, x, n, dk);
        float bb[3];
        R.rng3(rng_sub(dk, 1u), bb);
        float b1 = bb[0], b2 = bb[1];
        if (pk.p <= 0.0f) continue;
        if (b1 + b2 > 1.0f) { b1 = 1.0f - b1; b2 = 1.0f - b2; }
        ETri em = etri_at(S, X, bu(pk.e.x));
        V3 lp = em.v0 + em.e1 * b1 + em.e2 * b2;
        V3 cr = cross(em.e1, em.e2);
        float a2 = length(cr);
        if (!(a2 > 0.0f)) continue;
        V3 ln = cr / a2;
        V3 dl = lp - x;
        float d2 = fmaxf(dot(dl, dl), 1e-8f);
        V3 l = dl * (1.0f / sqrtf(d2));
        float g = fabsf(dot(ln, l)) * (dot(n, n) == 0.0f ? 1.0f : fmaxf(dot(n, l), 0.0f)) / d2;
        if (m > 1u) g = fabsf(dot(ln, l)) * luminance(eval_bsdf_k(sf, lb, v, l, 1.0f)) / d2;
        float ph = pk.w / (pk.e.w * 1.0f) * g;
        float pdf_a = pk.p / (0.5f * a2);
        float w = ph / pdf_a;
        if (!(w > 0.0f)) continue;
        wsum += w;
        if (bb[2] * wsum < w) { pb0 = b1; pb1 = b2; pick_ph = ph; pick_i = bu(pk.e.x); pick_pdf = pdf_a; }
    }
    if (pick_ph <= 0.0f) return r;
    ETri em = etri_at(S, X, pick_i);
    V3 lp = em.v0 + em.e1 * pb0 + em.e2 * pb1;
    V3 ln = normalize(cross(em.e1, em.e2));
    V3 dl = lp - x;
    float d2 = dot(dl, dl);
    float dist = sqrtf(d2);
    V3 l = dl / dist;
    float cos_l = dot(ln, -l);
    if ((em.flags & EMITTER_CARD) == 0u) cos_l = fabsf(cos_l);
    if (cos_l <= 0.0f) return r;
    r.le = emitter_radiance(S, X, em);
    r.l = l;
    r.dist = dist;
    r.pdf_w = pick_pdf * d2 / cos_l;
    r.w = (wsum / (float)m) / pick_ph * cos_l / d2;
    return r;
}
// pathtrace.wgsl:2344-2374 sample_emitter
__device__ ES sample_emitter(const DScene& S, const Sections& X, const Params& P, const Rng& R, V3 x, V3 n, uint32_t rd) {
    ES r{v3(0.0f), V3{0.0f, 1.0f, 0.0f}, 0.0f, 0.0f, 0.0f};
    EPick pk = emitter_draw(S, X, P, R, x, n, rd);
    if (pk.p <= 0.0f) return r;
    ETri em = etri_at(S, X, bu(pk.e.x));
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
    float dist = sqrtf(d2);
    V3 l = dl / dist;
    float cos_l = dot(ln, -l);
    if ((em.flags & EMITTER_CARD) == 0u) cos_l = fabsf(cos_l);
    if (cos_l <= 0.0f) return r;
    r.le = emitter_radiance(S, X, em);
    r.l = l;
    r.dist = dist;
    r.pdf_w = pk.p / area * d2 / cos_l;
    r.w = 1.0f / r.pdf_w;
    return r;
}

}  // namespace trt
