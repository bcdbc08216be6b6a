"""The atmosphere's sky oracle (oracle/sky.cpp) pinned to renderer/src/sky.rs's own known answers and checks.

Each test restates one of the reference's tests (sky.rs:1003-1045 overcast, 1069-1096 from space, 1211-1225 the fast
exponential, 1228-1251 the columns, 1254-1275 the sun table, 1278-1311 the sun's transmittance, 1315-1341 its table,
1344-1389 the day sky, 1391-1411 twilight, 1423-1440 no bands), with the reference's inputs and bounds.
"""
import math

import numpy as np
import pytest

import oracle

R_GROUND, R_TOP = 6360.0, 6460.0
RAYLEIGH = np.array([5.802e-3, 13.558e-3, 33.1e-3])
MIE_S, MIE_A = 3.996e-3, 0.444e-3
OZONE = np.array([0.650e-3, 1.881e-3, 0.085e-3])
VEIL = 1.65


def lum(v):
    return 0.2126 * v[0] + 0.7152 * v[1] + 0.0722 * v[2]


def planet(elevation_deg, azimuth_deg):
    e, a = math.radians(elevation_deg), math.radians(azimuth_deg)
    return np.array([math.cos(e) * math.cos(a), math.cos(e) * math.sin(a), math.sin(e)], np.float32)


def sun_at(elevation_deg):
    e = math.radians(elevation_deg)
    return np.array([math.cos(e), math.sin(e), 0.0], np.float32)


@pytest.fixture(scope="module")
def earth():
    s = oracle.Sky(1.0, 1.0, 0.8, (0.401978,) * 3)
    yield s
    s.close()


@pytest.fixture(scope="module")
def black():
    s = oracle.Sky(1.0, 1.0, 0.8, (0.0,) * 3)
    yield s
    s.close()


def test_fast_exponential():
    worst, worst_near = 0.0, 0.0
    for i in range(-8690, 201, 7):
        x = i * 0.01
        e = oracle.sky_exp4([x, x - 0.003, 0.0, -1e-9])
        err = max(abs(e[0] / math.exp(x) - 1.0), abs(e[1] / math.exp(x - 0.003) - 1.0))
        worst = max(worst, err)
        if abs(x) < 2.0:
            worst_near = max(worst_near, err)
        assert e[2] == 1.0 and abs(e[3] - 1.0) < 1e-7
    assert worst < 5e-6 and worst_near < 3e-7, (worst, worst_near)
    assert oracle.sky_exp4([-1000.0, 0, 0, 0])[0] < 2e-38


def test_columns_are_integrated_exactly():
    up = oracle.sky_columns(R_GROUND, 1.0)
    assert abs(up[0] - 8.0 * (1.0 - math.exp(-100.0 / 8.0))) < 1e-6, up
    assert abs(up[1] - 1.2) < 1e-6 and abs(up[2] - 15.0) < 0.03, up
    n = 400_000
    for h, mu in [(0.0, 0.0), (0.0, 0.02), (0.0, 0.3), (3.0, 0.0), (20.0, 0.05), (60.0, 0.0), (-3.0, 0.0)]:
        r = R_GROUND + h
        d = -r * mu + math.sqrt(max(r * r * (mu * mu - 1.0) + R_TOP * R_TOP, 0.0))
        t = (np.arange(n) + 0.5) / n * d
        alt = np.sqrt(r * r + t * t + 2.0 * r * mu * t) - R_GROUND
        dens = np.stack([np.exp(-alt / 8.0), np.exp(-alt / 1.2), np.maximum(1.0 - np.abs(alt - 25.0) / 15.0, 0.0)])
        ref = (dens * (d / n)).sum(1)
        fast = oracle.sky_columns(r, mu)
        for c in range(3):
            tol = (2e-3 if c == 2 else 2e-4) * max(ref[c], 1.0)
            assert abs(fast[c] - ref[c]) < tol, (h, mu, fast, ref)


# sky.rs:1317-1330: sun elevation (degrees), rayleigh scale, mie scale, then R, G, B.
SUN_TABLE = [
    [90.0, 1.0, 1.0, 0.924612, 0.84226, 0.716526],
    [45.0, 1.0, 1.0, 0.89537, 0.784979, 0.624876],
    [20.0, 1.0, 1.0, 0.799125, 0.611592, 0.384148],
    [10.0, 1.0, 1.0, 0.659276, 0.400327, 0.166401],
    [5.0, 1.0, 1.0, 0.488058, 0.206397, 0.042848],
    [2.0, 1.0, 1.0, 0.291951, 0.0684695, 0.00389411],
    [0.0, 1.0, 1.0, 0.0935232, 0.00763352, 3.24136e-05],
    [-1.0, 1.0, 1.0, 0.00821672, 0.000199967, 3.94459e-08],
    [-3.0, 1.0, 1.0, 0.0, 0.0, 0.0],
    [30.0, 2.0, 5.0, 0.700244, 0.50156, 0.250179],
    [3.0, 0.5, 20.0, 0.0428066, 0.0215879, 0.00795393],
    [15.0, 0.0, 0.0, 0.960424, 0.897494, 0.990766],
]


@pytest.mark.parametrize("row", SUN_TABLE)
def test_sun_transmittance_table(row):
    e = np.float32(math.radians(np.float32(row[0])))
    d = np.array([math.cos(e) * 0.6, math.sin(e), math.cos(e) * 0.8], np.float32) * 3.0
    t = oracle.sky_sun_transmittance(d, row[1], row[2], 0.8, (0.0,) * 3)
    for c in range(3):
        assert abs(float(t[c]) - row[3 + c]) <= 1e-3 * row[3 + c] + 1e-9, (row, t)


def test_sun_transmittance_is_smooth_and_reddens():
    zenith = oracle.sky_sun_transmittance(sun_at(90.0))
    for c in range(3):
        medium = RAYLEIGH[c] * 8.0 * (1.0 - math.exp(-12.5)) + (MIE_S + MIE_A) * 1.2 + OZONE[c] * 15.0
        veil = VEIL * (RAYLEIGH[c] + MIE_S + MIE_A)
        assert abs(float(zenith[c]) - math.exp(-(medium + veil))) < 1e-4, zenith
    last = zenith
    for i in range(0, 1901, 3):
        elevation = 90.0 - i * 0.05
        t = oracle.sky_sun_transmittance(sun_at(elevation))
        assert t[0] >= t[1] >= t[2] >= 0.0, (elevation, t)
        assert (t <= last + 1e-6).all(), (elevation, t, last)
        assert (last - t).max() < 0.012 * 3, (elevation, t, last)
        if elevation < -3.0:
            assert t.max() < 1e-6, (elevation, t)
        last = t
    level = oracle.sky_sun_transmittance(sun_at(0.0))
    assert 0.05 < level[0] < 0.15 and level[1] < 0.02 and level[2] < 1e-3, level
    bare = oracle.sky_sun_transmittance(sun_at(45.0), 0.0, 0.0)
    assert bare.min() > 0.95 and bare[1] < bare[2], bare
    hazy = oracle.sky_sun_transmittance(sun_at(45.0), 1.0, 10.0)
    assert hazy[0] < oracle.sky_sun_transmittance(sun_at(45.0))[0] * 0.95, hazy


def test_sun_table_matches_the_quadrature(earth):
    worst = 0.0
    for i in range(0, 150, 2):
        r = R_GROUND + 100.0 * (i / 150.0) ** 3
        for k in range(0, 501, 2):
            mu = -0.25 + 1.25 * (k / 500.0) ** 2
            exact, table = earth.transmittances(r, mu)
            worst = max(worst, float(np.abs(exact - table).max()))
    assert worst < 6e-3, worst


def test_day_sky_is_physical(earth, black):
    for elevation in [75.0, 40.0, 15.0]:
        sun = planet(elevation, 0.0)
        n, m = 24, 48
        sky = np.zeros(3)
        for i in range(n):
            z = (i + 0.5) / n
            for k in range(m):
                phi = (k + 0.5) / m * 2.0 * math.pi
                h = math.sqrt(1.0 - z * z)
                l = black.radiance(0.0, [h * math.cos(phi), h * math.sin(phi), z], sun)
                assert l.min() >= 0.0 and l.max() < 5.0 and np.isfinite(l).all(), l
                sky += l * z * (2.0 * math.pi / (n * m))
        # the black ground's transmittance toward the sun: the sun table agrees with it within 6e-3
        direct, _ = black.transmittances(R_GROUND, float(sun[2]))
        total, top = sky + direct * sun[2], sun[2]
        assert total.max() < top, (elevation, total, top)
        assert total.min() > 0.6 * top, (elevation, total, top)
        assert sky[2] > sky[1] > sky[0], sky
    sun = planet(60.0, 0.0)
    zenith, horizon = earth.radiance(0.0, planet(90.0, 0.0), sun), earth.radiance(0.0, planet(3.0, 180.0), sun)
    assert zenith[2] / zenith[0] > 1.5 * horizon[2] / horizon[0], (zenith, horizon)
    assert lum(horizon) > 2.0 * lum(zenith), (zenith, horizon)
    for e, az in [(10.0, 40.0), (45.0, 90.0), (80.0, 170.0), (2.0, 5.0)]:
        left, right = earth.radiance(0.0, planet(e, az), sun), earth.radiance(0.0, planet(e, -az), sun)
        assert np.abs(left - right).max() < 1e-5 * left.max(), (left, right)
        turned = earth.radiance(0.0, planet(e, az + 77.0), planet(60.0, 77.0))
        assert np.abs(left - turned).max() < 1e-4 * left.max(), (left, turned)
    near, far = earth.radiance(0.0, planet(60.0, 8.0), sun), earth.radiance(0.0, planet(60.0, 120.0), sun)
    assert near[0] > 3.0 * far[0], (near, far)
    assert lum(earth.radiance(10.0, planet(90.0, 0.0), sun)) < 0.5 * lum(zenith)
    down = earth.radiance(1.0, planet(-60.0, 90.0), sun)
    assert 0.09 < down[1] < 0.16, down


def test_low_sun_reddens_and_twilight_fades(earth):
    sunset = planet(2.0, 0.0)
    glow, overhead = earth.radiance(0.0, planet(3.0, 0.0), sunset), earth.radiance(0.0, planet(90.0, 0.0), sunset)
    assert glow[0] > 2.0 * glow[1] and glow[1] > 2.0 * glow[2], glow
    assert overhead[2] > 1.5 * overhead[0], overhead
    last = float("inf")
    for elevation in [30.0, 10.0, 2.0, 0.0, -2.0, -4.0, -6.0, -9.0, -12.0]:
        l = lum(earth.radiance(0.0, planet(60.0, 90.0), planet(elevation, 0.0)))
        assert 0.0 <= l < last, (elevation, l, last)
        assert elevation < -5.0 or l > 5e-5, (elevation, l)
        last = l
    assert last < 2e-6, last
    assert (earth.radiance(0.0, planet(60.0, 90.0), planet(-30.0, 0.0)) == 0.0).all()


def test_sky_from_space(earth):
    sun = planet(40.0, 0.0)
    dip = math.degrees(oracle.sky_horizon_elevation(400.0))
    assert abs(dip + 19.83) < 0.05, dip
    top = -math.degrees(math.acos(R_TOP / (R_GROUND + 400.0)))
    for az in [0.0, 90.0, 180.0]:
        assert (earth.radiance(400.0, planet(90.0, az), sun) == 0.0).all()
        assert (earth.radiance(400.0, planet(top + 0.2, az), sun) == 0.0).all()
        limb = earth.radiance(400.0, planet(dip + 0.1, az), sun)
        assert lum(limb) > 0.01 and limb[2] > limb[0], (az, limb)
        high = earth.radiance(400.0, planet(dip + 1.5, az), sun)
        assert lum(high) < 0.5 * lum(limb), (az, high, limb)
    for e, az in [(90.0, 0.0), (10.0, 0.0), (-5.0, 180.0), (-10.2, 90.0)]:
        below, above = earth.radiance(99.9, planet(e, az), sun), earth.radiance(100.1, planet(e, az), sun)
        tol = 0.03 * max(lum(below), lum(above)) + 1e-6
        assert abs(lum(below) - lum(above)) <= tol, (e, az, below, above)


def _roughness(tex, column):
    w_h = tex.shape[0]
    at = lambda row: lum(tex[row, column, :3])
    second = lambda row: (at(row - 1) - 2.0 * at(row) + at(row + 1)) / at(row)
    last = w_h // 2 - w_h // 16
    size = max(abs(second(r)) for r in range(1, last + 1))
    change = max(abs(second(r + 1) - second(r)) for r in range(1, last))
    return size, change


def test_bake_has_no_bands(earth):
    w, h = 256, 128
    for elevation in [60.0, 10.0, 2.0, -3.0]:
        tex, _, _ = earth.bake(sun_at(elevation), (1.0, 1.0, 1.0), 0.0, w, h)
        assert np.isfinite(tex).all() and (tex >= 0.0).all()
        for column in [0, w // 4, w // 2]:
            size, change = _roughness(tex, column)
            most, jump = (0.02, 0.004) if elevation > 0.0 else (0.05, 0.015)
            assert size < most and change < jump, (elevation, column, size, change)


def test_full_cover_is_the_cie_overcast_sky():
    a = oracle.Sky(1.0, 10.0, 0.8, (0.3,) * 3)
    sun = np.array([0.3, 0.5, -0.8], np.float32)
    sun /= np.linalg.norm(sun)
    lux = (100_000.0,) * 3
    w, h = 256, 128
    clear = a.bake(sun, lux, 10.0, w, h)
    oc = a.bake(sun, lux, 10.0, w, h, cover=1.0)
    dt, dp = math.pi / h, 2.0 * math.pi / w
    th = (np.arange(h) + 0.5) * dt
    k = np.maximum(np.cos(th), 0.0) * np.sin(th) * dt * dp

    def e_h(b):
        tex, s, _ = b
        return float((lum(np.moveaxis(tex[..., :3], -1, 0)) * k[:, None]).sum() + lum(s * sun[1]))

    assert (oc[1] == 0.0).all()
    ratio = e_h(oc) / e_h(clear)
    assert abs(ratio - 0.3) < 0.01, ratio
    row = lambda e_deg: min(int((90.0 - e_deg) / 180.0 * h), h - 1)
    e_of = lambda r: math.pi / 2.0 - (r + 0.5) * math.pi / h
    z, ten = row(89.0), row(10.0)
    expect = (1.0 + 2.0 * math.sin(e_of(z))) / (1.0 + 2.0 * math.sin(e_of(ten)))
    for x in [0, w // 3, 2 * w // 3]:
        got = lum(oc[0][z, x]) / lum(oc[0][ten, x])
        assert abs(got / expect - 1.0) < 1e-3, (got, expect)
        c = oc[0][ten, x]
        assert abs(c[0] - c[2]) < 1e-3 * c[1], c
    half = a.bake(sun, lux, 10.0, w, h, cover=0.5)
    assert np.linalg.norm(half[1] - clear[1] * 0.5) < 1e-3 * np.linalg.norm(clear[1])
    kk = (ten, 7)
    assert abs(lum(half[0][kk]) - 0.5 * (lum(clear[0][kk]) + lum(oc[0][kk]))) < 1e-3 * lum(clear[0][kk])
    a.close()


def test_planet_bake_dips_its_horizon(earth):
    w, h = 256, 128
    for altitude_km in [0.002, 10.0, 400.0, 2000.0]:
        tex, _, hv = earth.bake(sun_at(30.0), (120_000.0,) * 3, altitude_km * 1000.0, w, h, planet=True)
        dip = oracle.sky_horizon_elevation(max(altitude_km, 0.005))
        limb = int(math.floor(np.float32(hv) * h))
        elev = lambda y: math.pi / 2.0 - (y + 0.5) / h * math.pi
        assert elev(limb) - 0.5 * math.pi / h <= dip + 1e-5 and dip < elev(limb) + 0.5 * math.pi / h + 1e-5, limb
        for y in range(h):
            row = tex[y]
            l = float(lum(row[:, :3].T).sum()) / w
            if y > limb:
                assert l == 0.0, (altitude_km, y)
            elif y == limb:
                assert l > 0.0 and ((row[:, 3] > 0.0) & (row[:, 3] <= 1.0)).all(), (altitude_km, y)
            else:
                assert (row[:, 3] == 1.0).all()
            if altitude_km > 100.0 and elev(y) > -math.acos(R_TOP / (R_GROUND + altitude_km)) + 0.03:
                assert l == 0.0, (altitude_km, y)
        back = tex[limb, w // 2, :3] / tex[limb, w // 2, 3]
        assert back[2] > 0.0, (altitude_km, back)
    flat, _, hv = earth.bake(sun_at(30.0), (1.0,) * 3, 400_000.0, w, h)
    assert hv == 0.0 and (flat[..., 3] == 1.0).all()


def env_cdf_numpy(tex):
    """lib.rs:916-941 build_env_cdf in float32, each running sum sequential as the reference's loop."""
    h, w = tex.shape[:2]
    f = np.float32
    sin_t = np.sin(((np.arange(h, dtype=f) + f(0.5)) / f(h) * f(math.pi)).astype(f)).astype(f)
    lum = (f(0.2126) * tex[..., 0] + f(0.7152) * tex[..., 1]) + f(0.0722) * tex[..., 2]
    terms = np.maximum(lum, f(0)) * sin_t[:, None] + f(1e-12)
    acc = np.cumsum(terms.astype(f), axis=1, dtype=f)
    rows = acc[:, -1].copy()
    cond = (acc / rows[:, None]).astype(f)
    total = f(0)
    for r in rows:
        total = f(total + r)
    marg = np.cumsum((rows / total).astype(f), dtype=f)
    return np.concatenate([marg, cond.ravel()])


def test_host_env_packing_matches_build_env_cdf():
    from threert_b200 import _native as N
    import ctypes as C
    rng = np.random.default_rng(3)
    tex = (rng.random((32, 64, 4)) * np.linspace(0.0, 3.0, 64)[None, :, None]).astype(np.float32)
    cdf = np.zeros(32 + 32 * 64, np.float32)
    env = np.zeros(32 * 64 * 4, np.uint16)
    b = C.c_float()
    assert N.lib().trt_prep_env(tex.ctypes.data_as(C.POINTER(C.c_float)), 64, 32,
                                env.ctypes.data_as(C.POINTER(C.c_uint16)), cdf.ctypes.data_as(C.POINTER(C.c_float)),
                                C.byref(b)) == 0
    want = env_cdf_numpy(tex)
    # (numpy's float32 sin may differ from the C library's sinf by an ulp: compare to 2 ulps.)
    assert np.allclose(cdf, want, rtol=3e-7, atol=0), np.abs(cdf - want).max()
    assert (env == tex.astype(np.float16).view(np.uint16).ravel()).all()
    lum = (np.float32(0.2126) * tex[..., 0] + np.float32(0.7152) * tex[..., 1]) + np.float32(0.0722) * tex[..., 2]
    assert b.value == lum.max()


def test_atmosphere_city_prepares_and_takes_a_host_bake():
    from threert_b200 import prep, scenes
    d = scenes.city(n_objects=30, width=24, height=16, seed=5, extent=40.0, n_emitters=20, box_segments=1,
                    sphere_slices=6, sphere_stacks=5, sky_size=(64, 32))
    P = prep.prepare(d)
    assert P.sky_pending is not None and (P.env_w, P.env_h) == (64, 32)
    atm, sun_light = P.sky_pending
    assert sun_light == 0 and atm.width == 64 and atm.height == 32
    assert np.allclose(np.array(atm.sun_dir), -np.array(d.lights[0].direction), atol=1e-6)
    sky = oracle.Sky(atm.rayleigh_scale, atm.mie_scale, atm.mie_g, tuple(atm.ground_albedo))
    tex, sun, hv = sky.bake(tuple(atm.sun_dir), tuple(atm.sun_lux), atm.altitude_m, 64, 32)
    sky.close()

    class Res:
        sun_illuminance = tuple(float(v) for v in sun)
        horizon_v = hv

    prep.apply_sky(P, tex, Res, sun_light)
    assert P.sky_pending is None
    at = int(P.params[136])
    cdf = P.words[at:at + 32 + 64 * 32].view(np.float32)
    assert np.allclose(cdf, env_cdf_numpy(tex), rtol=3e-7, atol=0)
    lt = (int(P.params[126]) + 2) * 4
    assert (P.tables[lt:lt + 3].view(np.float32) == sun).all()
    assert P.params.view(np.float32)[24] == 1.0 and P.params.view(np.float32)[25] == 64.0
    # the sun through the air: dimmer and redder than above it
    assert sun[0] < 90000.0 and sun[2] < sun[0]
    # the baked scene renders on the oracle: the sky lights the ground
    O = oracle.Oracle(P)
    acc, st = O.render(P.params, 1)
    assert st["closest_rays"] > 0 and np.isfinite(acc).all()
