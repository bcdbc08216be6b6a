"""The sky bake on the device (trt_sky_bake, trt_scene_set_sky) against the oracle's restatement of sky.rs.

Tables and texels within 2e-5 relative of the oracle's (the same f64 and f32 arithmetic; the device's f64 exp, pow,
sqrt and its f32 sin / cos differ from the host's libm in the last bit); the environment packed on the device
(RGBA16F, CDF, brightest luminance, the sun's colour, Params) bit for bit what the host prep packs from the same
bake; the pass renders the baked city as the oracle does."""
import math

import numpy as np
import pytest

import oracle
from threert_b200 import _native as N
from threert_b200 import prep

from util import small_city

pytestmark = pytest.mark.gpu


def atmosphere(elevation_deg=30.0, azimuth_deg=35.0, w=256, h=128, altitude_m=10.0, planet=False, cover=0.0,
               glow=(0.0,) * 7, ground=(0.401978,) * 3, rayleigh=1.0, mie=1.0, g=0.8, lux=(90000.0,) * 3):
    e, a = math.radians(elevation_deg), math.radians(azimuth_deg)
    d = (math.cos(e) * math.cos(a), math.sin(e), math.cos(e) * math.sin(a))
    f3 = lambda v: (N.f32 * 3)(*v)
    return N.Atmosphere(f3(d), f3(lux), rayleigh, mie, g, f3(ground), altitude_m, 1 if planet else 0, f3(glow[:3]),
                        f3(glow[3:6]), glow[6], cover, w, h)


def oracle_bake(atm):
    sky = oracle.Sky(atm.rayleigh_scale, atm.mie_scale, atm.mie_g, tuple(atm.ground_albedo))
    glow = tuple(atm.glow_uniform) + tuple(atm.glow_horizon) + (atm.glow_height,)
    out = sky.bake(tuple(atm.sun_dir), tuple(atm.sun_lux), atm.altitude_m, atm.width, atm.height, glow,
                   atm.cloud_cover, bool(atm.planet))
    tables = sky.tables()
    sky.close()
    return out, tables


def rel_err(got, want):
    scale = np.maximum(np.abs(want), 1e-6 * np.abs(want).max() + 1e-30)
    return (np.abs(got - want) / scale).max()


def test_tables_match_the_oracle(gpu):
    atm = atmosphere()
    _, _, tab = gpu.bake_sky(atm, tables=True)
    (_, _, _), (sun, scat, ground) = oracle_bake(atm)
    n_sun, n_sc = sun.size, scat.size
    assert rel_err(tab[:n_sun], sun.ravel()) < 2e-5
    assert rel_err(tab[n_sun:n_sun + n_sc], scat.ravel()) < 2e-5
    assert rel_err(tab[n_sun + n_sc:], ground.ravel()) < 2e-5


@pytest.mark.parametrize("kw", [dict(elevation_deg=60.0), dict(elevation_deg=10.0), dict(elevation_deg=2.0),
                                dict(elevation_deg=-3.0), dict(elevation_deg=28.0, w=1024, h=512),
                                dict(elevation_deg=30.0, planet=True, altitude_m=400_000.0),
                                dict(elevation_deg=25.0, cover=0.5, glow=(0.1, 0.2, 0.3, 1.0, 0.8, 0.5, 0.06)),
                                dict(elevation_deg=40.0, rayleigh=2.0, mie=5.0, g=0.6, ground=(0.1, 0.3, 0.2))])
def test_bake_matches_the_oracle(gpu, kw):
    atm = atmosphere(**kw)
    tex, res = gpu.bake_sky(atm)
    (want, sun, hv), _ = oracle_bake(atm)
    assert np.isfinite(tex).all() and (tex >= 0).all()
    assert rel_err(tex, want) < 2e-5, rel_err(tex, want)
    assert np.abs(np.array(res.sun_illuminance) - sun).max() <= 1e-5 * max(np.abs(sun).max(), 1e-30)
    assert abs(res.horizon_v - hv) <= 1e-7


def test_tables_are_kept_for_the_same_atmosphere(gpu):
    a, b = atmosphere(elevation_deg=20.0), atmosphere(elevation_deg=50.0)
    _, r1 = gpu.bake_sky(a)
    _, r2 = gpu.bake_sky(b)
    assert r2.tables_ms == 0.0
    _, r3 = gpu.bake_sky(atmosphere(elevation_deg=50.0, mie=2.0))
    assert r3.tables_ms > 0.0


def test_scene_set_sky_packs_as_the_host_does(gpu):
    P = prep.prepare(small_city(sky="atmosphere"))
    atm, sun_light = P.sky_pending
    S = gpu.upload(P)  # the host path: bake on the device, pack on the host (prep.apply_sky)
    host_env, host_words, host_tables = P.env_half.copy(), P.words.copy(), P.tables.copy()
    host_params = P.params.copy()
    # Turn the sun, bake in place, then back: the device path must land where the host path did.
    params = P.params.copy()
    moved = atmosphere(elevation_deg=12.0, w=atm.width, h=atm.height)
    S.set_sky(moved, sun_light, P.info["env_nee_floor"], params)
    env_moved = S.read(5, 0, host_env.nbytes, np.uint16)
    assert (env_moved != host_env).any()
    r = S.set_sky(atm, sun_light, P.info["env_nee_floor"], params)
    env = S.read(5, 0, host_env.nbytes, np.uint16)
    words = S.read(4, 0, host_words.nbytes, np.uint32)
    tables = S.read(3, 0, host_tables.nbytes, np.uint32)
    assert (env == host_env).all()
    assert (words == host_words).all()
    assert (tables == host_tables).all()
    assert (params == host_params).all()
    assert r.brightest > 0.0
    S.close()


def test_baked_city_renders_as_the_oracle_does(gpu):
    from test_gpu_pass import image_parity
    P = prep.prepare(small_city(sky="atmosphere"))
    S = gpu.upload(P)
    assert P.sky_pending is None and P.params.view(np.float32)[24] == 1.0
    acc_g = S.render_raw(P.params, 4)[0]
    acc_o, _ = oracle.Oracle(P).render(P.params, 4)
    frac, mean_err = image_parity(acc_g, acc_o, P.width, P.height, 4)
    assert frac >= 0.99 and mean_err <= 0.01, (frac, mean_err)
    S.close()
