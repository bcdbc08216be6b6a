"""Parity on the benchmarked configurations at their full sizes, through the C ABI, against the oracle on the same
buffers: the Cornell box at 256 x 256 and 16 spp (config 0), the 1,984,402-triangle city at 1280 x 720 (config 1,
the bench's workload), and the 5,000-walker crowd after one deformation in one pose group and in 5,000 (config 2).

The reference's own standard for its walk is brute-force agreement on its real trees (renderer/src/units.rs:1442-1535,
renderer/src/lib.rs:1649 through prepare_as); here the oracle's walk, itself pinned to brute force, stands for it.
Traversal: the hit or miss agrees on >= 99.99 % of rays, t within 1e-6 relative, and a different triangle only at an
exact tie. Images at matched seed and spp: per-pixel luminance within 3 combined standard errors on >= 99 % of
pixels, image means within 1 %, first-hit albedo and normal sums equal to the shading's rounding. The device's
transcendentals, the one arithmetic the oracle does not share bit for bit, are bounded in ulps."""
import dataclasses

import numpy as np
import pytest

import oracle
from threert_b200 import crowd, prep, scenes
from threert_b200 import _native as N
from threert_b200.gpu import RAY_DTYPE, frame_of

from util import luma, random_rays

pytestmark = pytest.mark.gpu

MISS = 0xFFFFFFFF
CITY_W, CITY_H, CITY_DEPTH = 1280, 720, 4
CITY_FRAME = 5  # the bench's first timed frame


def camera_rays(params, w, h):
    """The pinhole camera's ray through every pixel centre (pathtrace.wgsl:4002-4026 without the sample's jitter)."""
    f = params[0:16].view(np.float32)
    pos, tan_h = f[0:3], f[3]
    fwd, aspect, right, up = f[4:7], f[7], f[8:11], f[12:15]
    gx, gy = np.meshgrid(np.arange(w, dtype=np.float64), np.arange(h, dtype=np.float64))
    ndcx = (gx.ravel() + 0.5) / w * 2.0 - 1.0
    ndcy = 1.0 - (gy.ravel() + 0.5) / h * 2.0
    d = fwd[None] + right[None] * (ndcx * tan_h * aspect)[:, None] + up[None] * (ndcy * tan_h)[:, None]
    r = np.zeros(w * h, RAY_DTYPE)
    r["o"] = pos
    r["d"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r["tmax"] = np.float32(3.0e38)
    r["mode"] = 0
    return r


def check_hits(O, params, rays, got, want, min_both=1000):
    """Hit or miss on >= 99.99 % of rays; t within 1e-6 relative; a different triangle only at an exact tie (the GPU's
    own triangle lies at the oracle's t). Returns the closest-hit rays that hit in both."""
    hg, hw = got["tri"] != MISS, want["tri"] != MISS
    agree = (hg == hw).mean()
    assert agree >= 0.9999, agree
    both = hg & hw & (rays["mode"] == 0)
    assert both.sum() >= min_both, both.sum()
    rel = np.abs(got["t"][both] / want["t"][both] - 1)
    assert rel.max() <= 1e-6, (rel.max(), (rel > 1e-6).sum())
    differ = both & ((got["tri"] != want["tri"]) | (got["inst"] != want["inst"]))
    if differ.any():
        t_own = O.intersect(params, rays[differ], got[differ])
        tie = np.abs(t_own / want["t"][differ] - 1) <= 1e-6
        assert (differ.sum() - tie.sum()) <= 1e-4 * both.sum(), (differ.sum(), tie.sum())
    return both


def first_hit_guides_agree(acc_g, acc_o):
    """First-hit albedo and normal sums: equal up to the shading's rounding on all but <= 1e-4 of pixels. (A camera ray
    that meets two surfaces at exactly the same t may take either: the binary walks take the oracle's, the wide walk
    the one its octant order meets first, and the two can differ in material.)"""
    same = (np.isclose(acc_g[:, 4:7], acc_o[:, 4:7], rtol=1e-4, atol=1e-5).all(1)
            & np.isclose(acc_g[:, 8:11], acc_o[:, 8:11], rtol=1e-4, atol=1e-4).all(1))
    assert (~same).mean() <= 1e-4, ((~same).sum(), len(same))


def check_image(acc_g, acc_o, w, h, spp):
    """3 SE on >= 99 % of pixels, means within 1 %, first-hit guides equal; returns (within 3 SE, within 1e-3)."""
    fg, fo = frame_of(acc_g, w, h, spp), frame_of(acc_o, w, h, spp)
    lg, lo = luma(fg.color), luma(fo.color)
    se = np.sqrt(fg.variance + fo.variance)
    ok = np.abs(lg - lo) <= 3 * se + 1e-4 * np.abs(lo) + 1e-6
    assert ok.mean() >= 0.99, ok.mean()
    mg, mo = fg.color.mean((0, 1)), fo.color.mean((0, 1))
    assert np.abs(mg / np.maximum(mo, 1e-12) - 1).max() <= 0.01, (mg, mo)
    first_hit_guides_agree(acc_g, acc_o)
    # Matched seed and samples: both follow the same random numbers, so most pixels take the same paths and agree
    # closely, not only statistically.
    close = np.abs(lg - lo) <= 1e-3 * np.maximum(np.abs(lo), 1e-3)
    return ok.mean(), close.mean()


def test_cornell_box_at_256_16spp_matches_the_oracle(gpu):
    """Config 0 as benched: 256 x 256, 16 spp, depth 5, clamp off, the whole image."""
    P = prep.prepare(scenes.cornell(256, 256))
    spp = 16
    S = gpu.upload(P)
    acc_g, st = S.render_raw(P.params, spp)
    acc_o, so = oracle.Oracle(P).render(P.params, spp)
    S.close()
    assert st.closest_rays == so["closest_rays"], (st.closest_rays, so["closest_rays"])
    within, close = check_image(acc_g, acc_o, 256, 256, spp)
    print(f"cornell 256x256x16: {within:.5f} within 3 SE, {close:.5f} within 1e-3")
    assert close >= 0.9, close


@pytest.fixture(scope="module")
def city(gpu):
    """Config 1 as benched: 4,000 objects, 1,984,402 triangles, 4,002 units, the atmosphere baked on the device."""
    P = prep.prepare(scenes.city(width=CITY_W, height=CITY_H, max_depth=CITY_DEPTH))
    S = gpu.upload(P)  # (the sky is baked on the device and written into P: the oracle reads the same buffers)
    params = prep.set_camera(P.params, scenes.city_camera(CITY_FRAME, 240, 1, CITY_W, CITY_H))
    yield P, S, params
    S.close()


@pytest.mark.parametrize("flags", [0, N.TRT_RENDER_WIDE])
def test_city_trace_at_full_size_matches_the_oracle(gpu, city, flags):
    """Every camera ray of a 720p frame (921,600) and 300,000 rays of every mode from around the camera and inside the
    city's bounds, against the oracle's walk of the same trees."""
    P, S, params = city
    Pf = dataclasses.replace(P, params=params)
    rays = np.concatenate([camera_rays(params, CITY_W, CITY_H), random_rays(Pf, 300000, seed=11, spread=20.0)])
    got = S.trace(params, rays, flags=flags)
    O = oracle.Oracle(P)
    want, _ = O.trace(params, rays)
    both = check_hits(O, params, rays, got, want, min_both=500000)
    if not flags & N.TRT_RENDER_WIDE:  # the binary walks keep the reference's node order: any-hit rays stop alike
        anyhit = (got["tri"] != MISS) & (want["tri"] != MISS) & (rays["mode"] != 0)
        same = (got["tri"][anyhit] == want["tri"][anyhit]) & (got["inst"][anyhit] == want["inst"][anyhit])
        assert anyhit.sum() > 10000 and same.mean() >= 0.9999, (anyhit.sum(), (~same).sum())
    print(f"city trace ({'wide' if flags else 'binary'}): {len(rays)} rays, {both.sum()} closest hits in both")


@pytest.mark.parametrize("flags", [0, N.TRT_RENDER_WIDE])
def test_city_frame_at_720p_matches_the_oracle(gpu, city, flags):
    """The benched frame (1280 x 720, depth 4, sun, atmosphere sky, 400 emitter triangles under the light tree) at
    matched seed: its first sample alone, and 4 samples for the per-pixel standard errors, the whole image."""
    P, S, params = city
    O = oracle.Oracle(P)
    acc1, st1 = S.render_raw(params, 1, flags=flags)
    ref1, so1 = O.render(params, 1)
    assert abs(st1.closest_rays / so1["closest_rays"] - 1) < 1e-4, (st1.closest_rays, so1["closest_rays"])
    assert abs(st1.shadow_rays / so1["shadow_rays"] - 1) < 1e-3, (st1.shadow_rays, so1["shadow_rays"])
    l1g, l1o = luma(acc1[:, 0:3]), luma(ref1[:, 0:3])
    close1 = (np.abs(l1g - l1o) <= 1e-3 * np.maximum(np.abs(l1o), 1e-3)).mean()
    m1g, m1o = acc1[:, 0:3].mean(0), ref1[:, 0:3].mean(0)
    assert np.abs(m1g / m1o - 1).max() <= 0.01, (m1g, m1o)
    first_hit_guides_agree(acc1, ref1)
    spp = 4
    acc_g, _ = S.render_raw(params, spp, flags=flags)
    acc_o, _ = O.render(params, spp)
    within, close = check_image(acc_g, acc_o, CITY_W, CITY_H, spp)
    print(f"city 720p ({'wide' if flags else 'binary'}): 1 spp {close1:.5f} within 1e-3; 4 spp {within:.5f} within "
          f"3 SE, {close:.5f} within 1e-3")
    assert close1 >= 0.9 and close >= 0.85, (close1, close)


@pytest.mark.parametrize("groups,flags", [(1, 0), (1, N.TRT_RENDER_WIDE), (5000, 0)])
def test_crowd_trace_after_deform_matches_the_oracle(gpu, groups, flags):
    """Config 2 at full size (5,000 walkers of 20,160 triangles on a 49,928-triangle ground; one pose group: 70,488
    triangles, 5,000 pose groups: 100,850,328): one frame's records and palettes, trt_deform on the device (skin, leaf
    gather, refit, top rebuild), then the walk against the oracle's on the deformed buffers read back from the device:
    the binary walk, and in one pose group the wide walk too (its BVH refit on the device, its top tree of 5,000 units
    collapsed again). (The deformation itself is checked bit for bit against the oracle's in test_gpu_deform.py.)"""
    c = crowd.crowd(n=5000, groups=groups, width=CITY_W, height=CITY_H, max_depth=3)
    P = prep.prepare(c.desc)
    corners, jobs = crowd.deform_jobs(P, c)
    S = gpu.upload(P)
    S.deform_setup(corners, jobs)
    t = 0.75
    t_inst, _ = crowd.records(P)
    recs = np.ascontiguousarray(crowd.frame_records(P, c, t))
    S.update(3, t_inst * 16, recs)
    st = S.deform(P.params, crowd.palettes(t, c.phase, c.scale), stats=True)
    assert st["errors"] == 0
    params = prep.set_camera(P.params, crowd.crowd_camera(3, CITY_W, CITY_H, c.extent))
    vertices = S.read(0, 0, P.vertices.nbytes, np.float32).reshape(P.vertices.shape)
    leaves = S.read(1, 0, P.leaves.nbytes, np.float32).reshape(P.leaves.shape)
    nodes = S.read(2, 0, P.nodes.nbytes, np.uint32).reshape(P.nodes.shape)
    tables = S.read(3, 0, P.tables.nbytes, np.uint32).reshape(P.tables.shape)
    want_scene = dataclasses.replace(P, vertices=vertices, leaves=leaves, nodes=nodes, tables=tables, params=params)
    rays = np.concatenate([camera_rays(params, CITY_W, CITY_H)[::3],
                           random_rays(want_scene, 200000, seed=13, spread=5.0)])
    got = S.trace(params, rays, flags=flags)
    S.close()
    O = oracle.Oracle(want_scene)
    want, _ = O.trace(params, rays)
    both = check_hits(O, params, rays, got, want, min_both=100000)
    print(f"crowd ({groups} pose groups, {P.info['n_tris']} tris, {'wide' if flags else 'binary'}): {len(rays)} rays, "
          f"{both.sum()} closest hits")


def ulps(got32, truth64):
    """|got - truth| in units of the last place of float32 at the truth."""
    t32 = np.abs(truth64).astype(np.float32)
    spacing = np.spacing(t32).astype(np.float64)
    spacing = np.maximum(spacing, np.float64(np.finfo(np.float32).smallest_subnormal))
    return np.abs(got32.astype(np.float64) - truth64) / spacing


def test_device_transcendentals_within_their_documented_ulps(gpu):
    """cosf, sinf, acosf and atan2f as the shading calls them, over the arguments it gives them (sampled angles in
    [0, 2 pi), polar angles in [0, pi], cosines in [-1, 1], direction components), against float64 truth. The bounds
    are CUDA's documented maximum errors for these functions (sinf, cosf, acosf: 2 ulp; atan2f: 3 ulp), so the image
    can differ from the oracle's (IEEE libm, within an ulp) only by that much in those functions' results."""
    rng = np.random.default_rng(17)
    phi = np.concatenate([np.linspace(0, 2 * np.pi, 1 << 20, endpoint=False, dtype=np.float32),
                          (2 * np.pi * rng.random(1 << 18)).astype(np.float32)])
    report = {}
    for fn, ref, name in ((N.TRT_MATH_COS, np.cos, "cosf"), (N.TRT_MATH_SIN, np.sin, "sinf")):
        got = gpu.math_eval(fn, phi)
        truth = ref(phi.astype(np.float64))
        err = ulps(got, truth)
        report[name] = float(err.max())
        assert err.max() <= 2.0, (name, err.max(), phi[np.argmax(err)])
    c = np.concatenate([np.linspace(-1, 1, 1 << 20, dtype=np.float32), rng.uniform(-1, 1, 1 << 18).astype(np.float32),
                        np.float32([-1.0, 1.0, 0.0])])
    err = ulps(gpu.math_eval(N.TRT_MATH_ACOS, c), np.arccos(c.astype(np.float64)))
    report["acosf"] = float(err.max())
    assert err.max() <= 2.0, err.max()
    d = rng.normal(size=(1 << 20, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    x, z = d[:, 0].astype(np.float32), (-d[:, 2]).astype(np.float32)
    err = ulps(gpu.math_eval(N.TRT_MATH_ATAN2, x, z), np.arctan2(x.astype(np.float64), z.astype(np.float64)))
    report["atan2f"] = float(err.max())
    assert err.max() <= 3.0, err.max()
    print("max ulps:", report)
