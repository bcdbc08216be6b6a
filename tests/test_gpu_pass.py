"""The CUDA pass against the CPU oracle, through the C ABI, on the same seeded scenes and buffers.

Traversal: hit triangle identical on >= 99.99 % of rays (edge ties aside), t within 1e-6 relative. Images at
matched seed and spp: per-pixel luminance within 3 combined standard errors on >= 99 % of pixels, the image means
within 1 %. Known answers: the reference's analytic render tests, full frames on the GPU."""
import numpy as np
import pytest

import oracle
from threert_b200 import RenderError, prep, scenes
from threert_b200 import _native as N
from threert_b200.gpu import frame_of

from util import luma, random_rays, region_mean, scaled_units_scene, small_city

pytestmark = pytest.mark.gpu


def trace_parity(gpu, P, flags, n=20000):
    S = gpu.upload(P)
    rays = random_rays(P, n, seed=7, spread=2.0)
    got = S.trace(P.params, rays, flags=flags)
    want, _ = oracle.Oracle(P).trace(P.params, rays)
    S.close()
    O = oracle.Oracle(P)
    hit_g, hit_w = got["tri"] != 0xFFFFFFFF, want["tri"] != 0xFFFFFFFF
    assert (hit_g == hit_w).mean() >= 0.9999
    both = hit_g & hit_w & (rays["mode"] == 0)
    rel = np.abs(got["t"][both] / want["t"][both] - 1)
    assert rel.max() <= 1e-6, rel.max()
    # The same triangle on >= 99.99 % of rays; where not, an exact tie: the GPU's own triangle lies at the same t.
    differ = both & ((got["tri"] != want["tri"]) | (got["inst"] != want["inst"]))
    t_own = O.intersect(P.params, rays[differ], got[differ])
    tie = np.abs(t_own / want["t"][differ] - 1) <= 1e-6
    assert (differ.sum() - tie.sum()) <= 1e-4 * both.sum(), (differ.sum(), tie.sum())
    # Any-hit rays stop at the first triangle the walk meets. The binary walks (the shadow walk's split loop included)
    # keep the reference's node order, so it is the oracle's own; the wide walk orders a node's children by the ray's
    # octant, so only its hit or miss is the reference's.
    if not flags & N.TRT_RENDER_WIDE:
        anyhit = hit_g & hit_w & (rays["mode"] != 0)
        same = (got["tri"][anyhit] == want["tri"][anyhit]) & (got["inst"][anyhit] == want["inst"][anyhit])
        assert same.mean() >= 0.9999, (anyhit.sum(), (~same).sum())
    return both.sum()


@pytest.mark.parametrize("make", [small_city, scaled_units_scene, scenes.cornell])
@pytest.mark.parametrize("flags", [0, N.TRT_RENDER_WIDE])
def test_trace_matches_the_oracle(gpu, make, flags):
    assert trace_parity(gpu, prep.prepare(make()), flags) > 500


def image_parity(acc_g, acc_o, w, h, spp):
    fg, fo = frame_of(acc_g, w, h, spp), frame_of(acc_o, w, h, spp)
    lg, lo = luma(fg.color), luma(fo.color)
    se = np.sqrt(fg.variance + fo.variance)
    ok = np.abs(lg - lo) <= 3 * se + 1e-4 * np.abs(lo) + 1e-6
    mg, mo = fg.color.mean((0, 1)), fo.color.mean((0, 1))
    return ok.mean(), np.abs(mg / np.maximum(mo, 1e-12) - 1).max()


@pytest.mark.parametrize("flags", [0, N.TRT_RENDER_WIDE])
@pytest.mark.parametrize("make,spp", [(lambda: scenes.cornell(64, 64), 16), (small_city, 4),
                                      (lambda: small_city(sky="atmosphere"), 4), (scaled_units_scene, 4)])
def test_render_matches_the_oracle(gpu, make, spp, flags):
    P = prep.prepare(make())
    w, h = P.width, P.height
    acc_g = gpu.upload(P).render_raw(P.params, spp, flags=flags)[0]
    acc_o, st = oracle.Oracle(P).render(P.params, spp)
    assert st["tri_tests"] > w * h and st["shadow_rays"] > w * h // 4  # the camera sees the scene
    frac, mean_err = image_parity(acc_g, acc_o, w, h, spp)
    assert frac >= 0.99, frac
    assert mean_err <= 0.01, mean_err
    # albedo and normal sums are first-hit data: equal up to the shading's rounding
    assert np.allclose(acc_g[:, 4:7], acc_o[:, 4:7], rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("name,tol", [("furnace_diffuse", 0.02), ("directional_lambert", 0.02),
                                      ("emissive_nits", 0.01), ("emitter_grid", 0.02), ("furnace_metal", 0.03)])
def test_analytic_scene_on_the_gpu(gpu, name, tol):
    d, expected = getattr(scenes, name)()
    P = prep.prepare(d)
    f = gpu.render(P, P.params, 64)
    px = scenes.region_pixels(P.width, P.height, scenes.CENTER)
    got = luma(f.color.reshape(-1, 3)[px].mean(0))
    assert abs(got / expected - 1) <= tol, (name, got, expected)


def test_shadow_on_the_gpu(gpu):
    d, ra, rb = scenes.shadow_directional()
    P = prep.prepare(d)
    acc = gpu.upload(P).render_raw(P.params, 64)[0]
    a, b = luma(region_mean(acc, P.width, P.height, 64, ra)), luma(region_mean(acc, P.width, P.height, 64, rb))
    assert b > 0 and abs(a / b) <= 0.005


def test_resume_by_sample_range(gpu):
    """8 samples at once equal 4 then 4 more from sample 4 (TRT_RENDER_ACCUMULATE), bit for bit."""
    P = prep.prepare(scenes.cornell(48, 48))
    S = gpu.upload(P)
    a8 = S.render_raw(P.params, 8)[0]
    S.render_raw(P.params, 4, read=False)
    a44 = S.render_raw(P.params, 4, first_sample=4, flags=N.TRT_RENDER_ACCUMULATE)[0]
    assert np.array_equal(a8, a44)


SORTS = N.TRT_RENDER_SORT_RAYS | N.TRT_RENDER_SORT_SHADOWS


@pytest.mark.parametrize("walk", [0, N.TRT_RENDER_WIDE])
@pytest.mark.parametrize("sorts", [N.TRT_RENDER_SORT_RAYS, N.TRT_RENDER_SORT_SHADOWS, SORTS])
@pytest.mark.parametrize("make,spp", [(small_city, 3), (lambda: scenes.cornell(64, 64), 8)])
def test_sorted_queues_render_the_same_image(gpu, make, spp, sorts, walk):
    """A path's state, hit and random numbers are its own, so the coherence sorts change no bit of the image."""
    P = prep.prepare(make())
    S = gpu.upload(P)
    plain, st0 = S.render_raw(P.params, spp, flags=walk | N.TRT_RENDER_UNSORTED_HITS)
    # hits sorted by material too where the scene has more than 32 materials (the small city's 221; not the Cornell box)
    got, st1 = S.render_raw(P.params, spp, flags=walk | sorts)
    assert np.array_equal(plain, got)
    assert (st0.closest_rays, st0.shadow_rays, st0.paths) == (st1.closest_rays, st1.shadow_rays, st1.paths)


def test_counts_match_the_oracles_rays(gpu):
    P = prep.prepare(small_city())
    S = gpu.upload(P)
    _, st = S.render_raw(P.params, 2)
    _, so = oracle.Oracle(P).render(P.params, 2)
    assert st.closest_rays == so["closest_rays"] and st.paths == P.width * P.height * 2
    assert abs(st.shadow_rays / so["shadow_rays"] - 1) < 0.01


def test_bad_params_are_refused(gpu):
    P = prep.prepare(scenes.cornell(16, 16))
    S = gpu.upload(P)
    bad = P.params.copy()
    bad[124 + 7] = 1 << 30  # the instances' section past the tables
    with pytest.raises(RenderError, match="TRT_EINVAL"):
        S.render_raw(bad, 1)
    bad = P.params.copy()
    bad[22] = 100  # max bounces past the pass's counters
    with pytest.raises(RenderError, match="TRT_EINVAL"):
        S.render_raw(bad, 1)
    S.render_raw(P.params, 1)  # still usable


def test_a_cycle_in_the_tree_trips_the_guard(gpu):
    """A top tree whose root names itself as its left child: the walk stops at its iteration limit and the render
    reports it (the reference's loop guard, gpu.rs:4199-4205), without hanging or faulting."""
    P = prep.prepare(scenes.cornell(8, 8))
    top = int(P.params[70])
    P.nodes = P.nodes.copy()
    P.nodes[top, 3] = 0   # left_or_first 0: children top, top + 1
    P.nodes[top, 7] = 0
    S = gpu.upload(P)
    with pytest.raises(RenderError, match="TRT_EGUARD"):
        S.render_raw(P.params, 1)


def test_asynchronous_readback_gives_each_frame_its_accum(gpu):
    """TRT_RENDER_ASYNC_READBACK: three renders queued back to back, each copied to its own pinned buffer while the
    next renders into the scene's other accum; after trt_synchronize each buffer holds its frame's accum, bit for bit
    the synchronous render's. It does not combine with TRT_RENDER_ACCUMULATE."""
    import ctypes as C
    import torch
    P = prep.prepare(scenes.cornell(48, 48))
    S = gpu.upload(P)
    params = [np.ascontiguousarray(prep.params_with(P.params, seed=sd), np.uint32) for sd in (1, 2, 3)]
    want = [S.render_raw(p, 2)[0].copy() for p in params]
    bufs = [torch.zeros((48 * 48, N.PIXEL_FLOATS), dtype=torch.float32, pin_memory=True) for _ in params]
    L = N.lib()
    for p, b in zip(params, bufs):
        rc = L.trt_render(S.handle, p.ctypes.data_as(C.POINTER(C.c_uint32)), 0, 2, N.TRT_RENDER_ASYNC_READBACK,
                          C.cast(b.data_ptr(), C.POINTER(C.c_float)), None)
        assert rc == 0
    gpu.synchronize()
    for w, b in zip(want, bufs):
        assert np.array_equal(b.numpy(), w)
    assert np.array_equal(S.render_raw(params[1], 2)[0], want[1])  # a synchronous render after them
    with pytest.raises(RenderError, match="TRT_EINVAL"):
        S.render_raw(params[0], 2, flags=N.TRT_RENDER_ASYNC_READBACK | N.TRT_RENDER_ACCUMULATE)
    S.close()
