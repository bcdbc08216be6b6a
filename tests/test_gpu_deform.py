"""The per-frame deformation on the device (trt_deform) against the oracle: skinned vertices, gathered leaves and
refit mesh trees bit for bit (renderer/shaders/skin.wgsl, leaf_gather.wgsl, units.rs refit), the top tree node for
node as units.rs top_tree builds it over the same unit boxes, two frames in a row; then the render and the walk of
the deformed scene against the oracle on the same buffers."""
import dataclasses

import numpy as np
import pytest

import oracle
from threert_b200 import RenderError, crowd, prep
from threert_b200 import _native as N
from threert_b200.gpu import frame_of

from util import luma, random_rays, small_crowd

pytestmark = pytest.mark.gpu


def make_scene(n=160):
    c = small_crowd(n=n)
    P = prep.prepare(c.desc)
    corners, jobs = crowd.deform_jobs(P, c)
    return c, P, corners, jobs


@pytest.fixture(scope="module")
def scene():
    return make_scene()


def run_frame(S, P, c, t):
    t_inst, _ = crowd.records(P)
    recs = crowd.frame_records(P, c, t)
    S.update(3, t_inst * 16, recs)
    pal = crowd.palettes(t, c.phase, c.scale)
    st = S.deform(P.params, pal)
    return recs, pal, st


def oracle_frame(P, c, corners, jobs, recs, pal):
    """What the frame's buffers must hold: the oracle's skin, gather and refit, and the prep's top tree."""
    t_inst, _ = crowd.records(P)
    tables = P.tables.copy()
    tables[4 * t_inst: 4 * t_inst + 40 * c.n] = recs.ravel()
    w_ind = int(P.params[136 + 4])
    v, lv, nd = oracle.deform(jobs, corners, pal.reshape(-1, 12), P.vertices, P.leaves, P.nodes, P.words, w_ind)
    units = int(P.params[68 + 3])
    rec = tables[4 * t_inst: 4 * t_inst + 40 * units].reshape(units, 40)
    worlds = rec[:, 0:12].view(np.float32).reshape(units, 3, 4)
    f = nd.view(np.float32)
    boxes = np.concatenate([f[rec[:, 15], 0:3], f[rec[:, 15], 4:7]], 1)
    top, _ = prep.units_top(worlds, boxes)
    first = int(P.params[68 + 2])
    nd[first:first + 2 * units - 1] = top
    return dataclasses.replace(P, vertices=v, leaves=lv, nodes=nd, tables=tables)


def read_back(S, P):
    return (S.read(0, 0, P.vertices.nbytes, np.float32).reshape(P.vertices.shape),
            S.read(1, 0, P.leaves.nbytes, np.float32).reshape(P.leaves.shape),
            S.read(2, 0, P.nodes.nbytes, np.uint32).reshape(P.nodes.shape))


@pytest.mark.parametrize("n", [160, 700])  # 700: the top build's first levels take the CTA-wide kernel
def test_deform_matches_the_oracle(gpu, n):
    c, P, corners, jobs = make_scene(n)
    S = gpu.upload(P)
    S.deform_setup(corners, jobs)
    for t in (0.4, 1.3):  # two frames: the refit's counters are zero again after each
        recs, pal, st = run_frame(S, P, c, t)
        assert st["errors"] == 0
        want = oracle_frame(P, c, corners, jobs, recs, pal)
        v, lv, nd = read_back(S, P)
        assert np.array_equal(v, want.vertices)
        assert np.array_equal(lv, want.leaves)
        # boxes as floats (a zero's sign may differ between folds), links and counts as words
        assert np.array_equal(nd.view(np.float32)[:, [0, 1, 2, 4, 5, 6]], want.nodes.view(np.float32)[:, [0, 1, 2, 4, 5, 6]])
        assert np.array_equal(nd[:, [3, 7]], want.nodes[:, [3, 7]])
    S.close()


def test_render_after_deform_matches_the_oracle(gpu, scene):
    c, P, corners, jobs = scene
    S = gpu.upload(P)
    S.deform_setup(corners, jobs)
    recs, pal, _ = run_frame(S, P, c, 0.8)
    want = oracle_frame(P, c, corners, jobs, recs, pal)
    spp = 4
    acc_g = S.render_raw(P.params, spp)[0]
    acc_o, st = oracle.Oracle(want).render(P.params, spp)
    assert st["tri_tests"] > P.width * P.height
    fg, fo = frame_of(acc_g, P.width, P.height, spp), frame_of(acc_o, P.width, P.height, spp)
    se = np.sqrt(fg.variance + fo.variance)
    ok = np.abs(luma(fg.color) - luma(fo.color)) <= 3 * se + 1e-4 * np.abs(luma(fo.color)) + 1e-6
    assert ok.mean() >= 0.99
    assert np.allclose(acc_g[:, 4:7], acc_o[:, 4:7], rtol=1e-4, atol=1e-5)
    # the walk of the deformed scene: the oracle's hits on the same rays
    rays = random_rays(want, 20000, seed=5, spread=2.0)
    got = S.trace(P.params, rays)
    ref, _ = oracle.Oracle(want).trace(P.params, rays)
    hg, hw = got["tri"] != 0xFFFFFFFF, ref["tri"] != 0xFFFFFFFF
    assert (hg == hw).mean() >= 0.9999
    both = hg & hw & (rays["mode"] == 0)
    assert both.sum() > 1000
    assert np.abs(got["t"][both] / ref["t"][both] - 1).max() <= 1e-6
    assert ((got["tri"] == ref["tri"]) | ~both).mean() >= 0.9999
    # the wide walk, built now from the uploaded copies and brought to the deformed buffers on the device
    check_walk(S.trace(P.params, rays, flags=N.TRT_RENDER_WIDE), ref, rays)
    S.close()


def check_walk(got, ref, rays):
    """Hit or miss on >= 99.99 % of rays, t within 1e-6, the same triangle on >= 99.99 % of closest hits."""
    hg, hw = got["tri"] != 0xFFFFFFFF, ref["tri"] != 0xFFFFFFFF
    assert (hg == hw).mean() >= 0.9999, (hg != hw).sum()
    both = hg & hw & (rays["mode"] == 0)
    assert both.sum() > 1000
    assert np.abs(got["t"][both] / ref["t"][both] - 1).max() <= 1e-6
    assert ((got["tri"] == ref["tri"]) | ~both).mean() >= 0.9999


@pytest.mark.parametrize("n", [160, 700])
def test_wide_walk_follows_each_deformation(gpu, n):
    """A wide BVH in use is refit by each trt_deform on the device (its mesh nodes quantised again over the refit
    boxes, its triangle copies gathered again, the rebuilt top tree collapsed again): three frames in a row, each
    walked against the oracle on the frame's buffers; a wide BVH first built after the deformations (from the uploaded
    copies, then refit) gives the same hits bit for bit."""
    c, P, corners, jobs = make_scene(n)
    S = gpu.upload(P)
    S.deform_setup(corners, jobs)
    probe = random_rays(P, 1000, seed=1, spread=2.0)
    S.trace(P.params, probe, flags=N.TRT_RENDER_WIDE)  # built before the first deformation
    for i, t in enumerate((0.4, 1.3, 2.2)):
        recs, pal, st = run_frame(S, P, c, t)
        assert st["errors"] == 0 and st["wide_ms"] > 0, st
        want = oracle_frame(P, c, corners, jobs, recs, pal)
        rays = random_rays(want, 20000, seed=20 + i, spread=2.0)
        ref, _ = oracle.Oracle(want).trace(P.params, rays)
        got = S.trace(P.params, rays, flags=N.TRT_RENDER_WIDE)
        check_walk(got, ref, rays)
        binary = S.trace(P.params, rays)
        same = (got["tri"] != 0xFFFFFFFF) == (binary["tri"] != 0xFFFFFFFF)
        assert same.mean() >= 0.9999
    # the same three frames on a second scene whose wide BVH is built only after them
    S2 = gpu.upload(P)
    S2.deform_setup(corners, jobs)
    for t in (0.4, 1.3, 2.2):
        _, _, st = run_frame(S2, P, c, t)
        assert st["wide_ms"] == 0
    got2 = S2.trace(P.params, rays, flags=N.TRT_RENDER_WIDE)
    for f in ("tri", "inst", "t"):
        assert np.array_equal(got2[f], got[f]), f
    # a frame rendered with the wide walk: first-hit albedo and normals as the binary walk's
    acc_w = S2.render_raw(P.params, 1, flags=N.TRT_RENDER_WIDE)[0]
    acc_b = S2.render_raw(P.params, 1)[0]
    same = np.isclose(acc_w[:, 4:7], acc_b[:, 4:7], rtol=1e-4, atol=1e-5).all(1)
    assert same.mean() >= 0.999, (~same).sum()
    S.close()
    S2.close()


def test_deform_refuses_what_it_cannot_do(gpu, scene):
    c, P, corners, jobs = scene
    S = gpu.upload(P)
    with pytest.raises(RenderError):  # no setup yet
        S.deform(P.params, crowd.palettes(0.0, c.phase, c.scale))
    bad = jobs.copy()
    bad[0, 7] += 5  # nodes past the tree: its last nodes are not the children of one node
    with pytest.raises(RenderError):
        S.deform_setup(corners, bad)
    bad = jobs.copy()
    bad[0, 2] = len(corners)  # corners past those given
    with pytest.raises(RenderError):
        S.deform_setup(corners, bad)
    S.deform_setup(corners, jobs)
    with pytest.raises(RenderError):  # a palette too short for the last group
        S.deform(P.params, crowd.palettes(0.0, c.phase[:1], c.scale[:1]))
    # a node written after setup: set up again first
    S.update(2, 0, P.nodes[:1])
    with pytest.raises(RenderError):
        S.deform(P.params, crowd.palettes(0.0, c.phase, c.scale))
    S.close()
