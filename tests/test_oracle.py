"""The oracle against known answers: the reference's analytic render tests (tests/render/*.ts, values and
tolerances as they state them) and its traversal's brute-force parity (renderer/src/units.rs:1442-1535: the walk's
closest t bit-identical to a test of every triangle, the same triangle unless two share that t; any-hit agrees on
hit / no hit)."""
import numpy as np
import pytest

import oracle
from threert_b200 import prep, scenes

from util import luma, random_rays, region_mean, scaled_units_scene, small_city

SPP = 64


def center_radiance(d, spp=SPP):
    P = prep.prepare(d)
    w, h = P.width, P.height
    px = scenes.region_pixels(w, h, scenes.CENTER)
    acc, _ = oracle.Oracle(P).render(P.params, spp, pixels=px)
    return region_mean(acc, w, h, spp, scenes.CENTER)


@pytest.mark.parametrize("name,tol", [("furnace_diffuse", 0.02), ("directional_lambert", 0.02),
                                      ("emissive_nits", 0.01), ("emitter_grid", 0.02), ("furnace_metal", 0.03)])
def test_analytic_scene(name, tol):
    d, expected = getattr(scenes, name)()
    got = luma(center_radiance(d))
    assert abs(got / expected - 1) <= tol, (name, got, expected)


def test_emitter_far():
    d, expected = scenes.emitter_grid(step=2.0, height=150.0, side=1.0, nits=10000.0)
    got = luma(center_radiance(d, 256))
    assert abs(got / expected - 1) <= 0.02, (got, expected)


def test_metal_f0():
    d, expected = scenes.metal_f0()
    got = center_radiance(d)
    assert np.all(np.abs(got / np.array(expected) - 1) <= 0.03), got


def test_shadow_directional():
    d, ra, rb = scenes.shadow_directional()
    P = prep.prepare(d)
    w, h = P.width, P.height
    acc, _ = oracle.Oracle(P).render(P.params, SPP)
    a, b = luma(region_mean(acc, w, h, SPP, ra)), luma(region_mean(acc, w, h, SPP, rb))
    assert b > 0 and abs(a / b) <= 0.005, (a, b)


@pytest.mark.parametrize("make", [small_city, scaled_units_scene, scenes.cornell])
def test_the_walk_is_the_brute_force(make):
    P = prep.prepare(make())
    O = oracle.Oracle(P)
    rays = random_rays(P, 6000, seed=1, spread=2.0)
    walk, _ = O.trace(P.params, rays)
    brute, _ = O.trace(P.params, rays, brute=True)
    closest = rays["mode"] == 0
    hit_w, hit_b = walk["tri"] != 0xFFFFFFFF, brute["tri"] != 0xFFFFFFFF
    assert (hit_w == hit_b).all()
    c = closest & hit_w
    # t bit-identical to the brute force's, apart from coplanar triangles of two units a few ulps apart through
    # their transforms (the mesh tree's own slab test may prune the later one): within 1e-6 relative there.
    exact = walk["t"][c].view(np.uint32) == brute["t"][c].view(np.uint32)
    assert exact.mean() >= 0.995
    assert np.all(np.abs(walk["t"][c] / brute["t"][c] - 1) <= 1e-6)
    # The same triangle, unless two share that t: then the walk's own triangle lies at it too (an edge tie).
    differ = c & ((walk["tri"] != brute["tri"]) | (walk["inst"] != brute["inst"]))
    t_own = O.intersect(P.params, rays[differ], walk[differ])
    assert np.array_equal(t_own.view(np.uint32), walk["t"][differ].view(np.uint32))
    assert (~differ[c]).mean() >= 0.99
    assert hit_w.sum() > 100


def test_accumulation_is_additive():
    """Two renders of 4 samples each from sample 0 and 4 equal one of 8 (the resume the sample index allows)."""
    P = prep.prepare(scenes.cornell(width=24, height=24))
    O = oracle.Oracle(P)
    a8, _ = O.render(P.params, 8)
    a4, _ = O.render(P.params, 4)
    a4, _ = O.render(P.params, 4, first_sample=4, accum=a4)
    assert np.allclose(a8, a4, rtol=1e-5, atol=1e-6)
