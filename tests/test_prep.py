"""The host prep against the reference's own tests of the builders it restates: bvh.rs:410-458 (garbage in, the
depth cap), lib.rs:1145-1200 (the energy table), lib.rs:1459-1505 (the emitter guide table), ltree.rs's checks (every
entry's code leads to its leaf), units.rs:231-248 (mesh trees within MESH_DEPTH)."""
import ctypes as C
import math

import numpy as np
import pytest

from threert_b200 import _native as N
from threert_b200 import prep, scenes


def build_bvh(tris, max_depth=48):
    L = N.lib()
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    cap = max(16, 4 * len(t) + 4)
    nodes = np.zeros((cap, 8), np.uint32)
    order = np.zeros(max(1, len(t)), np.uint32)
    depth = C.c_uint32()
    n = L.trt_prep_bvh(t.ctypes.data_as(C.POINTER(C.c_float)), len(t), max_depth,
                       nodes.ctypes.data_as(C.POINTER(C.c_uint32)), cap, order.ctypes.data_as(C.POINTER(C.c_uint32)),
                       C.byref(depth))
    assert n > 0, L.trt_prep_last_error()
    return nodes[:n], order[:len(t)], depth.value


def check_tree(nodes, max_depth, max_leaf, n_items):
    L = N.lib()
    nodes = np.ascontiguousarray(nodes, np.uint32)
    d = C.c_uint32()
    rc = L.trt_prep_check_tree(nodes.ctypes.data_as(C.POINTER(C.c_uint32)), len(nodes), max_depth, max_leaf, n_items,
                               C.byref(d))
    return rc, d.value


def stream(seed):
    s = [seed]

    def f():
        s[0] = (s[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return (s[0] >> 8) / float(1 << 24)
    return f


def test_garbage_in_makes_a_tree_the_kernel_walks():
    rnd = stream(11)
    p = lambda s: np.array([rnd() - 0.5, rnd() - 0.5, rnd() - 0.5]) * s
    good = []
    for _ in range(600):
        c = p(20.0)
        good.append([c + p(1.0), c + p(1.0), c + p(1.0)])
    good = np.array(good, np.float32)
    mixed = good.copy()
    for k in range(0, len(mixed), 7):
        mixed[k, k % 3] = [np.nan, 0, 0] if k % 2 == 0 else [0, np.inf, 0]
    cases = {
        "mixed": mixed,
        "all bad": np.array([[[np.nan, 0, 0], [0, 0, 0], [1, 1, 1]], [[0, 0, 0], [0, np.inf, 0], [1, 1, 1]],
                             [[-np.inf] * 3, [0, 0, 0], [1, 1, 1]]], np.float32),
        "near the limit": np.array([[[3e38 * s] * 3, [1.5e38 * s] * 3, [0, 0, 0]] for s in [1, -1] * 100], np.float32),
        "one triangle a thousand times": np.repeat(good[:1], 1000, 0),
        "a needle": np.array([[[k * 1e-3, 0, 0], [k * 1e-3, 1e-4, 0], [k * 1e-3, 0, 1e-4]] for k in range(500)], np.float32),
    }
    for what, tris in cases.items():
        nodes, order, depth = build_bvh(tris)
        finite = np.isfinite(tris).all(axis=(1, 2))
        n_good = int(finite.sum())
        rc, d = check_tree(nodes, 48, 16, max(n_good, 1))
        assert rc == 0, what
        # Items whose box is not finite come last, in no leaf.
        assert sorted(order[n_good:].tolist()) == sorted(np.nonzero(~finite)[0].tolist()), what


def test_a_tree_is_no_deeper_than_its_stack():
    tris = np.array([[[2.0 ** k, 0, 0], [2.0 ** k, 1, 0], [2.0 ** k, 0, 1]] for k in range(120)], np.float32)
    free_nodes, free_order, free_depth = build_bvh(tris, 1000)
    assert free_depth > 20
    for cap in (8, 12, 20):
        _, _, d = build_bvh(tris, cap)
        assert d <= cap
    roomy_nodes, roomy_order, roomy_depth = build_bvh(tris, free_depth)
    assert roomy_depth == free_depth and (roomy_order == free_order).all() and (roomy_nodes == free_nodes).all()


def specular_albedo(mu, alpha, nr=48, nphi=8):
    out = (C.c_double * 2)()
    N.lib().trt_prep_specular_albedo(mu, alpha, nr, nphi, out)
    return out[0], out[1]


def quadrature(mu, alpha, n):
    """lib.rs:1125-1142: the lobe's value x cosine over the hemisphere at F = 1, midpoint rule."""
    a2 = alpha * alpha
    v = (math.sqrt(1 - mu * mu), mu)
    i = (np.arange(n) + 0.5) / n * (math.pi / 2)
    j = math.pi * (np.arange(2 * n) + 0.5) / (2 * n)
    st, c = np.sin(i)[:, None], np.cos(i)[:, None]
    x, z = st * np.cos(j)[None, :], st * np.sin(j)[None, :]
    h0, h1, h2 = v[0] + x, v[1] + c, z
    noh = h1 / np.sqrt(h0 * h0 + h1 * h1 + h2 * h2)
    d = (noh * a2 - noh) * noh + 1.0
    vis = 0.5 / (c * (mu * (1 - alpha) + alpha) + mu * (c * (1 - alpha) + alpha))
    s = (a2 / (math.pi * d * d) * vis * c * st).sum()
    return s * math.pi * math.pi / (2 * n * n)


def test_the_albedo_is_the_lobes_integral():
    for r, mu in [(0.3, 0.9), (0.5, 0.7071), (0.5, 0.2), (0.8, 0.5), (1.0, 1.0), (1.0, 0.1), (0.25, 0.4)]:
        a, b = specular_albedo(mu, r * r)
        q = quadrature(mu, r * r, 800)
        assert abs(a + b - q) < 1e-3, (r, mu, a + b, q)
    a, b = specular_albedo(0.5, 0.0)
    assert abs(a + b - 1) < 1e-12 and abs(b - 0.5 ** 5) < 1e-12
    a, b = specular_albedo(0.5, 0.02 * 0.02)
    assert abs(a + b - 1) < 2e-3 and abs(b - 0.5 ** 5) < 2e-3


def energy_table(P):
    first = int(P.params[124 + 9])
    t = P.tables.view(np.float32).reshape(-1, 4)[first:first + 512]
    return t.reshape(-1, 2)  # node i: (a, b)


def test_the_table_follows_the_albedo_between_its_nodes():
    d, _ = scenes.emissive_nits()
    lut = energy_table(prep.prepare(d))
    assert lut.shape == (1024, 2)
    assert np.all((lut >= 0) & (lut <= 1 + 1e-4))
    n = 32

    def lookup(r, mu):  # pathtrace.wgsl:1452-1461
        x, y = math.sqrt(min(max(mu, 0), 1)) * (n - 1), min(max(r, 0), 1) * (n - 1)
        x0, y0 = min(int(x), n - 2), min(int(y), n - 2)
        fx, fy = x - x0, y - y0
        i = y0 * n + x0
        mix = lambda p, q, t: p + (q - p) * t
        return mix(mix(lut[i], lut[i + 1], fx), mix(lut[i + n], lut[i + n + 1], fx), fy)
    worst, total = 0.0, 0.0
    for iy in range(48):
        r = 0.02 + 0.98 * (iy + 0.37) / 48
        for ix in range(48):
            mu = 0.01 + 0.99 * (ix + 0.61) / 48
            a, b = specular_albedo(mu, r * r, 96, 12)
            ta, tb = lookup(r, mu)
            e = max(abs(ta - a), abs(tb - b), abs(ta + tb - a - b) / (a + b))
            total += e / (48 * 48)
            worst = max(worst, e)
    assert worst < 0.02 and total < 0.002, (worst, total)


def many_emitters_scene(n=3000, light_tree=False):
    """3000 emitting triangles over six decades of area, some black (lib.rs:1459-1470's set-up)."""
    rnd = stream(11)
    tris, secs = [], []
    for i in range(n):
        s = 10 ** (-3.0 * rnd())
        c = np.array([300 * rnd(), 5.0, 100 * rnd()])
        tris.append([c, c + [s, 0, 0], c + [0, 0, s]])
        secs.append(0 if i % 9 == 0 else 1 + i % 3)
    mats = [prep.Material(emissive=(k * 3.0, k * 1.0, 0.5 * k)) for k in range(4)]
    mesh = prep.Mesh(np.array(tris, np.float32), sections=np.array(secs, np.uint32), n_sections=4)
    cam = prep.Camera.look_at((0, 50, 0), (1, 0, 1), 40, 16, 16)
    return prep.SceneDescription([mesh], mats, [prep.Instance(0, [0, 1, 2, 3])], cam, light_tree=light_tree)


def test_emitter_guide_finds_what_the_full_search_finds():
    P = prep.prepare(many_emitters_scene())
    n = int(P.params[21])
    first = int(P.params[124 + 4])
    t = P.tables.view(np.float32).reshape(-1, 4)[first:]
    tu = P.tables.reshape(-1, 4)[first:]
    header = n + (65536 + 1 + 3) // 4
    total = t[header, 0]
    assert total > 0 and np.all(t[header, 1:] == 0)
    cum = t[:n, 1]
    assert np.all(np.diff(cum) >= 0)
    guide = tu[n:header].reshape(-1)

    def search(lo, hi, u):
        return min(int(np.searchsorted(cum[lo:hi], u, side="left")) + lo, n - 1)
    rnd = stream(5)
    us = [int(rnd() * (1 << 24)) for _ in range(20000)]
    for k in range(0, 65537, 7):
        m = k << 8
        us += [x for x in (m - 1, m, m + 1) if 0 <= x < (1 << 24)]
    us += [min(int(c * (1 << 24)), (1 << 24) - 1) for c in cum]
    for m in us:
        u = np.float32(m / float(1 << 24))
        k = min(int(u * np.float32(65536)), 65535)
        assert search(int(guide[k]), int(guide[k + 1]), u) == search(0, n, u)


def test_light_tree_codes_lead_to_their_leaves():
    P = prep.prepare(many_emitters_scene(light_tree=True))
    nodes = P.tables.reshape(-1, 4)  # the light tree is the tables' first section
    codes = P.info["light_tree_codes"]
    assert len(codes) > 256
    LEAF = 0x80000000
    for k, c in enumerate(codes):
        depth = (int(c) >> 26) - 1
        i = 0
        for level in range(depth):
            w = int(nodes[i, 3])
            assert not (w & LEAF)
            i = w + ((int(c) >> level) & 1)
        w = int(nodes[i, 3])
        assert w & LEAF and (w & 0x1FFFFFFF) <= k < (w & 0x1FFFFFFF) + ((w >> 29) & 3) + 1


def test_scene_facts():
    P = prep.prepare(scenes.cornell())
    assert P.info["n_tris"] == 36 and P.info["n_units"] == 8 and P.info["n_emitters"] == 2
    assert P.info["light_tree_nodes"] == 0 and P.info["env_sampled"] == 0
    assert P.params.nbytes == 624
    d = scenes.city(n_objects=60, n_emitters=300, width=64, height=36)
    P = prep.prepare(d)
    assert P.info["n_units"] == 62 and P.info["n_emitters"] == 600 and P.info["light_tree_nodes"] > 0
    assert P.info["max_mesh_depth"] <= 45 and P.info["top_depth"] <= 18


def test_prep_refuses_bad_scenes():
    d = scenes.cornell()
    d.instances[0].mesh = 99
    with pytest.raises(ValueError):
        prep.prepare(d)
    d = scenes.cornell()
    d.meshes[0].positions = d.meshes[0].positions.copy()
    d.meshes[0].positions[0, 0, 0] = np.nan
    with pytest.raises(ValueError):
        prep.prepare(d)
