"""The emitters' re-weigh on the device (trt_scene_weigh_emitters) against the oracle's restatement of
emitter_weights.wgsl: the whole tables bit for bit after an edit of the emitters' materials, with and without the
light LOD; then the pass renders the re-weighed scene as the oracle does."""
import numpy as np
import pytest

import oracle
from threert_b200 import prep

from test_emitters import scale_emitters
from util import small_city

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lod", [False, True])
def test_device_reweigh_is_the_oracles(gpu, lod):
    P = prep.prepare(small_city())
    S = gpu.upload(P)
    edited, _ = scale_emitters(P.tables, P)
    S.update(3, 0, edited)
    cam = P.params[0:3].view(np.float32)
    fwd = P.params[4:7].view(np.float32)
    lo = (float(cam[0]), float(cam[1]), float(cam[2]), 8.0) if lod else None
    cu = (30.0, 80.0, 0.3, float(fwd[0]), float(fwd[1]), float(fwd[2])) if lod else None
    ms = S.weigh_emitters(P.params, P.info["light_tree_nodes"], lo, cu)
    got = S.read(3, 0, edited.nbytes, np.uint32)
    want = oracle.weigh_emitters(edited, P.words, P.params, P.info["light_tree_nodes"], lo, cu)
    assert (got == want).all(), np.flatnonzero(got != want)[:10]
    assert (got != edited).any() and ms > 0.0
    S.close()


def test_reweighed_scene_renders_as_the_oracle_does(gpu):
    from test_gpu_pass import image_parity
    P = prep.prepare(small_city())
    S = gpu.upload(P)
    edited, _ = scale_emitters(P.tables, P)
    S.update(3, 0, edited)
    S.weigh_emitters(P.params, P.info["light_tree_nodes"])
    P.tables = oracle.weigh_emitters(edited, P.words, P.params, P.info["light_tree_nodes"])
    acc_g = S.render_raw(P.params, 4)[0]
    acc_o, _ = oracle.Oracle(P).render(P.params, 4)
    frac, mean_err = image_parity(acc_g, acc_o, P.width, P.height, 4)
    assert frac >= 0.99 and mean_err <= 0.01, (frac, mean_err)
    S.close()


def tree_sections(S, P, nodes):
    """The tables' light-tree nodes, the emitter entries with their guide and header, and each emitter triangle's code,
    as the device holds them."""
    tp = P.params[124:136]
    tree, entries, lst = int(tp[0]), int(tp[4]), int(tp[11])
    n = int(P.params[21])
    t = S.read(3, 0, P.tables.nbytes, np.uint32).reshape(-1, 4)
    return t[tree:tree + nodes].copy(), t[entries:entries + n + 65536 // 4 + 2].copy(), t[lst + 2:lst + 4 * n:4, 3].copy()


def test_device_light_tree_is_the_preps(gpu):
    """ltree.rs:405-470 on the device over the scene's 280 emitter triangles: after the re-weigh, the tree's nodes
    (spheres, child words, powers), the emitter table in leaf order and every triangle's code are the host prep's,
    bit for bit, though the tree's sections were cleared first."""
    P = prep.prepare(small_city())
    nodes = P.info["light_tree_nodes"]
    assert nodes > 0
    want_s = gpu.upload(P)
    want_s.weigh_emitters(P.params, nodes)
    want = tree_sections(want_s, P, nodes)
    S = gpu.upload(P)
    tp = P.params[124:136]
    S.update(3, int(tp[0]) * 16, np.zeros((nodes, 4), np.uint32))  # no tree
    ent = P.tables.reshape(-1, 4)[int(tp[4]):int(tp[4]) + int(P.params[21])].copy()
    S.update(3, int(tp[4]) * 16, ent[::-1].copy())  # the emitters in reverse order
    params = P.params.copy()
    params[85] = 0
    got_nodes, ms = S.build_light_tree(params)
    assert got_nodes == nodes and ms > 0.0
    assert params[85] == P.params[85] and params[87] == P.params[87]  # the tree's entries; its candidates
    S.weigh_emitters(params, got_nodes)
    got = tree_sections(S, P, nodes)
    for g, w, name in zip(got, want, ("tree nodes", "emitter entries", "codes")):
        assert np.array_equal(g, w), (name, np.flatnonzero(g.ravel() != w.ravel())[:8])
    S.close()
    want_s.close()


def test_light_tree_rebuilt_after_the_emitters_moved(gpu):
    """The emitters moved (the same quads 25 m away, the scene prepared again) while the tables still hold the tree,
    order and codes of where they were: the device build makes the prep's tree of the moved scene, and the render is
    the oracle's on that scene within 3 SE."""
    from test_gpu_pass import image_parity
    P = prep.prepare(small_city())
    P2 = prep.prepare(small_city(emitter_offset=(25.0, 0.0, -15.0)))
    assert np.array_equal(P.params[124:136], P2.params[124:136]) and P.tables.shape == P2.tables.shape
    nodes = P2.info["light_tree_nodes"]
    want_s = gpu.upload(P2)
    want_s.weigh_emitters(P2.params, nodes)
    want = tree_sections(want_s, P2, nodes)
    S = gpu.upload(P2)
    tp = P.params[124:136]
    n = int(P.params[21])
    old = P.tables.reshape(-1, 4)
    S.update(3, int(tp[0]) * 16, old[int(tp[0]):int(tp[1])].copy())      # the old tree
    S.update(3, int(tp[4]) * 16, old[int(tp[4]):int(tp[4]) + n].copy())  # the old order
    stale = P2.tables.reshape(-1, 4)[int(tp[11]):int(tp[11]) + 4 * n].copy()
    stale[2::4, 3] = old[int(tp[11]) + 2:int(tp[11]) + 4 * n:4, 3]         # the old codes
    S.update(3, int(tp[11]) * 16, stale)
    params = P2.params.copy()
    got_nodes, _ = S.build_light_tree(params)
    S.weigh_emitters(params, got_nodes)
    got = tree_sections(S, P2, nodes)
    for g, w, name in zip(got, want, ("tree nodes", "emitter entries", "codes")):
        assert np.array_equal(g, w), (name, np.flatnonzero(g.ravel() != w.ravel())[:8])
    P2.tables = S.read(3, 0, P2.tables.nbytes, np.uint32).reshape(P2.tables.shape)
    acc_g = S.render_raw(params, 4)[0]
    acc_o, _ = oracle.Oracle(P2).render(params, 4)
    frac, mean_err = image_parity(acc_g, acc_o, P2.width, P2.height, 4)
    assert frac >= 0.99 and mean_err <= 0.01, (frac, mean_err)
    S.close()
    want_s.close()
