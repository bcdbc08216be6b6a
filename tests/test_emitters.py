"""The emitters' re-weigh (emitter_weights.wgsl) restated by the oracle, held to the prep's own tables.

The prep builds the emitter table as lib.rs:451-485 emitter_cdf does (one running sum) and the tree's powers as
ltree.rs builds them; the re-weigh makes them again from the records with the reference kernel's blocked scan. The
two agree to float rounding; after an edit of the emitters' materials the re-weigh agrees with a prep of the edited
scene."""
import numpy as np

import oracle
from threert_b200 import prep, scenes

from util import small_city

GUIDE4 = 65536 // 4


def emitter_view(P, tables=None):
    t = (P.tables if tables is None else tables).view(np.float32).reshape(-1, 4)
    n = int(P.params[21])
    e0 = int(P.params[124 + 4])
    entries = t[e0:e0 + n]
    guide = t[e0 + n:e0 + n + GUIDE4 + 1].view(np.uint32).ravel()[:65537]
    header = t[e0 + n + GUIDE4 + 1]
    tree = t[int(P.params[124]):int(P.params[124]) + P.info["light_tree_nodes"]]
    return entries, guide, header, tree


def check_close(P, got_tables, want_tables=None):
    e_g, g_g, h_g, t_g = emitter_view(P, got_tables)
    e_w, g_w, h_w, t_w = emitter_view(P, want_tables)
    assert (e_g[:, 0].view(np.uint32) == e_w[:, 0].view(np.uint32)).all()
    assert np.allclose(e_g[:, 2], e_w[:, 2], rtol=2e-6, atol=0), np.abs(e_g[:, 2] / e_w[:, 2] - 1).max()
    assert np.allclose(e_g[:, 3], e_w[:, 3], rtol=2e-6, atol=0)
    assert np.allclose(e_g[:, 1], e_w[:, 1], rtol=0, atol=2e-6)
    assert (g_g != g_w).sum() <= 8, (g_g != g_w).sum()
    assert abs(h_g[0] / h_w[0] - 1) < 2e-6 and abs(h_g[1] - h_w[1]) < 2e-6, (h_g, h_w)
    if len(t_w):
        assert np.allclose(t_g[:, 2], t_w[:, 2], rtol=1e-5, atol=0)
        assert (t_g[:, [0, 1, 3]].view(np.uint32) == t_w[:, [0, 1, 3]].view(np.uint32)).all()


def test_reweigh_matches_the_prep():
    for d in (small_city(), scenes.cornell()):
        P = prep.prepare(d)
        got = oracle.weigh_emitters(P.tables, P.words, P.params, P.info["light_tree_nodes"])
        check_close(P, got)


def scale_emitters(tables, P, every=3, factor=10.0, off=1):
    """The tables with every `every`-th emitter's material emission times `factor` and emitter `off`'s off."""
    t = tables.copy()
    f = t.view(np.float32).reshape(-1, 4)
    m0 = int(P.params[124 + 1])
    n_mat = (int(P.params[124 + 2]) - m0) // 18
    emissive = [m for m in range(n_mat) if f[m0 + m * 18 + 1, :3].max() > 0]
    for k, m in enumerate(emissive):
        if k == off:
            f[m0 + m * 18 + 1, :3] = 0.0
        elif k % every == 0:
            f[m0 + m * 18 + 1, :3] *= factor
    return t, emissive


def test_reweigh_after_an_edit_matches_a_new_prep():
    d = small_city()
    P = prep.prepare(d)
    edited, emissive = scale_emitters(P.tables, P)
    assert len(emissive) == 140
    got = oracle.weigh_emitters(edited, P.words, P.params, P.info["light_tree_nodes"])
    # The same edit in the scene description, prepared again (emission off: weight 0 but the tree keeps its shape).
    first = len(d.materials) - 140
    for k in range(140):
        m = d.materials[first + k]
        if k == 1:
            m.emissive = (0.0, 0.0, 0.0)
        elif k % 3 == 0:
            m.emissive = tuple(np.float32(v) * np.float32(10.0) for v in m.emissive)
    Q = prep.prepare(d)
    e_g, _, h_g, _ = emitter_view(P, got)
    e_w, _, h_w, _ = emitter_view(Q)
    # (The new prep leaves the switched-off emitter out of its list and numbers the rest anew: compare the weights
    # that are on, sorted, and the totals.)
    wg = np.sort(e_g[:, 2][e_g[:, 2] > 0])
    ww = np.sort(e_w[:, 2][e_w[:, 2] > 0])
    assert len(wg) == len(ww) == 2 * 139
    assert np.allclose(wg, ww, rtol=2e-6, atol=0), np.abs(wg / ww - 1).max()
    assert abs(h_g[0] / h_w[0] - 1) < 2e-6
