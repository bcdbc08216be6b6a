"""Config 2's host side and the deformation's CPU restatements: the humanoid, its poses, the instance records, the
oracle's skin / gather / refit (renderer/shaders/skin.wgsl, leaf_gather.wgsl, units.rs refit) and the top tree the
device rebuilds (units.rs top_tree over UnitBox::new)."""
import numpy as np

import oracle
from threert_b200 import crowd, prep

from util import small_crowd


def prepared():
    c = small_crowd()
    return c, prep.prepare(c.desc)


def numpy_skin(corners, palette):
    """The skin in float64: the oracle's f32 result must be within rounding of it."""
    b = corners[:, 3].view(np.uint32), corners[:, 7].view(np.uint32)
    idx = np.stack([b[0] & 0xffff, b[0] >> 16, b[1] & 0xffff, b[1] >> 16], 1)
    w = corners[:, 12:16].astype(np.float64)
    M = (palette.astype(np.float64)[idx] * w[:, :, None, None]).sum(1)
    return np.einsum("vij,vj->vi", M[..., :3], corners[:, :3].astype(np.float64)) + M[..., 3]


def test_humanoid_sizes():
    h = crowd.humanoid()
    assert len(h.mesh.positions) == 20160 and len(h.positions) == 10140
    assert np.allclose(h.weights.sum(1), 1.0) and h.bones.max() < crowd.N_BONES


def test_records_at_rest_are_the_preps():
    c, P = prepared()
    _, rec = crowd.records(P)
    assert np.array_equal(crowd.frame_records(P, c, 0.0), rec[:c.n])
    assert not np.array_equal(crowd.frame_records(P, c, 2.0), rec[:c.n])


def test_the_oracles_skin_follows_the_palette():
    c, P = prepared()
    corners, jobs = crowd.deform_jobs(P, c)
    pal = crowd.palettes(0.7, c.phase, c.scale)
    w_ind = int(P.params[136 + 4])
    v, _, _ = oracle.deform(jobs, corners, pal.reshape(-1, 12), P.vertices, P.leaves, P.nodes, P.words, w_ind)
    rows = v.reshape(-1, 3, 4)
    for g, j in enumerate(jobs):
        got = rows[j[0]:j[0] + j[1], 0, :3]
        want = numpy_skin(corners, pal[g])
        assert np.abs(got - want).max() < 1e-5
        # normals stay unit length
        assert np.allclose(np.linalg.norm(rows[j[0]:j[0] + j[1], 1, :3], axis=1), 1.0, atol=1e-5)


def test_refit_at_rest_is_the_built_tree():
    """Identity palettes leave the rest pose: the refit boxes are then the boxes the prep built."""
    c, P = prepared()
    corners, jobs = crowd.deform_jobs(P, c)
    corners = corners.copy()
    corners[:, 12:16] = [1.0, 0.0, 0.0, 0.0]  # one bone each, weight exactly 1
    ident = np.zeros((crowd.N_BONES * c.groups, 3, 4), np.float32)
    ident[:, :, :3] = np.eye(3)
    w_ind = int(P.params[136 + 4])
    v, lv, nd = oracle.deform(jobs, corners, ident.reshape(-1, 12), P.vertices, P.leaves, P.nodes, P.words, w_ind)
    rows, rest = v.reshape(-1, 3, 4), P.vertices.reshape(-1, 3, 4)
    assert np.array_equal(rows[:, 0], rest[:, 0])  # positions exactly; normals are normalised again
    assert np.abs(rows[:, 1, :3] - rest[:, 1, :3]).max() < 1e-6
    for j in jobs:
        r, n = j[6], j[7]
        assert np.array_equal(nd[r:r + n].view(np.float32), P.nodes[r:r + n].view(np.float32))
    # leaves: v0 and edges from the shared vertices, as the prep made them
    for j in jobs:
        t0, nt = j[4], j[5]
        a, b = lv.reshape(-1, 3, 4)[t0:t0 + nt], P.leaves.reshape(-1, 3, 4)[t0:t0 + nt]
        assert np.array_equal(a[:, :, :3], b[:, :, :3])


def test_units_top_is_the_prepared_top_tree():
    c, P = prepared()
    _, rec = crowd.records(P)
    units = len(rec)
    worlds = rec[:, 0:12].view(np.float32).reshape(units, 3, 4)
    nodes = P.nodes.view(np.float32)
    roots = rec[:, 15]
    boxes = np.concatenate([nodes[roots, 0:3], nodes[roots, 4:7]], 1)
    top, depth = prep.units_top(worlds, boxes)
    first = int(P.params[68 + 2])
    assert depth <= 18
    assert np.array_equal(top, P.nodes[first:first + 2 * units - 1])
