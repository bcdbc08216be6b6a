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
