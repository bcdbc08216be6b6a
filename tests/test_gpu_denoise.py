"""The denoiser fallback on the device (trt_denoise_atrous) against the oracle's denoise.rs restatement, and what it
does to the error against a converged render; the depth guide (TRT_RENDER_DEPTH)."""
import numpy as np
import pytest

import oracle
from threert_b200 import metrics, prep
from threert_b200 import _native as N
from threert_b200.gpu import frame_of

from util import small_city

pytestmark = pytest.mark.gpu


def test_atrous_matches_the_oracle_and_lowers_the_error(gpu):
    P = prep.prepare(small_city(width=96, height=64))
    S = gpu.upload(P)
    w, h = P.width, P.height
    acc, _ = S.render_raw(P.params, 4)
    got, ms = S.denoise_atrous(4)
    want = oracle.denoise(acc, w, h, 4)
    assert ms > 0
    # expf against libm's exp: a few ulps a weight
    assert np.allclose(got, want, rtol=2e-4, atol=1e-4 * float(np.abs(want).mean()))
    ref = frame_of(S.render_raw(P.params, 256)[0], w, h, 256).color
    noisy = frame_of(acc, w, h, 4).color
    assert metrics.delta_e(ref, got)["mean"] < metrics.delta_e(ref, noisy)["mean"]
    S.close()


def test_depth_guide_is_the_first_hit_distance(gpu):
    P = prep.prepare(small_city(width=48, height=32))
    S = gpu.upload(P)
    plain, _ = S.render_raw(P.params, 2)
    with_depth, _ = S.render_raw(P.params, 2, flags=N.TRT_RENDER_DEPTH)
    others = [k for k in range(20) if k != 12]  # x of the fourth vec4 holds the depth sum
    assert np.array_equal(plain[:, others], with_depth[:, others])  # nothing else changes
    assert np.all(plain[:, 12] == 0.0)
    depth = with_depth[:, 12] / with_depth[:, 3]
    # against the camera rays' hits: the mean over samples of t, 0 on escape; the walk's own t on sample 0's rays
    assert (depth > 0).mean() > 0.5 and np.isfinite(depth).all()
    S.close()
