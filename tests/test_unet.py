"""The learned denoiser's CPU oracle (oracle/unet_ref.py) pinned by finite differences, and the host-side transforms."""
import numpy as np

from oracle import unet_ref as R
from threert_b200 import unet


def test_parameter_layout_matches():
    assert unet.param_count() == sum(9 * cin * R.r64(cout) + R.r64(cout) for cin, cout, _ in R.LAYERS)
    p = unet.init_params(0)
    q = R.pack(R.unpack(p), p)
    # padding is zero in the initial parameters: packing what unpack reads gives them back
    assert np.array_equal(q.astype(np.float32), p)


def test_oracle_gradients_are_the_loss_slopes():
    rng = np.random.default_rng(0)
    p = unet.init_params(1).astype(np.float64)
    # nonzero biases so that the ReLUs are not all at a kink
    o = 0
    for cin, cout, _ in R.LAYERS:
        o += 9 * cin * R.r64(cout)
        p[o:o + cout] = rng.normal(0, 0.05, cout)
        o += R.r64(cout)
    feats = rng.normal(0, 1, (1, 8, 8, unet.N_FEAT))
    tgt = rng.normal(0, 1, (1, 8, 8, 3))
    loss, G, _ = R.loss_and_grads(R.unpack(p), feats, tgt)
    flat = R.pack(G, p)
    idx = rng.choice(np.flatnonzero(flat), 24, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy(); q[i] += eps
        lp, _, _ = R.loss_and_grads(R.unpack(q), feats, tgt)
        q[i] -= 2 * eps
        lm, _, _ = R.loss_and_grads(R.unpack(q), feats, tgt)
        num = (lp - lm) / (2 * eps)
        assert abs(num - flat[i]) <= 1e-4 * max(abs(num), abs(flat[i])) + 1e-9, (i, num, flat[i])


def test_features_and_their_inverse():
    h, w = 8, 16
    acc = np.zeros((h * w, 20), np.float32)
    acc[:, 3] = 4
    acc[:, 0:3] = 4 * np.linspace(0.1, 5.0, h * w)[:, None]
    acc[:, 4:7] = 2.0
    acc[:, 12] = 4 * 3.0
    f, s = unet.features(acc, w, h)
    assert f.shape == (h, w, unet.N_FEAT)
    rad = acc[:, 0:3] / 4
    back = unet.radiance(f[..., 0:3], s).reshape(-1, 3)
    assert np.allclose(back, rad, rtol=1e-5)
    assert np.allclose(f[..., 9], np.log1p(1.0))  # depth over its mean
