"""The learned denoiser trained end to end on the device on pairs the pass renders, then judged on a held-out city by
the reference's metric (ΔE against many more samples): what it gains over the same samples without it."""
import numpy as np
import pytest

from threert_b200 import unet
from threert_b200 import denoise_train as DT

pytestmark = pytest.mark.gpu


def test_a_trained_network_lowers_the_error_of_a_few_samples(gpu):
    F, T = DT.make_dataset(gpu, range(100, 124), 6, 128, 128, 256)
    net = unet.UNet(0, max_batch=16, max_h=256, max_w=256)
    try:
        net.set_params(unet.init_params(0))
        losses = DT.train(net, F, T, 3000, batch=16, lr=1e-3)
        assert np.mean(losses[-200:]) < 0.7 * np.mean(losses[:200])
        r = DT.judge(gpu, net, [900, 901], 256, 144, 4, 64, 2048)
    finally:
        net.close()
    # against the same 4 samples accumulated without it, and against 16 times the samples without it
    assert r["net"]["delta_e"] < 0.5 * r["plain_low"]["delta_e"], r
    assert r["net"]["delta_e"] < 2.0 * r["plain_high"]["delta_e"], r
