"""The denoiser fallback's restatement (oracle: renderer/src/denoise.rs) and the image metric (compare.rs ΔE)."""
import numpy as np

import oracle
from threert_b200 import metrics


def pixels(color, albedo, normal, spp=4, var=0.0):
    """Accum records of `spp` identical samples a pixel (h, w, 3 arrays), with luminance variance `var`."""
    h, w, _ = color.shape
    acc = np.zeros((h * w, 20), np.float32)
    lum = color.reshape(-1, 3) @ np.array([0.2126, 0.7152, 0.0722], np.float32)
    acc[:, 0:3] = color.reshape(-1, 3) * spp
    acc[:, 3] = spp
    acc[:, 4:7] = albedo.reshape(-1, 3) * spp
    acc[:, 7] = lum * spp
    acc[:, 8:11] = normal.reshape(-1, 3) * spp
    acc[:, 11] = (lum * lum + var * spp) * spp
    return acc


def test_a_flat_image_stays_flat():
    h, w = 24, 32
    c = np.full((h, w, 3), 0.4, np.float32)
    a = np.full((h, w, 3), 0.5, np.float32)
    n = np.zeros((h, w, 3), np.float32)
    n[..., 1] = 1.0
    out = oracle.denoise(pixels(c, a, n, var=0.01), w, h, 4)
    assert np.allclose(out, c, rtol=1e-5)


def test_noise_goes_down_and_edges_stay():
    rng = np.random.default_rng(0)
    h, w = 48, 48
    a = np.full((h, w, 3), 0.6, np.float32)
    a[:, w // 2:] = 0.1  # an albedo edge
    n = np.zeros((h, w, 3), np.float32)
    n[..., 2] = 1.0
    clean = a * 2.0
    noisy = (clean * rng.uniform(0.5, 1.5, (h, w, 1))).astype(np.float32)
    out = oracle.denoise(pixels(noisy, a, n, var=0.05), w, h, 4)
    err_in = np.abs(noisy - clean).mean()
    err_out = np.abs(out - clean).mean()
    assert err_out < 0.5 * err_in
    # no light crosses the albedo edge
    assert np.abs(out[:, w // 2 + 1:] - clean[:, w // 2 + 1:]).mean() < 0.5 * np.abs(noisy - clean)[:, w // 2 + 1:].mean()


def test_delta_e_of_equal_images_is_zero_and_grows_with_error():
    rng = np.random.default_rng(1)
    img = rng.uniform(0, 1, (16, 16, 3)).astype(np.float32)
    assert metrics.delta_e(img, img)["mean"] == 0.0
    d1 = metrics.delta_e(img, img * 1.05)["mean"]
    d2 = metrics.delta_e(img, img * 1.3)["mean"]
    assert 0 < d1 < d2


def test_lab_of_white_and_black():
    L = metrics.lab(np.array([[1.0, 1.0, 1.0], [0.0, 0.0, 0.0]]))
    assert abs(L[0, 0] - 100.0) < 0.1 and abs(L[0, 1]) < 0.1 and abs(L[0, 2]) < 0.1
    assert abs(L[1, 0]) < 1e-9
