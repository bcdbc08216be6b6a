"""Training and judging the learned denoiser on pairs this path tracer renders.

A pair is one view of a seeded procedural city (the city generator of config 1 at a smaller size, so that hundreds of
seeds prepare in seconds): a noisy render of 1-4 spp with its depth (TRT_RENDER_DEPTH) and a render of many more
samples drawn with another sampler seed (so that the two share no sample). The network is trained on the noisy
render's features against log1p(reference * s) and judged by the reference's metric (ΔE, renderer/src/compare.rs)
against a render of many samples of held-out seeds, beside the a-trous fallback.
"""
from __future__ import annotations

import time

import numpy as np

from . import metrics, prep, scenes
from . import _native as N
from .gpu import Gpu, frame_of
from .unet import UNet, features, radiance, target


def small_city(seed: int, width: int, height: int, n_objects: int = 300, extent: float = 100.0):
    return scenes.city(n_objects=n_objects, width=width, height=height, seed=seed, extent=extent, n_emitters=60,
                       box_segments=2, sphere_slices=12, sphere_stacks=10, max_depth=4, sky_size=(256, 128))


def views(P, seed: int, n: int, extent: float = 100.0) -> list[np.ndarray]:
    """n camera views along the scene's spline (random frames of 240)."""
    rng = np.random.default_rng(seed)
    out = []
    for f in rng.integers(0, 240, n):
        cam = scenes.city_camera(int(f), 240, seed, P.width, P.height, extent)
        out.append(prep.set_camera(P.params, cam))
    return out


def render_pair(S, params, spp_in: int, spp_ref: int, seed: int):
    """(features (h, w, 10), target (h, w, 3), reference radiance (h, w, 3), the noisy accum, s)."""
    w, h = int(params[16]), int(params[17])
    acc, _ = S.render_raw(prep.params_with(params, seed=seed), spp_in, flags=N.TRT_RENDER_DEPTH)
    f, s = features(acc, w, h)
    ref_acc, _ = S.render_raw(prep.params_with(params, seed=seed ^ 0x51ED270B), spp_ref)
    ref = frame_of(ref_acc, w, h, spp_ref).color
    return f, target(ref, s), ref, acc, s


def make_dataset(gpu: Gpu, seeds, views_per_scene: int, width: int, height: int, spp_ref: int,
                 spp_choices=(1, 2, 4), log=None):
    """Features and targets of every view of every seed's city: (N, h, w, 10), (N, h, w, 3)."""
    F, T = [], []
    rng = np.random.default_rng(12345)
    t0 = time.perf_counter()
    for sd in seeds:
        P = prep.prepare(small_city(int(sd), width, height))
        S = gpu.upload(P)
        for k, params in enumerate(views(P, int(sd), views_per_scene)):
            f, t, _, _, _ = render_pair(S, params, int(rng.choice(spp_choices)), spp_ref, int(sd) * 1000 + k)
            F.append(f)
            T.append(t)
        S.close()
    if log:
        log(f"dataset: {len(F)} pairs of {width}x{height} in {time.perf_counter() - t0:.1f} s")
    return np.stack(F), np.stack(T)


def train(net: UNet, F: np.ndarray, T: np.ndarray, steps: int, batch: int = 8, lr: float = 1e-3, crop: int = 64,
          seed: int = 0, log=None, log_every: int = 200) -> list[float]:
    """Adam on random crops of the pairs; the learning rate falls by 10 over the last third."""
    rng = np.random.default_rng(seed)
    n, h, w, _ = F.shape
    losses = []
    t0 = time.perf_counter()
    for it in range(steps):
        idx = rng.integers(0, n, batch)
        ys = rng.integers(0, h - crop + 1, batch) // 8 * 8
        xs = rng.integers(0, w - crop + 1, batch) // 8 * 8
        fb = np.stack([F[i, y:y + crop, x:x + crop] for i, y, x in zip(idx, ys, xs)])
        tb = np.stack([T[i, y:y + crop, x:x + crop] for i, y, x in zip(idx, ys, xs)])
        rate = lr if it < 2 * steps // 3 else lr * 0.1
        loss, _, _ = net.step(np.ascontiguousarray(fb), np.ascontiguousarray(tb), lr=rate)
        losses.append(loss)
        if log and (it + 1) % log_every == 0:
            log(f"step {it + 1}: loss {np.mean(losses[-log_every:]):.4f} ({time.perf_counter() - t0:.1f} s)")
    return losses


def judge(gpu: Gpu, net: UNet, seeds, width: int, height: int, spp_net: int, spp_plain: int, spp_truth: int,
          views_per_scene: int = 1) -> dict:
    """ΔE against `spp_truth` samples of held-out seeds: the network at spp_net, the a-trous fallback at spp_net and at
    spp_plain, the plain render at spp_plain; and each one's device time (render + filter)."""
    rows = []
    for sd in seeds:
        P = prep.prepare(small_city(int(sd), width, height))
        S = gpu.upload(P)
        for k, params in enumerate(views(P, int(sd) + 7, views_per_scene)):
            truth_acc, _ = S.render_raw(prep.params_with(params, seed=0xACE), spp_truth)
            truth = frame_of(truth_acc, width, height, spp_truth).color
            r = {}
            acc, st = S.render_timed(prep.params_with(params, seed=k + 1), spp_net, flags=N.TRT_RENDER_DEPTH)
            den, ms_net = net.denoise(S)
            r["net"] = (metrics.delta_e(truth, den)["mean"], st.device_ms + ms_net)
            at, ms_at = S.denoise_atrous(4)
            r["atrous_low"] = (metrics.delta_e(truth, at)["mean"], st.device_ms + ms_at)
            r["plain_low"] = (metrics.delta_e(truth, frame_of(acc, width, height, spp_net).color)["mean"], st.device_ms)
            acc, st = S.render_timed(prep.params_with(params, seed=k + 1), spp_plain)
            r["plain_high"] = (metrics.delta_e(truth, frame_of(acc, width, height, spp_plain).color)["mean"], st.device_ms)
            at, ms_at = S.denoise_atrous(4)
            r["atrous_high"] = (metrics.delta_e(truth, at)["mean"], st.device_ms + ms_at)
            rows.append(r)
        S.close()
    return {k: {"delta_e": float(np.mean([r[k][0] for r in rows])), "ms": float(np.mean([r[k][1] for r in rows]))}
            for k in rows[0]}
