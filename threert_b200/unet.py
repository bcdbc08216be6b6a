"""The learned denoiser from Python: the network (trt_unet_*), its inputs made from a render's accum, the training
pairs rendered by the pass itself, training and inference.

The network is the library's U-Net (include/threert_cuda.h): input a pixel's log1p(radiance * s), albedo, normal,
log1p(depth * sd) and log1p(variance * s^2), where s and sd normalise by the image's mean luminance and mean first-hit
distance; it predicts
log1p(radiance * s) of the converged image. Pairs for training are noisy renders (1-4 spp, TRT_RENDER_DEPTH) against
renders of many more samples of the same view; both come from this repository's path tracer.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from .gpu import Gpu, RenderError, Scene

LUM = np.array([0.2126, 0.7152, 0.0722], np.float32)
# (cin padded to 32, cout): the layers in the library's order
LAYERS = [(32, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128), (128, 128), (224, 96), (96, 96),
          (160, 64), (64, 64), (96, 32), (32, 32), (32, 3)]
N_FEAT = 11  # input channels a pixel: log radiance (3), albedo (3), normal (3), log depth, log variance
FAN_IN = [N_FEAT, 32, 32, 64, 64, 96, 96, 128, 224, 96, 160, 64, 96, 32, 32]  # the real input channels


def r64(v):
    return (v + 63) // 64 * 64


def param_count() -> int:
    return sum(9 * cin * r64(cout) + r64(cout) for cin, cout in LAYERS)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights over each layer's real inputs and outputs, zero elsewhere; zero biases."""
    rng = np.random.default_rng(seed)
    out = np.zeros(param_count(), np.float32)
    o = 0
    for (cin, cout), fan in zip(LAYERS, FAN_IN):
        cp = r64(cout)
        W = np.zeros((9, cin, cp), np.float32)
        gain = 1.0 if cout == 3 else 2.0
        W[:, :fan, :cout] = rng.normal(0.0, math.sqrt(gain / (9 * fan)), (9, fan, cout))
        out[o:o + W.size] = W.ravel()
        o += W.size + cp
    return out


def features(accum: np.ndarray, width: int, height: int) -> tuple[np.ndarray, float]:
    """The network's input (height, width, N_FEAT) from an accum with depth (TRT_RENDER_DEPTH), and the radiance scale s;
    the same transform the device applies (trt_unet_denoise_accum)."""
    px = np.asarray(accum, np.float32).reshape(-1, N.PIXEL_FLOATS)
    px = np.where(np.isfinite(px), px, 0.0)
    cnt = np.maximum(px[:, 3:4], 1.0)
    rad, alb, nrm = px[:, 0:3] / cnt, px[:, 4:7] / cnt, px[:, 8:11] / cnt
    depth = px[:, 12] / cnt[:, 0]
    lum = rad @ LUM
    s = 1.0 / max(float(lum.mean()), 1e-6)
    hit = depth > 0
    sd = 1.0 / max(float(depth[hit].sum()) / max(int(hit.sum()), 1), 1e-6)
    mean = px[:, 7] / cnt[:, 0]
    var = np.maximum(px[:, 11] / cnt[:, 0] - mean * mean, 0.0) / cnt[:, 0]
    f = np.concatenate([np.log1p(np.maximum(rad * s, 0.0)), alb, nrm, np.log1p(np.maximum(depth * sd, 0.0))[:, None],
                        np.log1p(np.maximum(var * s * s, 0.0))[:, None]], 1)
    return f.reshape(height, width, N_FEAT).astype(np.float32), s


def target(rgb: np.ndarray, s: float) -> np.ndarray:
    return np.log1p(np.maximum(np.asarray(rgb, np.float32) * s, 0.0)).astype(np.float32)


def radiance(pred: np.ndarray, s: float) -> np.ndarray:
    return np.maximum(np.expm1(pred), 0.0) / s


class UNet:
    """trt_unet: the network, its optimiser and its buffers on one device."""

    def __init__(self, device: int = 0, max_batch: int = 8, max_h: int = 128, max_w: int = 128):
        self.handle = C.c_void_p()
        rc = N.lib().trt_unet_create(device, max_batch, max_h, max_w, C.byref(self.handle))
        if rc != 0:
            raise RenderError(f"trt_unet_create failed ({N.ERRORS.get(rc, rc)})")

    def _check(self, rc, what):
        if rc != 0:
            raise RenderError(f"{what}: {N.ERRORS.get(rc, rc)}: {N.lib().trt_unet_last_error(self.handle).decode()}")

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == param_count()
        self._check(N.lib().trt_unet_set_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float))), "set_params")

    def params(self) -> np.ndarray:
        p = np.zeros(param_count(), np.float32)
        self._check(N.lib().trt_unet_get_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float))), "get_params")
        return p

    def forward(self, feats: np.ndarray) -> tuple[np.ndarray, float]:
        f = np.ascontiguousarray(feats, np.float32)
        b, h, w, _ = f.shape
        out = np.zeros((b, h, w, 3), np.float32)
        ms = C.c_float()
        self._check(N.lib().trt_unet_forward(self.handle, f.ctypes.data_as(C.POINTER(C.c_float)), b, h, w,
                                             out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(ms)), "forward")
        return out, ms.value

    def step(self, feats: np.ndarray, targets: np.ndarray, lr: float = 1e-3, update: bool = True,
             grads: bool = False) -> tuple[float, np.ndarray | None, float]:
        f = np.ascontiguousarray(feats, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        b, h, w, _ = f.shape
        loss = C.c_float()
        ms = C.c_float()
        g = np.zeros(param_count(), np.float32) if grads else None
        self._check(N.lib().trt_unet_train_step(self.handle, f.ctypes.data_as(C.POINTER(C.c_float)),
                                                t.ctypes.data_as(C.POINTER(C.c_float)), b, h, w, lr,
                                                1 if update else 0, C.byref(loss),
                                                g.ctypes.data_as(C.POINTER(C.c_float)) if grads else None,
                                                C.byref(ms)), "train_step")
        return loss.value, g, ms.value

    def hold_next_load(self):
        """trt_unet_hold_next_load: the next forward's first convolution withholds a copy, so that its bounded
        pipeline wait runs out and the call fails (a test of the error path)."""
        self._check(N.lib().trt_unet_hold_next_load(self.handle), "hold_next_load")

    def denoise(self, scene: Scene) -> tuple[np.ndarray, float]:
        """The scene's last accum (rendered with TRT_RENDER_DEPTH) denoised on the device: (h, w, 3), device ms."""
        ptr, nbytes = C.c_void_p(), C.c_uint64()
        scene.gpu._check(N.lib().trt_accum_device_ptr(scene.handle, C.byref(ptr), C.byref(nbytes)), "accum")
        w, h = scene.last_size
        out = np.zeros((h, w, 3), np.float32)
        ms = C.c_float()
        self._check(N.lib().trt_unet_denoise_accum(self.handle, ptr, w, h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                   C.byref(ms)), "denoise")
        return out, ms.value

    def close(self):
        if self.handle:
            N.lib().trt_unet_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
