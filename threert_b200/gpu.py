"""The pass from Python, shaped as the reference's host interface.

`Gpu.render` mirrors renderer/src/gpu.rs:4116 `Gpu::render(scene, ..., base: Params, spp, timings) -> Result<Frame>`:
it uploads the prepared buffers, runs `spp` samples (Params `size.z` is the sample index), reads `accum` back and
converts each 80-byte `Pixel` to a `Frame` (gpu.rs:4211-4232). Errors raise `RenderError` (the reference's
anyhow::Err), among them a traversal that hit its loop guard (gpu.rs:4199-4205).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .prep import Prepared, apply_sky


class RenderError(RuntimeError):
    pass


@dataclass
class Frame:
    """gpu.rs:2059-2076 Frame (without the live-only emission / specular split and the translucent overlay)."""
    width: int
    height: int
    color: np.ndarray      # (h, w, 3)
    albedo: np.ndarray
    normal: np.ndarray
    variance: np.ndarray   # (h, w): variance of the per-pixel mean luminance
    samples: int


def frame_of(accum: np.ndarray, width: int, height: int, spp: int) -> Frame:
    """gpu.rs:4219-4232: each Pixel over its sample count (at least 1), non-finite values as 0."""
    px = np.asarray(accum, np.float32).reshape(-1, N.PIXEL_FLOATS)
    c = np.maximum(px[:, 3:4], 1.0)
    p = np.where(np.isfinite(px), px, 0.0)
    mean = p[:, 7] / c[:, 0]
    var = np.maximum(p[:, 11] / c[:, 0] - mean * mean, 0.0) / c[:, 0]
    shape3 = (height, width, 3)
    return Frame(width, height, (p[:, 0:3] / c).reshape(shape3), (p[:, 4:7] / c).reshape(shape3),
                 (p[:, 8:11] / c).reshape(shape3), var.reshape(height, width), spp)


RAY_DTYPE = np.dtype([("o", np.float32, 3), ("tmax", np.float32), ("d", np.float32, 3), ("mode", np.uint32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("tri", np.uint32), ("u", np.float32), ("v", np.float32),
                      ("inst", np.uint32), ("part", np.uint32)])


class Scene:
    """A scene resident on the device (trt_scene)."""

    def __init__(self, gpu: "Gpu", prepared: Prepared):
        self.gpu = gpu
        self.prepared = prepared
        self.handle = C.c_void_p()
        L = N.lib()
        arrs = [prepared.vertices, prepared.leaves, prepared.nodes, prepared.tables, prepared.words, prepared.env_half]
        arrs = [np.ascontiguousarray(a) for a in arrs]
        d = N.SceneDesc(arrs[0].ctypes.data, arrs[0].nbytes, arrs[1].ctypes.data, arrs[1].nbytes,
                        arrs[2].ctypes.data, arrs[2].nbytes, arrs[3].ctypes.data, arrs[3].nbytes,
                        arrs[4].ctypes.data, arrs[4].nbytes, arrs[5].ctypes.data, prepared.env_w, prepared.env_h)
        gpu._check(L.trt_scene_upload(gpu.ctx, C.byref(d), C.byref(self.handle)), "trt_scene_upload")

    def close(self):
        # (A closed Gpu has freed its scenes with its context.)
        if self.handle and self.gpu.ctx:
            N.lib().trt_scene_free(self.handle)
        self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render_raw(self, params: np.ndarray, spp: int, first_sample: int = 0, flags: int = 0, read: bool = True,
                   stats: bool = True, out: np.ndarray | None = None):
        """Runs the pass; returns (accum as (w*h, 20) float32 or None, Stats or None). `out`: the array to read into."""
        L = N.lib()
        p = np.ascontiguousarray(params, dtype=np.uint32)
        w, h = int(p[16]), int(p[17])
        if out is not None and (out.dtype != np.float32 or out.shape != (w * h, N.PIXEL_FLOATS) or not out.flags.c_contiguous):
            raise ValueError("render_raw: `out` must be a C-contiguous (w*h, 20) float32 array")
        acc = (out if out is not None else np.empty((w * h, N.PIXEL_FLOATS), np.float32)) if read else None
        st = N.Stats() if stats else None
        self.last_size = (w, h)
        rc = L.trt_render(self.handle, p.ctypes.data_as(C.POINTER(C.c_uint32)), first_sample, spp, flags,
                          acc.ctypes.data_as(C.POINTER(C.c_float)) if read else None, C.byref(st) if stats else None)
        self.gpu._check(rc, "trt_render")
        return acc, st

    def read_accum(self, out: np.ndarray | None = None) -> np.ndarray:
        """The accum of the last render (trt_accum_read), as (w*h, 20) float32."""
        w, h = self.last_size
        acc = out if out is not None else np.empty((w * h, N.PIXEL_FLOATS), np.float32)
        self.gpu._check(N.lib().trt_accum_read(self.handle, acc.ctypes.data_as(C.POINTER(C.c_float)), acc.nbytes),
                        "trt_accum_read")
        return acc

    def render_timed(self, params: np.ndarray, spp: int, flags: int = 0):
        """render_raw whose Stats' device_ms is the render's alone (the accum read back after the timed call)."""
        _, st = self.render_raw(params, spp, flags=flags, read=False)
        return self.read_accum(), st

    def accum_copy(self, dst_device_ptr: int, nbytes: int):
        """trt_accum_copy: the accum into caller-owned device memory (e.g. a torch tensor's data_ptr()), waited for."""
        self.gpu._check(N.lib().trt_accum_copy(self.handle, C.c_void_p(dst_device_ptr), nbytes), "trt_accum_copy")

    def trace(self, params: np.ndarray, rays: np.ndarray, flags: int = 0) -> np.ndarray:
        L = N.lib()
        rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.zeros(len(rays), HIT_DTYPE)
        p = np.ascontiguousarray(params, dtype=np.uint32)
        rc = L.trt_trace(self.handle, p.ctypes.data_as(C.POINTER(C.c_uint32)),
                         rays.ctypes.data_as(C.POINTER(N.Ray)), len(rays), flags,
                         hits.ctypes.data_as(C.POINTER(N.Hit)))
        self.gpu._check(rc, "trt_trace")
        return hits

    def set_sky(self, atmosphere: N.Atmosphere, sun_light: int, env_nee_floor: float, params: np.ndarray) -> N.SkyResult:
        """Re-bakes the scene's atmosphere in place on the device (trt_scene_set_sky): texels, CDF, the sun light's
        colour, and `params` (uint32 (156,), updated in place). Returns the bake's results."""
        if params.dtype != np.uint32 or not params.flags.c_contiguous:
            raise ValueError("set_sky: params must be a C-contiguous uint32 array")
        r = N.SkyResult()
        self.gpu._check(N.lib().trt_scene_set_sky(self.handle, C.byref(atmosphere), sun_light, env_nee_floor,
                                                  params.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(r)),
                        "trt_scene_set_sky")
        return r

    def weigh_emitters(self, params: np.ndarray, tree_nodes: int, lod=None, cull=None) -> float:
        """Re-weighs the emitters on the device from the tables as they are now (trt_scene_weigh_emitters); lod: None
        or (x, y, z, d0); cull: None or (radius, far, cos, dx, dy, dz). Returns the device ms."""
        p = np.ascontiguousarray(params, np.uint32)
        lo = np.ascontiguousarray(lod, np.float32) if lod is not None else None
        cu = np.ascontiguousarray(cull, np.float32) if cull is not None else None
        ms = C.c_float()
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
        self.gpu._check(N.lib().trt_scene_weigh_emitters(self.handle, p.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                         tree_nodes, fp(lo), fp(cu), C.byref(ms)),
                        "trt_scene_weigh_emitters")
        return float(ms.value)

    def build_light_tree(self, params: np.ndarray) -> tuple[int, float]:
        """The light tree built again on the device from the emitter records as they are now
        (trt_scene_build_light_tree); `params` (uint32 (156,), C-contiguous) gets its tree words. Returns (the tree's
        nodes, device ms); then weigh_emitters(params, nodes) makes the powers, the CDF and the header."""
        if params.dtype != np.uint32 or not params.flags.c_contiguous:
            raise ValueError("build_light_tree: params must be a C-contiguous uint32 array")
        nodes, ms = C.c_uint32(), C.c_float()
        self.gpu._check(N.lib().trt_scene_build_light_tree(self.handle, params.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                           C.byref(nodes), C.byref(ms)), "trt_scene_build_light_tree")
        return int(nodes.value), float(ms.value)

    def read(self, which: int, offset: int, nbytes: int, dtype=np.uint8) -> np.ndarray:
        """Bytes [offset, offset + nbytes) of buffer `which` (0 vertices, 1 leaves, 2 nodes, 3 tables, 4 words, 5 the
        environment's RGBA16F texels)."""
        out = np.empty(nbytes, np.uint8)
        self.gpu._check(N.lib().trt_scene_read(self.handle, which, offset, out.ctypes.data, nbytes), "trt_scene_read")
        return out.view(dtype)

    def update(self, which: int, offset: int, data: np.ndarray):
        a = np.ascontiguousarray(data)
        self.gpu._check(N.lib().trt_scene_update(self.handle, which, offset, a.ctypes.data, a.nbytes),
                        "trt_scene_update")

    def deform_setup(self, corners: np.ndarray, meshes: np.ndarray):
        """corners: (n, 16) float32 skin corners (trt_corner); meshes: (m, 8) uint32 trt_deform_mesh rows."""
        c = np.ascontiguousarray(corners, np.float32).reshape(-1, 16)
        m = np.ascontiguousarray(meshes, np.uint32).reshape(-1, 8)
        d = N.DeformDesc(c.ctypes.data, len(c), m.ctypes.data_as(C.POINTER(N.DeformMesh)), len(m))
        self.gpu._check(N.lib().trt_deform_setup(self.handle, C.byref(d)), "trt_deform_setup")

    def deform(self, params: np.ndarray, palette: np.ndarray, stats: bool = True) -> dict | None:
        """One frame's deformation; palette: (n, 3, 4) float32 matrices. With stats, waits and returns the times."""
        p = np.ascontiguousarray(params, dtype=np.uint32)
        pal = np.ascontiguousarray(palette, np.float32).reshape(-1, 12)
        st = N.DeformStats() if stats else None
        rc = N.lib().trt_deform(self.handle, p.ctypes.data_as(C.POINTER(C.c_uint32)),
                                pal.ctypes.data_as(C.POINTER(C.c_float)), len(pal), 0, C.byref(st) if stats else None)
        self.gpu._check(rc, "trt_deform")
        return {f[0]: getattr(st, f[0]) for f in N.DeformStats._fields_} if stats else None

    def denoise_atrous(self, iterations: int = 4) -> tuple[np.ndarray, float]:
        """The fallback denoiser (denoise.rs) on the last render's accum: (h, w, 3) RGB and its device ms."""
        w, h = self.last_size
        out = np.empty((h, w, 3), np.float32)
        ms = C.c_float()
        self.gpu._check(N.lib().trt_denoise_atrous(self.handle, iterations, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                   C.byref(ms)), "trt_denoise_atrous")
        return out, ms.value

    def totals(self) -> dict:
        t = N.Totals()
        self.gpu._check(N.lib().trt_scene_totals(self.handle, C.byref(t)), "trt_scene_totals")
        return {f[0]: getattr(t, f[0]) for f in N.Totals._fields_}

    def reset_totals(self):
        N.lib().trt_scene_reset_totals(self.handle)

    def set_profiling(self, on: bool):
        N.lib().trt_scene_set_profiling(self.handle, 1 if on else 0)


class Gpu:
    """One device context (trt_ctx): a CUDA stream and the scenes uploaded through it."""

    def __init__(self, device: int = 0):
        L = N.lib()
        self.ctx = C.c_void_p()
        rc = L.trt_create(C.byref(N.Options(device, 0)), C.byref(self.ctx))
        if rc != 0:
            raise RenderError(f"trt_create failed ({N.ERRORS.get(rc, rc)}): no sm_100 device {device}?")

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = N.lib().trt_last_error(self.ctx).decode()
            raise RenderError(f"{what}: {N.ERRORS.get(rc, rc)}: {msg}")

    def device_info(self) -> tuple[str, int]:
        name = C.create_string_buffer(256)
        sms = C.c_int()
        self._check(N.lib().trt_device_info(self.ctx, name, 256, C.byref(sms)), "trt_device_info")
        return name.value.decode(), sms.value

    def upload(self, prepared: Prepared) -> Scene:
        """Uploads a prepared scene; an atmosphere sky still to bake is baked on this device first and written into
        `prepared` (prep.apply_sky), so that its buffers are then the scene's."""
        if prepared.sky_pending is not None:
            atm, sun_light = prepared.sky_pending
            tex, res = self.bake_sky(atm)
            apply_sky(prepared, tex, res, sun_light)
        return Scene(self, prepared)

    def bake_sky(self, atmosphere: N.Atmosphere, tables: bool = False):
        """trt_sky_bake: (texels (height, width, 4) float32, SkyResult[, the tables as TRT_SKY_TABLE_FLOATS floats])."""
        tex = np.zeros((atmosphere.height, atmosphere.width, 4), np.float32)
        tab = np.zeros(N.SKY_TABLE_FLOATS, np.float32) if tables else None
        r = N.SkyResult()
        self._check(N.lib().trt_sky_bake(self.ctx, C.byref(atmosphere), tex.ctypes.data_as(C.POINTER(C.c_float)),
                                         tab.ctypes.data_as(C.POINTER(C.c_float)) if tables else None, C.byref(r)),
                    "trt_sky_bake")
        return (tex, r, tab) if tables else (tex, r)

    def render(self, prepared: Prepared | Scene, base: np.ndarray, spp: int, timings: list | None = None,
               first_sample: int = 0, flags: int = 0) -> Frame:
        """gpu.rs:4116 Gpu::render: upload (unless given a resident Scene), `spp` samples, readback, Frame."""
        t0 = time.perf_counter()
        resident = isinstance(prepared, Scene)
        scene = prepared if resident else self.upload(prepared)
        try:
            if timings is not None and not resident:
                timings.append(("upload_ms", (time.perf_counter() - t0) * 1e3))
            acc, st = scene.render_raw(base, spp, first_sample=first_sample, flags=flags)
            if timings is not None:
                timings.append(("trace_ms", float(st.device_ms)))
        finally:
            if not resident:
                scene.close()
        w, h = int(base[16]), int(base[17])
        return frame_of(acc, w, h, spp)

    def math_eval(self, fn: int, x: np.ndarray, y: np.ndarray | None = None) -> np.ndarray:
        """trt_math_eval: the device's cosf / sinf / acosf / atan2f (N.TRT_MATH_*) over float32 arrays."""
        x = np.ascontiguousarray(x, np.float32)
        yy = None if y is None else np.ascontiguousarray(y, np.float32)
        out = np.zeros_like(x)
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
        self._check(N.lib().trt_math_eval(self.ctx, fn, fp(x), fp(yy), x.size, fp(out)), "trt_math_eval")
        return out

    def timer_start(self):
        self._check(N.lib().trt_timer_start(self.ctx), "trt_timer_start")

    def timer_stop(self) -> float:
        ms = C.c_float()
        self._check(N.lib().trt_timer_stop(self.ctx, C.byref(ms)), "trt_timer_stop")
        return float(ms.value)

    def synchronize(self):
        self._check(N.lib().trt_synchronize(self.ctx), "trt_synchronize")

    def close(self):
        if self.ctx:
            N.lib().trt_destroy(self.ctx)  # frees the scenes still uploaded through it
            self.ctx = C.c_void_p()
