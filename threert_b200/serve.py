"""Serving from Python: the library's request loop (trt_server_*), the request mix it is measured on, an open-loop
Poisson driver, the one-request-at-a-time baseline, and the autotuner that picks the server's wave size.

The reference serves JSON-line jobs one at a time (renderer/src/main.rs:345-397). `Server` keeps scenes resident and
lets the library's worker batch the samples of every request in flight into shared waves; a request submitted while
others run joins the next wave. Each result is the accum `Scene.render_raw` makes alone, bit for bit.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .gpu import Gpu, Scene
from .prep import params_with


@dataclass
class Request:
    scene: int            # index into the server's scene list
    params: np.ndarray    # 156-word Params (its size is the image's)
    spp: int
    id: int = 0
    accum: np.ndarray | None = None
    done: dict = field(default_factory=dict)
    denoise: bool = False             # the server's learned denoiser on its result (rgb) instead of the accum
    rgb: np.ndarray | None = None     # (h * w, 3) float32, the denoised image

    @property
    def paths(self) -> int:
        return int(self.params[16]) * int(self.params[17]) * self.spp


class Server:
    """trt_server: a worker thread, its streams and wave state on the Gpu's device."""

    def __init__(self, gpu: Gpu, wave_slots: int = 0, max_active: int = 0, hbm_reserve: int = 0, flags: int = 0,
                 launch_mode: int = 0, denoiser=None, denoise_max_spp: int = 4):
        """denoiser: None, or a threert_b200.unet.UNet the server owns until closed (requests with denoise=True)."""
        self.gpu = gpu
        self.handle = C.c_void_p()
        self.denoiser = denoiser
        o = N.ServerOptions(wave_slots, max_active, hbm_reserve, flags, launch_mode,
                            denoiser.handle if denoiser is not None else None, denoise_max_spp)
        gpu._check(N.lib().trt_server_create(gpu.ctx, C.byref(o), C.byref(self.handle)), "trt_server_create")
        self.live: dict[int, Request] = {}
        self.pool: dict[int, list] = {}  # pinned result buffers by pixel count, free for reuse
        self.pinned: dict[int, object] = {}  # the pinned allocation behind each buffer, by address

    def _buffer(self, pixels: int, cols: int = N.PIXEL_FLOATS) -> np.ndarray:
        """A result buffer in pinned host memory (the read-back then runs at full speed, off the worker's path)."""
        free = self.pool.get((pixels, cols))
        if free:
            return free.pop()
        return pinned_buffer(pixels, self.pinned, cols)

    def reserve(self, requests: list[Request]):
        """Allocates, ahead of time, a pinned result buffer for each of these requests (pinned allocations take
        milliseconds: made while submitting, they would hold the submitter back)."""
        need: dict[tuple, int] = {}
        for r in requests:
            key = (int(r.params[16]) * int(r.params[17]), 3 if r.denoise else N.PIXEL_FLOATS)
            need[key] = need.get(key, 0) + 1
        for key, n in need.items():
            have = self.pool.setdefault(key, [])
            while len(have) < n:
                have.append(pinned_buffer(key[0], self.pinned, key[1]))

    def release(self, req: Request):
        """Returns a finished request's result buffer to the pool (its accum is not to be read after this)."""
        for name in ("accum", "rgb"):
            a = getattr(req, name)
            if a is not None:
                self.pool.setdefault(a.shape, []).append(a)
                setattr(req, name, None)

    def clock(self) -> float:
        """The server's clock (ms since it was created), the one request times are on."""
        now = C.c_double()
        self.gpu._check(N.lib().trt_server_clock(self.handle, C.byref(now)), "trt_server_clock")
        return now.value

    def submit(self, scene: Scene, req: Request, at_ms: float | None = None) -> int:
        """Queues the request now, or (at_ms) for its arrival at that time on the server's clock."""
        p = np.ascontiguousarray(req.params, dtype=np.uint32)
        px = int(p[16]) * int(p[17])
        rid = C.c_uint64()
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
        if req.denoise:
            req.accum, req.rgb = None, self._buffer(px, 3)
        else:
            req.accum, req.rgb = self._buffer(px), None
        self.gpu._check(N.lib().trt_server_submit_at(self.handle, scene.handle,
                                                     p.ctypes.data_as(C.POINTER(C.c_uint32)), req.spp, fp(req.accum),
                                                     fp(req.rgb), -1.0 if at_ms is None else float(at_ms),
                                                     C.byref(rid)), "trt_server_submit_at")
        req.id = rid.value
        self.live[req.id] = req
        return req.id

    def poll(self, wait_ms: int = 0) -> list[Request]:
        buf = (N.RequestDone * 64)()
        n = C.c_uint32()
        self.gpu._check(N.lib().trt_server_poll(self.handle, buf, 64, C.byref(n), wait_ms), "trt_server_poll")
        out = []
        for i in range(n.value):
            d = {f[0]: getattr(buf[i], f[0]) for f in N.RequestDone._fields_}
            r = self.live.pop(d["id"])
            r.done = d
            out.append(r)
        return out

    def stats(self) -> dict:
        st = N.ServerStats()
        self.gpu._check(N.lib().trt_server_stats_get(self.handle, C.byref(st)), "trt_server_stats_get")
        return {f[0]: getattr(st, f[0]) for f in N.ServerStats._fields_}

    def close(self):
        if self.handle:
            N.lib().trt_server_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# The serving mix: resolutions and sample counts a request draws from (uniformly).
RESOLUTIONS = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
SPPS = [1, 16, 64]


def pinned_buffer(pixels: int, keep: dict, cols: int = N.PIXEL_FLOATS) -> np.ndarray:
    """A (pixels, cols) float32 array in pinned host memory; `keep` holds the allocation for as long as it is used."""
    import torch
    t = torch.empty((pixels, cols), dtype=torch.float32, pin_memory=True)
    a = t.numpy()
    keep[a.ctypes.data] = t
    return a


def mix_requests(bases: list[np.ndarray], n: int, seed: int = 0, resolutions=RESOLUTIONS, spps=SPPS,
                 max_bounces: int = 4, denoise_max_spp: int = 0) -> list[Request]:
    """n requests over the scenes whose base Params are `bases`: scene, resolution and spp drawn uniformly; those of
    at most `denoise_max_spp` samples denoised (0: none)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        k = int(rng.integers(len(bases)))
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        p = params_with(bases[k], width=w, height=h, max_bounces=max_bounces)
        spp = int(spps[int(rng.integers(len(spps)))])
        out.append(Request(k, p, spp, denoise=spp <= denoise_max_spp))
    return out


def run_stream(server: Server, scenes: list[Scene], requests: list[Request], rate: float, seed: int = 1,
               timeout_s: float = 600.0, keep: bool = True, lead_ms: float = 5.0) -> dict:
    """Hands the requests to the server at once with Poisson arrival times of `rate` a second on its clock, the first
    `lead_ms` from now (an open loop the library's worker paces: no host thread times the arrivals), and waits for
    every one: latencies (done - arrival, ms), the span from the first arrival to the last completion, rays."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(requests)) if rate > 0 else np.zeros(len(requests))
    server.reserve(requests)
    before = server.stats()
    done: list[Request] = []
    t0 = time.perf_counter()
    at = server.clock() + lead_ms + np.cumsum(gaps) * 1e3
    for r, a in zip(requests, at):
        server.submit(scenes[r.scene], r, at_ms=float(a))
    while len(done) < len(requests) and time.perf_counter() - t0 < timeout_s:
        got = server.poll(wait_ms=20)
        if not keep:
            for r in got:
                server.release(r)
        done += got
    if len(done) < len(requests):
        raise TimeoutError(f"{len(done)} of {len(requests)} requests done in {timeout_s} s")
    after = server.stats()
    lat = np.array([r.done["done_ms"] - r.done["submit_ms"] for r in done])
    span = (max(r.done["done_ms"] for r in done) - min(r.done["submit_ms"] for r in done)) * 1e-3
    rays = (after["closest_rays"] + after["shadow_rays"]) - (before["closest_rays"] + before["shadow_rays"])
    return {"requests": len(done), "failed": sum(r.done["status"] != 0 for r in done),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "span_s": span, "rays": int(rays), "mrays_per_s": rays / span / 1e6,
            "paths": int(after["paths"] - before["paths"]), "steps": int(after["steps"] - before["steps"]),
            "busy_s": (after["busy_ms"] - before["busy_ms"]) * 1e-3}


def run_serial(gpu: Gpu, scenes: list[Scene], requests: list[Request], denoiser=None) -> dict:
    """The reference's way: each request rendered alone through trt_render and read back before the next starts (a
    denoised request: rendered with its depth guide, denoised by `denoiser`, its image read back)."""
    rays = 0
    lat = []
    keep, bufs = {}, {}
    for r in requests:  # pinned read-back buffers, as the server's
        px = int(r.params[16]) * int(r.params[17])
        if px not in bufs:
            bufs[px] = pinned_buffer(px, keep)
    busy_ms = 0.0
    t0 = time.perf_counter()
    for r in requests:
        t = time.perf_counter()
        S = scenes[r.scene]
        if r.denoise:
            _, st = S.render_raw(r.params, r.spp, flags=N.TRT_RENDER_DEPTH, read=False)
            _, ms_net = denoiser.denoise(S)
            busy_ms += ms_net
        else:
            acc, st = S.render_raw(r.params, r.spp, out=bufs[int(r.params[16]) * int(r.params[17])])
        busy_ms += float(st.device_ms)
        lat.append((time.perf_counter() - t) * 1e3)
        rays += st.closest_rays + st.shadow_rays
    span = time.perf_counter() - t0
    # The share of the span the device was busy with the requests' kernels: 1 / it bounds what batching can gain.
    return {"requests": len(requests), "span_s": span, "rays": int(rays), "mrays_per_s": rays / span / 1e6,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "gpu_busy_frac": busy_ms * 1e-3 / span}


def autotune(gpu: Gpu, scenes: list[Scene], requests: list[Request], candidates=(1 << 20, 2 << 20, 4 << 20),
             flags_options=(0, N.TRT_RENDER_UNSORTED_HITS)) -> tuple[dict, list]:
    """Times the requests back to back (all submitted at once) under each wave size and sort setting; returns the
    fastest options and every trial (Mrays/s). The wave must hold the largest request's image."""
    need = max(((int(r.params[16]) + 7) // 8) * ((int(r.params[17]) + 3) // 4) * 32 for r in requests)
    trials = []
    for slots in candidates:
        if slots < need:
            continue
        for flags in flags_options:
            srv = Server(gpu, wave_slots=slots, flags=flags)
            try:
                best_run = None
                for _ in range(2):  # the better of two runs (the first also warms the server's pools)
                    copies = [Request(r.scene, r.params, r.spp) for r in requests]
                    res = run_stream(srv, scenes, copies, rate=0.0, keep=False)
                    if best_run is None or res["mrays_per_s"] > best_run["mrays_per_s"]:
                        best_run = res
            finally:
                srv.close()
            trials.append({"wave_slots": slots, "flags": flags, "mrays_per_s": best_run["mrays_per_s"],
                           "span_s": best_run["span_s"]})
    best = max(trials, key=lambda t: t["mrays_per_s"])
    return best, trials
