#!/usr/bin/env python
"""Benchmark of the path-trace pass on the procedural city (config 1).

Workload: 1,984,402 triangles (4,000 seeded boxes and UV spheres, 4,002 units), 200 emissive quads under a light
tree, a 90,000-lux sun and a baked gradient sky; 1280 x 720, 1 spp, max depth 4; the camera on a seeded Catmull-Rom
spline of 240 frames. A step is one frame: one wave of 921,600 paths through every bounce, closest-hit and shadow
rays. `value` counts every ray traced (closest + shadow) per second of device time, all ranks together.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one rank per GPU; each rank renders its own frames of the spline (no collective on the
data path: weak scaling), and the time is the max over ranks. `--impl reference` times the reference algorithm's
CPU restatement (the oracle) on the host's cores over a bounded sample of each frame's pixels: the reference's own
WGSL pass needs a graphics stack that neither this machine nor the GPU box has.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FRAMES = 240
WIDTH, HEIGHT, DEPTH, SPP = 1280, 720, 4, 1
WORKLOAD = ("procedural city 1984402 tris / 4002 units, 1280x720, 1 spp, depth 4, sun + atmosphere sky (baked on the "
            "device, 1024x512) + 400 emitter tris")
METRIC = "Mrays/s (closest + shadow rays, city 720p 1 spp depth 4)"
# Algorithmic bytes a walk reads: a node record, a triangle's leaf record, the part of a unit record the walk reads.
NODE_BYTES, LEAF_BYTES, UNIT_BYTES = 32, 48, 64
WIDE_NODE_BYTES = 80  # a wide node: five 16-byte loads


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def rank_frames(rank: int, world: int, warmup: int, steps: int, frames: int = FRAMES):
    """The frames of the spline a rank renders: warm-up frames, then timed frames, interleaved across ranks so that
    the ranks' timed frames are disjoint (weak scaling: every rank renders `steps` frames)."""
    warm = [(rank + world * i) % frames for i in range(warmup)]
    timed = [(rank + world * (warmup + i)) % frames for i in range(steps)]
    return warm, timed


def reduce_over_ranks(dist, ms: float, e2e_ms: float, rays: float, device=None):
    """The job's time is the slowest rank's (max), its rays every rank's (sum)."""
    if dist is None:
        return ms, e2e_ms, rays
    import torch
    t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    r = torch.tensor([rays], dtype=torch.float64, device=device)
    dist.all_reduce(r, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(r[0])


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def walk_profile(walk: str):
    """The ncu figures of the two walks on this workload, from the committed summary: per kernel, averaged over the
    depths of one frame: DRAM bytes a launch, L1 / L2 hit rates, issue active, lanes active a warp instruction."""
    p = ROOT / "profiles" / f"walks_{walk}_city720p.md"
    if not p.exists():
        return {}
    for line in p.read_text().splitlines():
        if line.startswith("figures:"):
            try:
                return json.loads(line.split(":", 1)[1])
            except ValueError:
                return {}
    return {}


class ClockSampler:
    """nvidia-smi's clocks and throttle reasons of one GPU every 200 ms while it runs."""

    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 10:
                self.rows.append(f)

    def stop(self):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in self.rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[6 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def city_scene():
    from threert_b200 import prep, scenes
    t = time.perf_counter()
    d = scenes.city(width=WIDTH, height=HEIGHT, max_depth=DEPTH)
    P = prep.prepare(d)
    log(f"city: {P.info['n_tris']} tris, {P.info['n_units']} units, prep {time.perf_counter() - t:.1f} s")
    return P


def frame_params(P, frame: int):
    from threert_b200 import prep, scenes
    cam = scenes.city_camera(frame % FRAMES, FRAMES, 1, WIDTH, HEIGHT)
    return prep.set_camera(P.params, cam)


def cpu_sample(P, frames, budget_s: float, threads: int = 0):
    """The oracle over a sample of pixels of the given frames, about `budget_s` of work; rays/s, and what it was."""
    import oracle
    O = oracle.Oracle(P)
    rng = np.random.default_rng(12345)
    n_pix = WIDTH * HEIGHT
    # Calibrate on a small sample, then size the sample to the budget.
    cal = rng.choice(n_pix, 2048, replace=False).astype(np.uint32)
    t = time.perf_counter()
    _, st = O.render(frame_params(P, frames[0]), SPP, pixels=cal, threads=threads)
    dt = max(time.perf_counter() - t, 1e-3)
    px_per_s = len(cal) / dt
    per_frame = int(max(2048, min(n_pix, px_per_s * budget_s / len(frames))))
    rays, secs = 0, 0.0
    for f in frames:
        px = rng.choice(n_pix, per_frame, replace=False).astype(np.uint32)
        t = time.perf_counter()
        _, st = O.render(frame_params(P, f), SPP, pixels=px, threads=threads)
        secs += time.perf_counter() - t
        rays += st["closest_rays"] + st["shadow_rays"]
    cores = threads if threads > 0 else oracle.hardware_threads()
    return rays / secs, cores, f"{per_frame} random pixels x {len(frames)} frames ({per_frame * len(frames)} paths)"


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def bake_sky_on_host(P):
    """The city's atmosphere baked by the oracle's restatement of sky.rs on the host (the CPU arm uses no GPU), written
    into P as the device bake would be (prep.apply_sky)."""
    if P.sky_pending is None:
        return
    import oracle
    from threert_b200 import prep
    atm, sun_light = P.sky_pending
    sky = oracle.Sky(atm.rayleigh_scale, atm.mie_scale, atm.mie_g, tuple(atm.ground_albedo))
    glow = tuple(atm.glow_uniform) + tuple(atm.glow_horizon) + (atm.glow_height,)
    tex, sun, hv = sky.bake(tuple(atm.sun_dir), tuple(atm.sun_lux), atm.altitude_m, atm.width, atm.height, glow,
                            atm.cloud_cover, bool(atm.planet))
    sky.close()

    class _Baked:
        sun_illuminance = tuple(float(v) for v in sun)
        horizon_v = hv

    prep.apply_sky(P, tex, _Baked, sun_light)


def run_reference(args, rank, world):
    """The reference algorithm on the host's cores (its CPU restatement): rank 0 alone."""
    if rank != 0:
        return
    P = city_scene()
    bake_sky_on_host(P)
    steps = max(1, args.steps)
    warm = max(0, args.warmup)
    # Whole run about 100 s: warm-up frames get a small sample, timed frames share the rest.
    if warm:
        cpu_sample(P, list(range(warm)), 5.0)
    value, cores, sample = cpu_sample(P, [warm + i for i in range(steps)], 90.0)
    mrays = value / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": mrays, "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames": FRAMES, "cpu": cpu_model()},
            "cpu_baseline": {"value": mrays, "unit": "Mrays/s", "cores": cores, "kind": "port",
                             "sample": sample + " of the city frames; the reference's WGSL pass needs a graphics "
                                       "stack this box does not have, so its C++ restatement stands in"},
            "e2e": {"value": mrays, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


SPLIT_METRIC = "Mrays/s (closest + shadow rays, one city 720p frame of --spp samples split by sample ranges over the GPUs)"


def run_split(args, rank, world, local, dist):
    """One image across the GPUs: each step is one frame of the city at `--spp` samples; rank r renders its range of
    the samples (threert_b200.split.sample_range) into its accum, copies it into a tensor on its device and one NCCL
    sum-reduce brings the ranks' Pixel records to rank 0 (strong scaling: the frame's work is fixed as N grows). Each
    rank's step time is the device time of its render (CUDA events on the pass's stream) plus that of the reduce
    (CUDA events on torch's stream); the job's is the slowest rank's."""
    import torch
    from threert_b200 import Gpu
    from threert_b200.split import render_split, sample_range
    P = city_scene()
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    S = gpu.upload(P)
    acc = torch.zeros(WIDTH * HEIGHT * 20, dtype=torch.float32, device=f"cuda:{local}")
    frames = [warm for warm in range(args.warmup)] + [args.warmup + i for i in range(args.steps)]

    def step(f):
        t = time.perf_counter()
        st = render_split(S, frame_params(P, f), args.spp, rank, world, None, acc)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if dist:
            dist.reduce(acc, dst=0, op=dist.ReduceOp.SUM)
        e1.record()
        torch.cuda.synchronize()
        return float(st.device_ms) + e0.elapsed_time(e1), st.closest_rays + st.shadow_rays

    for f in frames[:args.warmup]:
        step(f)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms, rays = 0.0, 0
    for f in frames[args.warmup:]:
        m, r = step(f)
        ms += m
        rays += r
    ms_all, _, rays_all = reduce_over_ranks(dist, ms, ms, float(rays), device=f"cuda:{local}")
    first, k = sample_range(rank, world, args.spp)
    line = {"metric": SPLIT_METRIC, "value": rays_all / (ms_all * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD.replace("1 spp", f"{args.spp} spp a frame"), "split": "samples",
                       "samples_per_rank": k, "device": name, "sms": sms,
                       "parallelism": f"sample ranges x{world}, NCCL sum-reduce of the 80-byte Pixel records"},
            "e2e": {"value": rays_all / (ms_all * 1e-3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": 624,
                    "d2h_bytes_per_step": 0}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    S.close()
    gpu.close()


CROWD_DEPTH = 3
CROWD_METRIC = "Mrays/s (closest + shadow rays, crowd 720p 1 spp depth 3, skin + refit + top rebuild each frame)"


def run_crowd(args, rank, world, local, dist):
    """Config 2: 5,000 walking humanoids (20,160 triangles each, 30 bones) in `--groups` pose groups on a 49,928-
    triangle ground under config 1's lights; each frame writes the walkers' records (trt_scene_update), deforms the
    scene on the device (trt_deform: skin, leaf gather, refit of every group's tree, the top tree rebuilt) and renders
    it. The frame's records and palettes are made before the timed region; their copies to the device are in it."""
    import torch
    from threert_b200 import Gpu, crowd, prep
    from threert_b200 import _native as N
    t0 = time.perf_counter()
    c = crowd.crowd(n=5000, groups=args.groups, width=WIDTH, height=HEIGHT, max_depth=CROWD_DEPTH)
    P = prep.prepare(c.desc)
    corners, jobs = crowd.deform_jobs(P, c)
    log(f"crowd: {P.info['n_tris']} tris, {P.info['n_units']} units, {args.groups} pose groups, "
        f"prep {time.perf_counter() - t0:.1f} s")
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    S = gpu.upload(P)
    S.deform_setup(corners, jobs)
    t_inst, _ = crowd.records(P)
    warm_frames, frames = rank_frames(rank, world, args.warmup, args.steps)
    inputs = {}
    for f in set(warm_frames + frames):
        t = f / crowd.FPS
        cam = crowd.crowd_camera(f, WIDTH, HEIGHT, c.extent)
        inputs[f] = (prep.set_camera(P.params, cam), np.ascontiguousarray(crowd.frame_records(P, c, t)),
                     np.ascontiguousarray(crowd.palettes(t, c.phase, c.scale).reshape(-1, 12)))
    L = N.lib()
    # --walk wide: the wide BVH (built once, before the frames) is refit by each trt_deform on the device
    rflags = N.TRT_RENDER_WIDE if args.walk == "wide" else 0

    def frame(f, acc_ptr=None):
        params, rec, pal = inputs[f]
        gpu._check(L.trt_scene_update(S.handle, 3, t_inst * 16, rec.ctypes.data, rec.nbytes), "trt_scene_update")
        p = params.ctypes.data_as(C.POINTER(C.c_uint32))
        gpu._check(L.trt_deform(S.handle, p, pal.ctypes.data_as(C.POINTER(C.c_float)), len(pal), 0, None), "trt_deform")
        gpu._check(L.trt_render(S.handle, p, 0, SPP, rflags, acc_ptr, None), "trt_render")

    def barrier():
        if dist:
            dist.barrier()

    for f in warm_frames:
        frame(f)
    gpu.synchronize()
    S.reset_totals()
    S.set_profiling(True)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    barrier()
    gpu.synchronize()
    clocks.start()
    gpu.timer_start()
    for f in frames:
        frame(f)
    ms = gpu.timer_stop()
    clk = clocks.stop()
    barrier()
    tot = S.totals()
    S.set_profiling(False)
    rays = tot["closest_rays"] + tot["shadow_rays"]
    # The deformation's own stages, frame by frame, untimed above.
    ds = [S.deform(inputs[f][0], inputs[f][2], stats=True) for f in frames[:8]]
    deform = {k: float(np.mean([d[k] for d in ds])) for k in ("device_ms", "skin_ms", "refit_ms", "top_ms", "wide_ms")}
    # End to end: the same frames with the accum read back into pinned memory.
    acc = torch.empty((WIDTH * HEIGHT, N.PIXEL_FLOATS), dtype=torch.float32, pin_memory=True)
    acc_ptr = C.cast(acc.data_ptr(), C.POINTER(C.c_float))
    barrier()
    gpu.synchronize()
    gpu.timer_start()
    for f in frames:
        frame(f, acc_ptr)
    e2e_ms = gpu.timer_stop()
    barrier()
    ms, e2e_ms, rays_all = reduce_over_ranks(dist, ms, e2e_ms, float(rays), device="cuda")
    rec_bytes = inputs[frames[0]][1].nbytes + inputs[frames[0]][2].nbytes + 624
    line = {
        "metric": CROWD_METRIC, "value": rays_all / (ms * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"crowd: 5000 walkers x 20160 tris in {args.groups} pose groups "
                               f"({P.info['n_tris']} tris), 49928-tri ground, 1280x720, 1 spp, depth 3",
                   "frames_per_rank": args.steps, "pose_groups": args.groups, "walk": args.walk,
                   "per_step": "records + palette H2D, trt_deform (skin, leaf gather, refit, top rebuild"
                               + (", wide BVH refit" if rflags else "") + "), render",
                   "device": name, "sms": sms, "parallelism": f"replicas x{world}"},
        "e2e": {"value": rays_all / (e2e_ms * 1e-3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": rec_bytes,
                "d2h_bytes_per_step": WIDTH * HEIGHT * 80},
        "gpu_launches": int(tot["launches"]),
        "clocks": clk,
        "deform_ms_per_step": deform,
        "stage_ms_per_step": {"extend": tot["extend_ms"] / args.steps, "shadow": tot["shadow_ms"] / args.steps,
                              "shade": tot["shade_ms"] / args.steps, "sort": tot["sort_ms"] / args.steps},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    S.close()
    gpu.close()


SERVE_METRIC = "aggregate Mrays/s, serving mix (8 resident scenes; Poisson requests of 256^2..1080p, 1/16/64 spp)"


def serve_scenes():
    """Config 4's resident scenes: two Cornell boxes, three cities and three crowds of different seeds."""
    from threert_b200 import crowd, prep, scenes
    t = time.perf_counter()
    descs = [scenes.cornell(256, 256, seed=0x5EED), scenes.cornell(256, 256, seed=0x1234)]
    descs += [scenes.city(width=WIDTH, height=HEIGHT, max_depth=DEPTH, seed=s) for s in (1, 2, 3)]
    descs += [crowd.crowd(n=5000, groups=1, width=WIDTH, height=HEIGHT, max_depth=DEPTH, seed=s).desc
              for s in (11, 12, 13)]
    Ps = [prep.prepare(d) for d in descs]
    log(f"serve: 8 scenes prepared in {time.perf_counter() - t:.1f} s")
    return Ps


def run_serve(args, rank, world, local):
    """The serving loop on one GPU (replicas beyond: each rank serves its own stream). The mix: each request a
    scene, a resolution of {256^2, 512^2, 1280x720, 1920x1080} and 1, 16 or 64 spp, depth 4, arriving as a seeded
    Poisson stream; then a stream of 720p 1-spp requests. Requests of at most 4 samples get the learned denoiser
    (configs' serving mix): the server denoises them on the device and returns the image. Each stream is also
    rendered one request at a time (trt_render, the denoiser where asked, the read-back) as the reference's serve loop
    does: the baseline of the ratio."""
    from threert_b200 import Gpu, unet
    from threert_b200 import serve as SV
    from threert_b200.prep import params_with
    Ps = serve_scenes()
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    S = [gpu.upload(P) for P in Ps]
    bases = [P.params for P in Ps]
    # The autotuner: wave size and the material sort, on a short burst of the mix (spp 1 and 16).
    tune_reqs = SV.mix_requests(bases, 24, seed=100 + rank, spps=[1, 16])
    best, trials = SV.autotune(gpu, S, tune_reqs)
    log(f"autotune: {trials} -> {best}")
    net = unet.UNet(local, max_batch=1, max_h=1080, max_w=1920)
    net.set_params(np.load(args.denoiser_params) if args.denoiser_params else unet.init_params(0))
    srv = SV.Server(gpu, wave_slots=best["wave_slots"], flags=best["flags"], denoiser=net)
    same = lambda rs: [SV.Request(r.scene, r.params, r.spp, denoise=r.denoise) for r in rs]
    warm = SV.mix_requests(bases, 8, seed=200 + rank, spps=[1])
    SV.run_stream(srv, S, warm, rate=0.0)
    mix = SV.mix_requests(bases, args.requests, seed=300 + rank, denoise_max_spp=4)
    res = SV.run_stream(srv, S, mix, rate=args.rate, seed=400 + rank, keep=False)
    serial = SV.run_serial(gpu, S, same(mix), denoiser=net)
    log(f"mix: served {res}, serial {serial}")
    # 720p, 1 spp, over the three cities: the latency stream.
    rng = np.random.default_rng(500 + rank)
    hd = [SV.Request(int(k), params_with(bases[int(k)], max_bounces=DEPTH), 1, denoise=True)
          for k in rng.integers(2, 5, args.requests)]
    res_hd = SV.run_stream(srv, S, hd, rate=args.rate_720p, seed=600 + rank, keep=False)
    # ... and the same requests all at once (throughput at saturation) against one at a time.
    sat_hd = SV.run_stream(srv, S, same(hd), rate=0.0, keep=False)
    serial_hd = SV.run_serial(gpu, S, same(hd), denoiser=net)
    # 256 x 256, 1 spp over all eight scenes, as fast as they come: where one-at-a-time rendering idles the GPU.
    small = [SV.Request(int(k), params_with(bases[int(k)], width=256, height=256, max_bounces=DEPTH), 1, denoise=True)
             for k in rng.integers(0, 8, 4 * args.requests)]
    res_small = SV.run_stream(srv, S, small, rate=args.rate_small, seed=700 + rank, keep=False)
    serial_small = SV.run_serial(gpu, S, same(small), denoiser=net)
    srv.close()
    net.close()
    line = {
        "metric": SERVE_METRIC, "value": res["mrays_per_s"] * world, "unit": "Mrays/s", "n_gpus": world,
        "steps": res["steps"], "warmup": len(warm), "ms_per_step": res["busy_s"] * 1e3 / max(1, res["steps"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"serving mix: {args.requests} requests at {args.rate} req/s Poisson over 8 resident "
                               "scenes (2 Cornell, 3 city, 3 crowd)", "device": name, "sms": sms,
                   "autotuned": best, "autotune_trials": trials, "parallelism": f"replicas x{world}",
                   "denoiser": "the learned U-Net on requests of <= 4 spp (" +
                               (f"parameters {args.denoiser_params}" if args.denoiser_params else
                                "initial parameters: timing only") + ")",
                   "denoised": int(sum(r.denoise for r in mix))},
        "p50_ms": res["p50_ms"], "p99_ms": res["p99_ms"], "span_s": res["span_s"],
        "serial": {"mrays_per_s": serial["mrays_per_s"], "span_s": serial["span_s"]},
        "speedup_over_serial": res["mrays_per_s"] / serial["mrays_per_s"],
        "stream_720p_1spp": {"rate": args.rate_720p, "requests": len(hd), "p50_ms": res_hd["p50_ms"],
                             "p99_ms": res_hd["p99_ms"], "mrays_per_s_at_rate": res_hd["mrays_per_s"],
                             "mrays_per_s_saturated": sat_hd["mrays_per_s"],
                             "serial_mrays_per_s": serial_hd["mrays_per_s"],
                             "serial_p50_ms": serial_hd["p50_ms"],
                             "speedup_over_serial": sat_hd["mrays_per_s"] / serial_hd["mrays_per_s"]},
        "stream_256_1spp": {"rate": args.rate_small, "requests": len(small), "p50_ms": res_small["p50_ms"],
                            "p99_ms": res_small["p99_ms"], "mrays_per_s": res_small["mrays_per_s"],
                            "serial_mrays_per_s": serial_small["mrays_per_s"],
                            "serial_p50_ms": serial_small["p50_ms"],
                            "speedup_over_serial": res_small["mrays_per_s"] / serial_small["mrays_per_s"]},
        "e2e": {"value": res["mrays_per_s"] * world, "unit": "Mrays/s", "h2d_bytes_per_step": 624,
                "d2h_bytes_per_step": int(np.mean([(12 if r.denoise else 80) * int(r.params[16]) * int(r.params[17])
                                                   for r in mix]))},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for s_ in S:
        s_.close()
    gpu.close()


DENOISE_METRIC = "mean ΔE against 4096 spp at 1280x720: the learned denoiser at 4 spp"


def run_denoise(args, rank, world, local):
    """The learned denoiser, trained here: pairs rendered by the pass (procedural cities of many seeds, 128 x 128,
    1-4 spp with depth against 256 spp), Adam on the device, then judged at 1280 x 720 on held-out seeds against 4096
    spp, beside the a-trous fallback and the plain path at 64 spp (ΔE as renderer/src/compare.rs reports it)."""
    from threert_b200 import Gpu, unet
    from threert_b200 import denoise_train as DT
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    t0 = time.perf_counter()
    F, T = DT.make_dataset(gpu, range(100, 100 + args.scenes), args.views, 128, 128, 256, log=log)
    t_data = time.perf_counter() - t0
    net = unet.UNet(local, max_batch=16, max_h=720, max_w=1280)
    net.set_params(unet.init_params(rank))
    t0 = time.perf_counter()
    losses = DT.train(net, F, T, args.train_steps, batch=16, lr=1e-3, seed=rank, log=log, log_every=2000)
    t_train = time.perf_counter() - t0
    if args.save:
        np.save(args.save, net.params())
    r = DT.judge(gpu, net, [900 + 10 * rank, 901 + 10 * rank], WIDTH, HEIGHT, 4, 64, 4096)
    log(f"judged: {r}")
    line = {
        "metric": DENOISE_METRIC, "value": r["net"]["delta_e"], "unit": "ΔE (CIE76, mean)", "n_gpus": world,
        "steps": args.train_steps, "warmup": 0, "ms_per_step": r["net"]["ms"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
        "config": {"workload": "learned denoiser: 4-level U-Net 32/64/96/128, trained on pairs rendered by the pass, "
                               "judged at 1280x720 on two held-out procedural cities against 4096 spp",
                   "pairs": int(len(F)), "pair_size": "128x128, 1-4 spp vs 256 spp", "batch": 16, "crop": 64,
                   "device": name, "sms": sms},
        "judged": r,
        "target_met": bool(r["net"]["delta_e"] <= r["plain_high"]["delta_e"]
                           and r["net"]["ms"] <= 0.25 * r["plain_high"]["ms"]),
        "training": {"dataset_s": t_data, "train_s": t_train, "first_loss": float(np.mean(losses[:100])),
                     "last_loss": float(np.mean(losses[-100:]))},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    net.close()
    gpu.close()


CORNELL_METRIC = "Mrays/s (closest + shadow rays, Cornell box 256x256, 16 spp, depth 5)"


def run_cornell(args, rank, world, local):
    """Config 0: the Cornell box (36 triangles) at 256 x 256, 16 spp a frame, depth 5, clamp off; a step is one frame
    of 16 samples (trt_render), device-timed. Its working set sits in L1 / L2: the walks' issue rate, not HBM, bounds
    it. CPU baseline: the oracle on the host's threads, the same frames."""
    from threert_b200 import Gpu, prep, scenes
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    P = prep.prepare(scenes.cornell(256, 256))
    S = gpu.upload(P)
    spp = 16
    for k in range(args.warmup):
        S.render_raw(prep.params_with(P.params, seed=1000 + k), spp, read=False)
    ms, rays, paths = 0.0, 0, 0
    for k in range(args.steps):
        _, st = S.render_raw(prep.params_with(P.params, seed=k + 1), spp, read=False)
        ms += st.device_ms
        rays += st.closest_rays + st.shadow_rays
        paths += st.paths
    t = time.perf_counter()
    acc, st = S.render_raw(P.params, spp)
    e2e_ms = (time.perf_counter() - t) * 1e3
    line = {
        "metric": CORNELL_METRIC, "value": rays * world / (ms * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "Cornell box 36 tris, 256x256, 16 spp a step, depth 5", "device": name, "sms": sms},
        "paths_per_s": paths / (ms * 1e-3), "rays_per_path": rays / max(1, paths),
        "e2e": {"value": (st.closest_rays + st.shadow_rays) / (e2e_ms * 1e-3) / 1e6, "unit": "Mrays/s",
                "h2d_bytes_per_step": 624, "d2h_bytes_per_step": 256 * 256 * 80},
    }
    if not args.no_cpu and rank == 0:
        import oracle
        O = oracle.Oracle(P)
        t = time.perf_counter()
        _, cs = O.render(P.params, spp)
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": (cs["closest_rays"] + cs["shadow_rays"]) / dt / 1e6, "unit": "Mrays/s",
                                "cores": oracle.hardware_threads(), "kind": "port",
                                "sample": "one frame of 16 spp on every host thread"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    S.close()
    gpu.close()


SKY_METRIC = "ms per sky re-bake on the device (atmosphere 1024x512, a moving sun: sky.rs bake_atmosphere_tables)"


def run_sky(args, rank, world, local):
    """The atmosphere's sky on the device: the tables once (Luts::build), then a re-bake each step with the sun moved
    a quarter degree (a dynamic sun: the tables kept), 1024 x 512 as the offline bake's size; and the same re-bake
    into a resident scene in place (trt_scene_set_sky: texels, CDF, the sun's colour). CPU baseline: the oracle's
    restatement of sky.rs on all host threads (the reference bakes with rayon on all cores)."""
    import math
    import ctypes as C
    from threert_b200 import Gpu, prep, scenes
    from threert_b200 import _native as N
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    d = scenes.city(n_objects=60, width=64, height=36, n_emitters=20, sky_size=(1024, 512))
    P = prep.prepare(d)
    atm, sun_light = P.sky_pending

    def at(elev_deg):
        e, a = math.radians(elev_deg), math.radians(35.0)
        atm.sun_dir = (N.f32 * 3)(math.cos(e) * math.cos(a), math.sin(e), math.cos(e) * math.sin(a))
        return atm

    _, cold = gpu.bake_sky(at(28.0))
    S = gpu.upload(P)
    elevs = [28.0 + 0.25 * k for k in range(args.warmup + args.steps)]
    for e in elevs[:args.warmup]:
        gpu.bake_sky(at(e))
        S.set_sky(at(e), sun_light, P.info["env_nee_floor"], P.params.copy())
    bake_ms, scene_ms, wall = [], [], []
    for e in elevs[args.warmup:]:
        _, r = gpu.bake_sky(at(e))
        bake_ms.append(r.bake_ms)
        t = time.perf_counter()
        r2 = S.set_sky(at(e), sun_light, P.info["env_nee_floor"], P.params.copy())
        wall.append((time.perf_counter() - t) * 1e3)
        scene_ms.append(r2.bake_ms)
    ms = float(np.mean(bake_ms))
    line = {
        "metric": SKY_METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "atmosphere sky bake 1024x512 (orders 2-4, 12 / 16 Simpson steps), sun moving "
                               "0.25 degrees a step from 28 degrees", "device": name, "sms": sms},
        "tables_ms": cold.tables_ms, "first_bake_ms": cold.bake_ms,
        "scene_rebake_ms": float(np.mean(scene_ms)),
        "e2e": {"value": float(np.mean(wall)), "unit": "ms", "h2d_bytes_per_step": 2048,
                "d2h_bytes_per_step": 24},
    }
    if not args.no_cpu and rank == 0:
        import oracle
        t = time.perf_counter()
        sky = oracle.Sky(atm.rayleigh_scale, atm.mie_scale, atm.mie_g, tuple(atm.ground_albedo))
        t_tables = (time.perf_counter() - t) * 1e3
        t = time.perf_counter()
        n_cpu = 3
        for k in range(n_cpu):
            a = at(28.0 + 0.25 * k)
            sky.bake(tuple(a.sun_dir), tuple(a.sun_lux), a.altitude_m, 1024, 512)
        t_bake = (time.perf_counter() - t) * 1e3 / n_cpu
        sky.close()
        line["cpu_baseline"] = {"value": t_bake, "unit": "ms", "cores": min(oracle.hardware_threads(), 32),
                                "kind": "port", "sample": f"{n_cpu} bakes of 1024x512 after the tables "
                                                          f"({t_tables:.0f} ms)",
                                "tables_ms": t_tables}
    if rank == 0:
        print(json.dumps(line), flush=True)
    S.close()
    gpu.close()


TRUTH_SPP = 4096


def run_extras(gpu, S, P, frame: int, args, flags: int) -> dict:
    """The rest of the headline metric on the benched frame (rank 0): ΔE against a 4096-spp render of the same frame
    (renderer/src/compare.rs, as threert_b200.metrics computes it) for the plain path at 1, 4 and 64 spp and for the
    learned denoiser at 4 spp, the denoiser trained here first on pairs the pass renders (small procedural cities of
    other seeds, 128 x 128, 1-4 spp against 256 spp); the plain path at the denoiser's device time (ΔE at equal ms);
    and serving: 720p 1-spp denoised requests of the city's spline frames through the library's server, a saturated
    burst for its capacity, then a Poisson stream at 70 % of it for p50 / p99, against one request at a time."""
    from threert_b200 import metrics, prep, unet
    from threert_b200 import denoise_train as DT
    from threert_b200 import serve as SV
    from threert_b200 import _native as N
    from threert_b200.gpu import frame_of
    out = {}
    params = frame_params(P, frame)
    t0 = time.perf_counter()
    truth_acc, st_t = S.render_raw(prep.params_with(params, seed=0xACE), TRUTH_SPP, flags=flags)
    truth = frame_of(truth_acc, WIDTH, HEIGHT, TRUTH_SPP).color
    log(f"extras: truth {TRUTH_SPP} spp in {st_t.device_ms / 1e3:.1f} s")
    de = lambda img: metrics.delta_e(truth, img)["mean"]
    plain = {}
    for spp in (1, 4, 64):
        acc, st = S.render_timed(params, spp, flags=flags)
        plain[spp] = {"delta_e": de(frame_of(acc, WIDTH, HEIGHT, spp).color), "ms": float(st.device_ms)}
    # The learned denoiser, trained on the device by the library's own kernels.
    t1 = time.perf_counter()
    F, T = DT.make_dataset(gpu, range(100, 100 + args.extras_scenes), 16, 128, 128, 256)
    t_data = time.perf_counter() - t1
    net = unet.UNet(0, max_batch=16, max_h=HEIGHT, max_w=WIDTH)
    net.set_params(unet.init_params(0))
    t1 = time.perf_counter()
    losses = DT.train(net, F, T, args.extras_train_steps, batch=16, lr=1e-3, seed=0)
    t_train = time.perf_counter() - t1
    del F, T
    acc, st = S.render_timed(params, 4, flags=flags | N.TRT_RENDER_DEPTH)
    den, ms_net = net.denoise(S)
    at, ms_at = S.denoise_atrous(4)
    ms_den = float(st.device_ms) + ms_net
    # The plain path at the denoised frame's device time: as many samples as that time renders (a sample's time from
    # the 64-sample render, where the per-call overhead is spread thin).
    spp_eq = max(1, int(round(ms_den / max(plain[64]["ms"] / 64.0, 1e-6))))
    acc_eq, st_eq = S.render_timed(params, spp_eq, flags=flags)
    learned = {"delta_e": de(den), "ms": ms_den, "network_ms": ms_net}
    out["delta_e"] = {
        "truth_spp": TRUTH_SPP, "frame": frame, "metric": "mean ΔE (CIE76) of 8-bit sRGB at a fixed exposure",
        "ms": "device time of the render (and the filter), its accum left on the device",
        "plain_1spp": plain[1], "plain_4spp": plain[4], "plain_64spp": plain[64],
        "atrous_4spp": {"delta_e": de(at), "ms": float(st.device_ms) + ms_at},
        "learned_4spp": learned,
        "plain_at_equal_ms": {"spp": spp_eq, "delta_e": de(frame_of(acc_eq, WIDTH, HEIGHT, spp_eq).color),
                              "ms": float(st_eq.device_ms)},
        "target_met": bool(learned["delta_e"] <= plain[64]["delta_e"] and ms_den <= 0.25 * plain[64]["ms"]),
        "training": {"pairs": 16 * args.extras_scenes, "steps": args.extras_train_steps, "dataset_s": t_data,
                     "train_s": t_train, "first_loss": float(np.mean(losses[:100])),
                     "last_loss": float(np.mean(losses[-100:]))},
        "held_out": "trained on small procedural cities of seeds 100+, judged on the benched city (seed 1)"}
    # Serving 720p 1-spp denoised requests on the resident city.
    reqs = lambda n, off: [SV.Request(0, frame_params(P, off + 3 * k), 1, denoise=True) for k in range(n)]
    srv = SV.Server(gpu, denoiser=net)
    try:
        SV.run_stream(srv, [S], reqs(8, 100), rate=0.0, keep=False)  # warm-up: pools, graphs
        sat = SV.run_stream(srv, [S], reqs(64, 1), rate=0.0, keep=False)
        cap = 64 / sat["span_s"]
        at_rate = SV.run_stream(srv, [S], reqs(128, 2), rate=0.7 * cap, seed=7, keep=False)
    finally:
        srv.close()
    serial = SV.run_serial(gpu, [S], reqs(64, 1), denoiser=net)
    out["serve_720p"] = {
        "requests": "1280x720, 1 spp, depth 4, denoised by the learned U-Net on the device, image read back",
        "capacity_req_per_s": cap, "rate_req_per_s": 0.7 * cap, "p50_ms": at_rate["p50_ms"],
        "p99_ms": at_rate["p99_ms"], "mrays_per_s_at_rate": at_rate["mrays_per_s"],
        "mrays_per_s_saturated": sat["mrays_per_s"], "serial_mrays_per_s": serial["mrays_per_s"],
        "serial_p50_ms": serial["p50_ms"], "speedup_over_serial": sat["mrays_per_s"] / serial["mrays_per_s"],
        "serial_gpu_busy_frac": serial["gpu_busy_frac"],
        "speedup_bound": 1.0 / max(serial["gpu_busy_frac"], 1e-9)}
    net.close()
    log(f"extras: {time.perf_counter() - t0:.1f} s")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--walk", default="binary", choices=["binary", "wide"],
                    help="the reference's binary trees (fastest measured here) or the 8-wide quantised BVH")
    ap.add_argument("--sort", default="hits",
                    help="coherence sorts on the device: 'none', or a comma list of rays, hits, shadows "
                         "(hits by material is the pass's default; the other two measured slower here)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extras", action="store_true",
                    help="city: skip the image-quality and serving figures (ΔE against 4096 spp, the learned "
                         "denoiser at equal ms, 720p serving latency)")
    ap.add_argument("--extras-train-steps", type=int, default=20000, help="city extras: the denoiser's Adam steps")
    ap.add_argument("--extras-scenes", type=int, default=32, help="city extras: procedural cities for training")
    ap.add_argument("--workload", default="city", choices=["city", "crowd", "serve", "denoise", "sky", "cornell"],
                    help="city (the headline workload), the crowd with its per-frame deformation, the serving mix, "
                         "the learned denoiser (trained, then judged), the atmosphere's sky bake, or the Cornell box")
    ap.add_argument("--scenes", type=int, default=64, help="denoise: procedural cities rendered for training")
    ap.add_argument("--views", type=int, default=16, help="denoise: views of each")
    ap.add_argument("--train-steps", type=int, default=40000, help="denoise: Adam steps")
    ap.add_argument("--save", default="", help="denoise: where to save the trained parameters (.npy)")
    ap.add_argument("--denoiser-params", default="", help="serve: the learned denoiser's parameters (.npy)")
    ap.add_argument("--requests", type=int, default=64, help="serve: requests a stream")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: the mix's arrival rate (requests a second)")
    ap.add_argument("--rate-720p", type=float, default=60.0, help="serve: the 720p stream's arrival rate")
    ap.add_argument("--rate-small", type=float, default=2000.0, help="serve: the 256^2 stream's arrival rate")
    ap.add_argument("--groups", type=int, default=1, help="crowd: pose groups (skinned copies of the humanoid)")
    ap.add_argument("--split", default="frames", choices=["frames", "samples"],
                    help="city on N GPUs: disjoint frames a rank (weak scaling), or one frame's samples split by "
                         "sample ranges with an NCCL sum-reduce of the accum (strong scaling)")
    ap.add_argument("--spp", type=int, default=16, help="split samples: samples a frame")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.workload != "city":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the CPU arm times the city workload only"}))
            return
        run_reference(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    if args.workload == "cornell":
        run_cornell(args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload == "sky":
        run_sky(args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload == "denoise":
        run_denoise(args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload == "serve":
        run_serve(args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload == "city" and args.split == "samples":
        run_split(args, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return
    if args.workload == "crowd":
        run_crowd(args, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return

    from threert_b200 import Gpu
    from threert_b200 import _native as N

    P = city_scene()
    gpu = Gpu(local)
    name, sms = gpu.device_info()
    S = gpu.upload(P)
    flags = N.TRT_RENDER_WIDE if args.walk == "wide" else 0
    sorts = [] if args.sort == "none" else args.sort.split(",")
    if "hits" not in sorts:
        flags |= N.TRT_RENDER_UNSORTED_HITS
    flags |= (N.TRT_RENDER_SORT_RAYS if "rays" in sorts else 0) | (N.TRT_RENDER_SORT_SHADOWS if "shadows" in sorts else 0)
    warm_frames, frames = rank_frames(rank, world, args.warmup, args.steps)
    params = {f: frame_params(P, f) for f in set(frames + warm_frames)}

    def barrier():
        if dist:
            dist.barrier()

    for f in warm_frames:
        S.render_raw(params[f], SPP, flags=flags, read=False, stats=False)
    gpu.synchronize()

    # Timed: K frames, device time on the pass's own stream.
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    S.reset_totals()
    S.set_profiling(True)
    clocks = ClockSampler(uuid)
    barrier()
    gpu.synchronize()
    clocks.start()
    gpu.timer_start()
    for f in frames:
        S.render_raw(params[f], SPP, flags=flags, read=False, stats=False)
    ms = gpu.timer_stop()
    clk = clocks.stop()
    barrier()
    tot = S.totals()
    S.set_profiling(False)
    rays = tot["closest_rays"] + tot["shadow_rays"]
    launches = tot["launches"]
    ext_avg_ms = tot["extend_ms"] / max(1, tot["extend_launches"])

    # End to end through the C ABI: each frame's Params from the host, its accum read back into pinned memory. First
    # as the reference's render returns (the call waits for its read-back), then with the read-back of each frame
    # overlapping the next frame's render (TRT_RENDER_ASYNC_READBACK: two host buffers in turn); the timer's stop
    # waits for the last copy.
    accs = [torch.empty((WIDTH * HEIGHT, N.PIXEL_FLOATS), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    acc_ptrs = [C.cast(a.data_ptr(), C.POINTER(C.c_float)) for a in accs]
    L = N.lib()
    pinned = {f: torch.from_numpy(params[f].astype(np.uint32).view(np.int32)).pin_memory() for f in frames}
    barrier()
    gpu.synchronize()
    gpu.timer_start()
    for f in frames:
        p = C.cast(pinned[f].data_ptr(), C.POINTER(C.c_uint32))
        gpu._check(L.trt_render(S.handle, p, 0, SPP, flags, acc_ptrs[0], None), "trt_render")
    e2e_sync_ms = gpu.timer_stop()
    barrier()
    gpu.synchronize()
    gpu.timer_start()
    for k, f in enumerate(frames):
        p = C.cast(pinned[f].data_ptr(), C.POINTER(C.c_uint32))
        gpu._check(L.trt_render(S.handle, p, 0, SPP, flags | N.TRT_RENDER_ASYNC_READBACK, acc_ptrs[k % 2], None),
                   "trt_render")
    e2e_ms = gpu.timer_stop()
    barrier()

    # The walks' reads over the same frames, untimed (a counting walk).
    S.reset_totals()
    for f in frames:
        S.render_raw(params[f], SPP, flags=flags | N.TRT_RENDER_COUNT, read=False, stats=False)
    cnt = S.totals()
    node_bytes = WIDE_NODE_BYTES if args.walk == "wide" else NODE_BYTES
    ext_bytes = (cnt["node_visits"] * node_bytes + cnt["tri_tests"] * LEAF_BYTES + cnt["unit_entries"] * UNIT_BYTES)
    sha_bytes = (cnt["shadow_node_visits"] * node_bytes + cnt["shadow_tri_tests"] * LEAF_BYTES
                 + cnt["shadow_unit_entries"] * UNIT_BYTES)
    per_ray = lambda k, n: cnt[k] / max(1, n)
    walk_counts = {
        "closest": {"rays": int(cnt["closest_rays"]), "nodes": per_ray("node_visits", cnt["closest_rays"]),
                    "tris": per_ray("tri_tests", cnt["closest_rays"]),
                    "units": per_ray("unit_entries", cnt["closest_rays"])},
        "shadow": {"rays": int(cnt["shadow_rays"]), "nodes": per_ray("shadow_node_visits", cnt["shadow_rays"]),
                   "tris": per_ray("shadow_tri_tests", cnt["shadow_rays"]),
                   "units": per_ray("shadow_unit_entries", cnt["shadow_rays"])},
        "node_bytes": node_bytes}
    ext_bytes_per_launch = ext_bytes / max(1, cnt["extend_launches"])
    sha_bytes_per_launch = sha_bytes / max(1, cnt["shadow_launches"])
    sha_avg_ms = tot["shadow_ms"] / max(1, tot["shadow_launches"])

    ms, e2e_ms, rays_all = reduce_over_ranks(dist, ms, e2e_ms, float(rays), device="cuda")
    e2e_sync_ms, _, _ = reduce_over_ranks(dist, e2e_sync_ms, e2e_sync_ms, 0.0, device="cuda")

    peak, peak_kind = measured_peaks()
    prof = walk_profile(args.walk)

    def roof(kernel, bytes_per_launch, launch_ms, rays_walked):
        """Algorithmic bytes a launch (node records, leaf records, unit records the walk reads, counted by the
        walk itself) over the launch's device time, against the measured HBM copy bandwidth. The walks' reads are
        mostly L1 / L2 hits: the profile's DRAM traffic and lane figures say what bounds them."""
        achieved = bytes_per_launch / (launch_ms * 1e-3) / 1e9 if launch_ms > 0 else None
        pf = prof.get(kernel, {})
        traffic = pf.get("dram_bytes_per_launch")
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic, "kernel": kernel,
                "peak_kind": f"{peak_kind} hbm_gbs", "bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms,
                "bytes_per_ray": bytes_per_launch * (cnt["extend_launches"] if kernel == "k_extend"
                                                     else cnt["shadow_launches"]) / max(1, rays_walked),
                "dram_frac_of_peak": (traffic / (launch_ms * 1e-3) / 1e9 / peak) if traffic and launch_ms else None,
                "l1_hit_pct": pf.get("l1_hit_pct"), "l2_hit_pct": pf.get("l2_hit_pct"),
                "issue_active_pct": pf.get("issue_active_pct"), "lanes_active_of_32": pf.get("lanes"),
                "limiter": pf.get("limiter"), "profile": f"profiles/walks_{args.walk}_city720p.md" if pf else None}

    rooflines = {"k_extend": roof("k_extend", ext_bytes_per_launch, ext_avg_ms, cnt["closest_rays"]),
                 "k_shadow": roof("k_shadow", sha_bytes_per_launch, sha_avg_ms, cnt["shadow_rays"])}
    dominant = "k_shadow" if tot["shadow_ms"] >= tot["extend_ms"] else "k_extend"
    # The walks run beside other kernels (each depth's shadow walk beside the next depth's closest-hit walk, the two
    # half-waves side by side): a launch's events span its share of the GPU, not the GPU alone. The frame's aggregate
    # says the same against the frame's own time.
    walk_frame_gbs = (ext_bytes + sha_bytes) / max(1, args.steps) / (ms / args.steps * 1e-3) / 1e9
    for r_ in rooflines.values():
        r_["concurrency"] = ("launched beside other kernels (the other half-wave's, and the next depth's closest-hit "
                             "walk beside each shadow walk): the launch's event span is its share of the GPU")
        r_["walks_frame_achieved"] = walk_frame_gbs
        r_["walks_frame_frac"] = walk_frame_gbs / peak
    line = {
        "metric": METRIC, "value": rays_all / (ms * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "frames_per_rank": args.steps, "walk": args.walk, "sort": args.sort,
                   "l2": "inputs larger than L2: 221 MB of scene buffers, each step a new camera along the spline",
                   "device": name, "sms": sms, "parallelism": f"replicas x{world}, frames split across ranks"},
        "e2e": {"value": rays_all / (e2e_ms * 1e-3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": 624,
                "d2h_bytes_per_step": WIDTH * HEIGHT * 80,
                "readback": "each frame's 73.7 MB accum into pinned host memory, overlapping the next frame's render "
                            "(TRT_RENDER_ASYNC_READBACK); the timer's stop waits for the last copy",
                "value_readback_waited": rays_all / (e2e_sync_ms * 1e-3) / 1e6},
        "gpu_launches": int(launches),
        "roofline": rooflines[dominant],
        "rooflines": rooflines,
        "clocks": clk,
        "rays_per_path": rays / max(1, tot["paths"]),
        "walk_counts": walk_counts,
        "paths_per_s": tot["paths"] * world / (ms * 1e-3),
        "stage_ms_per_step": {"extend": tot["extend_ms"] / args.steps, "shadow": tot["shadow_ms"] / args.steps,
                              "shade": tot["shade_ms"] / args.steps, "sort": tot["sort_ms"] / args.steps},
    }
    if rank == 0 and not args.no_extras:
        try:
            line.update(run_extras(gpu, S, P, frames[0], args, flags))
        except Exception as e:  # (the throughput line stands without them)
            line["extras_error"] = f"{type(e).__name__}: {e}"
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, sample = cpu_sample(P, frames[:4], 20.0)
        line["cpu_baseline"] = {"value": v / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "port",
                                "sample": sample + f"; host CPU: {cpu_model()}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    S.close()
    gpu.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
