"""Small, self-contained runs of the library's kernels for profilers (`ncu ... python -m threert_b200.profile_cases
CASE`): each case prepares its input, runs the kernels of interest a few times and exits.

  city     one warm-up and two frames of the city at 1280 x 720, 1 spp, depth 4 (k_extend, k_shade, k_shadow, ...)
  city_wide  the same frames walking the 8-wide BVH
  unet     the learned denoiser's network on a 1280 x 720 image, three times (k_conv), and one training step on a
           batch of 16 crops of 64 x 64 (k_conv, k_wgrad)
  crowd    the crowd's deformation, three frames, at K pose groups (k_skin, k_refit_leaves, k_refit, k_top_*)
  sky      the atmosphere's tables and three 1024 x 512 bakes with the sun moving, then a re-bake into a resident
           scene (the sky kernels, the environment's texels and CDF)
  emitters the city's emitters re-weighed three times (the emitter-weight kernels)
  cornell  three frames of the Cornell box, 256 x 256, 16 spp
"""
from __future__ import annotations

import sys

import numpy as np


def city(flags: int = 0):
    from threert_b200 import Gpu, prep, scenes
    P = prep.prepare(scenes.city())
    g = Gpu(0)
    S = g.upload(P)
    for f in range(3):
        cam = scenes.city_camera(f, 240, 1, P.width, P.height)
        S.render_raw(prep.set_camera(P.params, cam), 1, flags=flags, read=False, stats=False)
    g.synchronize()
    S.close()
    g.close()


def unet_case():
    from threert_b200 import unet
    net = unet.UNet(0, max_batch=16, max_h=720, max_w=1280)
    net.set_params(unet.init_params(0))
    rng = np.random.default_rng(0)
    f = rng.normal(0, 1, (1, 720, 1280, unet.N_FEAT)).astype(np.float32)
    for _ in range(3):
        net.forward(f)
    fb = rng.normal(0, 1, (16, 64, 64, unet.N_FEAT)).astype(np.float32)
    tb = rng.normal(0, 1, (16, 64, 64, 3)).astype(np.float32)
    net.step(fb, tb)
    net.close()


def crowd_case(groups: int):
    from threert_b200 import Gpu, crowd, prep
    c = crowd.crowd(n=5000, groups=groups)
    P = prep.prepare(c.desc)
    corners, jobs = crowd.deform_jobs(P, c)
    g = Gpu(0)
    S = g.upload(P)
    S.deform_setup(corners, jobs)
    t_inst, _ = crowd.records(P)
    for f in range(3):
        t = f / crowd.FPS
        S.update(3, t_inst * 16, crowd.frame_records(P, c, t))
        S.deform(P.params, crowd.palettes(t, c.phase, c.scale))
    S.close()
    g.close()


def sky_case():
    import math
    from threert_b200 import Gpu, prep, scenes
    from threert_b200 import _native as N
    g = Gpu(0)
    P = prep.prepare(scenes.city(n_objects=60, width=64, height=36, n_emitters=20, sky_size=(1024, 512)))
    atm, sun_light = P.sky_pending
    for k in range(3):
        e, a = math.radians(28.0 + 0.25 * k), math.radians(35.0)
        atm.sun_dir = (N.f32 * 3)(math.cos(e) * math.cos(a), math.sin(e), math.cos(e) * math.sin(a))
        g.bake_sky(atm)
    S = g.upload(P)
    S.set_sky(atm, sun_light, P.info["env_nee_floor"], P.params.copy())
    g.synchronize()
    S.close()
    g.close()


def emitters_case():
    from threert_b200 import Gpu, prep, scenes
    P = prep.prepare(scenes.city())
    g = Gpu(0)
    S = g.upload(P)
    for _ in range(3):
        S.weigh_emitters(P.params, P.info["light_tree_nodes"])
    g.synchronize()
    S.close()
    g.close()


def cornell_case():
    from threert_b200 import Gpu, prep, scenes
    P = prep.prepare(scenes.cornell(256, 256))
    g = Gpu(0)
    S = g.upload(P)
    for k in range(3):
        S.render_raw(prep.params_with(P.params, seed=k + 1), 16, read=False, stats=False)
    g.synchronize()
    S.close()
    g.close()


if __name__ == "__main__":
    case = sys.argv[1] if len(sys.argv) > 1 else "city"
    if case == "city":
        city()
    elif case == "city_wide":
        from threert_b200 import _native as N
        city(N.TRT_RENDER_WIDE)
    elif case == "unet":
        unet_case()
    elif case == "crowd":
        crowd_case(int(sys.argv[2]) if len(sys.argv) > 2 else 1)
    elif case == "sky":
        sky_case()
    elif case == "emitters":
        emitters_case()
    elif case == "cornell":
        cornell_case()
    else:
        raise SystemExit(f"unknown case {case}")
