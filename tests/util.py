"""Shared helpers of the tests: scenes with rotated, scaled and shifted units; random rays; region metrics."""
import math

import numpy as np

from threert_b200 import prep, scenes
from threert_b200.gpu import RAY_DTYPE, frame_of


def luma(c):
    c = np.asarray(c)
    return 0.2126 * c[..., 0] + 0.7152 * c[..., 1] + 0.0722 * c[..., 2]


def small_city(seed=3, n_objects=80, width=64, height=36, n_emitters=140, max_depth=4, sky="gradient",
               emitter_offset=(0.0, 0.0, 0.0)):
    """A city small enough for the oracle: boxes turned about y (units with normal rows), spheres placed by a
    translation alone (UNIT_SHIFTED), a ground, emissive quads past the light tree's 256 triangles."""
    return scenes.city(n_objects=n_objects, width=width, height=height, seed=seed, extent=60.0, n_emitters=n_emitters,
                       box_segments=2, sphere_slices=10, sphere_stacks=8, max_depth=max_depth, sky_size=(64, 32),
                       sky=sky, emitter_offset=emitter_offset)


def scaled_units_scene():
    """Units placed by rotation, non-uniform scale, and a mirror (a negative determinant), and one by translation."""
    meshes = [scenes.box_mesh(1, 1, 1, 2), scenes.sphere_mesh(0.5, 12, 8)]
    mats = [prep.lambert(0.6), prep.Material(base=(0.9, 0.6, 0.3), metallic=1.0, roughness=0.3)]
    inst = []
    rng = np.random.default_rng(4)
    for k in range(24):
        a = rng.uniform(0, 2 * math.pi)
        s = rng.uniform(0.5, 2.0, 3)
        if k % 5 == 0:
            s[0] = -s[0]
        w = scenes.translate_rot_y(rng.uniform(-6, 6, 3), a, s)
        if k % 3 == 0:
            w = scenes.translate_rot_y(rng.uniform(-6, 6, 3))
        inst.append(prep.Instance(k % 2, [k % 2], w, object=k))
    cam = prep.Camera.look_at((0, 4, 14), (0, 0, 0), 50, 48, 32)
    sun = prep.DirLight(direction=(-0.3, -1.0, -0.2), intensity=5000.0)
    return prep.SceneDescription(meshes, mats, inst, cam, lights=[sun], sky=prep.Sky("color", color=(200.0, 300.0, 500.0)),
                                 preset=prep.Preset(max_bounces=4))


def random_rays(P, n, seed=0, modes=(0, 1, 2), spread=1.0):
    """Rays from around the scene's camera and from inside its bounds, every mode, some with a short tmax."""
    rng = np.random.default_rng(seed)
    nodes = P.nodes.view(np.float32).reshape(-1, 8)
    top = int(P.params[70])
    lo, hi = nodes[top, 0:3], nodes[top, 4:7]
    cam = P.params[0:3].view(np.float32)
    r = np.zeros(n, RAY_DTYPE)
    k = n // 2
    r["o"][:k] = cam + rng.normal(0, spread, (k, 3))
    r["o"][k:] = lo + (hi - lo) * rng.random((n - k, 3))
    d = rng.normal(0, 1, (n, 3))
    # Half the rays aimed at points inside the scene's bounds, half in any direction.
    aim = rng.random(n) < 0.5
    d[aim] = lo + (hi - lo) * rng.random((aim.sum(), 3)) - r["o"][aim]
    r["d"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r["tmax"] = np.where(rng.random(n) < 0.2, rng.uniform(0.1, 50.0, n), 3.0e38).astype(np.float32)
    r["mode"] = rng.choice(modes, n)
    return r


def region_mean(acc, w, h, spp, region):
    f = frame_of(acc, w, h, spp)
    px = scenes.region_pixels(w, h, region)
    return f.color.reshape(-1, 3)[px].mean(0)


def small_crowd(n=160, groups=3, width=64, height=36, max_depth=3, sky="gradient"):
    """Config 2 small enough for the oracle: a lighter humanoid (30 capsules of 8 x 9 quads), n walkers in `groups`
    pose groups, a small ground, 12 lamps."""
    from threert_b200 import crowd
    body = crowd.humanoid(segments=8, hemi_rings=3, body_rings=4)
    return crowd.crowd(n=n, groups=groups, width=width, height=height, max_depth=max_depth, extent=12.0,
                       ground_segments=12, n_emitters=12, body=body, sky_size=(64, 32), sky=sky)
