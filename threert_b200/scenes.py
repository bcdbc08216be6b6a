"""Seeded synthetic scenes: the Cornell box (config 0), the procedural city (config 1), and the analytic known-answer
scenes of the reference's render tests (tests/render/*.ts), as `SceneDescription`s for `prep.prepare`.

No dataset is involved: every scene is generated from its seed. Mesh helpers build model-space triangles with corner
normals the way three.js geometries do (planes, boxes, UV spheres).
"""
from __future__ import annotations

import math

import numpy as np

from .prep import (Camera, DirLight, Instance, Material, Mesh, Preset, SceneDescription, Sky, lambert)

# ---- geometry ---------------------------------------------------------------------------------------------------


def quad(corners, normal=None) -> tuple[np.ndarray, np.ndarray]:
    """Two triangles over four corners (counter-clockwise seen from the normal's side)."""
    c = np.asarray(corners, np.float64)
    tris = np.stack([c[[0, 1, 2]], c[[0, 2, 3]]])
    n = np.cross(c[1] - c[0], c[2] - c[0]) if normal is None else np.asarray(normal, np.float64)
    n = n / np.linalg.norm(n)
    return tris.astype(np.float32), np.broadcast_to(n, tris.shape).astype(np.float32).copy()


def plane_mesh(size: float, segments: int = 1, y: float = 0.0) -> Mesh:
    """A plane in x-z facing +y (three.js PlaneGeometry rotated -90 degrees about x)."""
    h = size * 0.5
    xs = np.linspace(-h, h, segments + 1)
    tris, nrm = [], []
    for i in range(segments):
        for j in range(segments):
            x0, x1, z0, z1 = xs[i], xs[i + 1], xs[j], xs[j + 1]
            t, n = quad([(x0, y, z1), (x1, y, z1), (x1, y, z0), (x0, y, z0)], (0, 1, 0))
            tris.append(t)
            nrm.append(n)
    return Mesh(np.concatenate(tris), np.concatenate(nrm))


def box_mesh(sx: float, sy: float, sz: float, segments: int = 1) -> Mesh:
    """A box centred on the origin, each face split into segments x segments quads, outward normals."""
    tris, nrm = [], []
    hx, hy, hz = sx / 2, sy / 2, sz / 2
    faces = [  # (normal, u axis, v axis, half extents along n, u, v)
        ((1, 0, 0), (0, 0, -1), (0, 1, 0), hx, hz, hy), ((-1, 0, 0), (0, 0, 1), (0, 1, 0), hx, hz, hy),
        ((0, 1, 0), (1, 0, 0), (0, 0, -1), hy, hx, hz), ((0, -1, 0), (1, 0, 0), (0, 0, 1), hy, hx, hz),
        ((0, 0, 1), (1, 0, 0), (0, 1, 0), hz, hx, hy), ((0, 0, -1), (-1, 0, 0), (0, 1, 0), hz, hx, hy)]
    for n, u, v, hn, hu, hv in faces:
        n, u, v = np.array(n, float), np.array(u, float), np.array(v, float)
        s = np.linspace(-1.0, 1.0, segments + 1)
        for i in range(segments):
            for j in range(segments):
                cs = [n * hn + u * hu * a + v * hv * b for a, b in
                      ((s[i], s[j]), (s[i + 1], s[j]), (s[i + 1], s[j + 1]), (s[i], s[j + 1]))]
                t, nn = quad(cs, n)
                tris.append(t)
                nrm.append(nn)
    return Mesh(np.concatenate(tris), np.concatenate(nrm))


def sphere_mesh(radius: float, slices: int, stacks: int) -> Mesh:
    """A UV sphere (three.js SphereGeometry's layout: `slices` around, `stacks` pole to pole) with smooth normals."""
    th = np.linspace(0.0, math.pi, stacks + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, slices + 1)
    P = np.stack([-np.cos(ph)[None, :] * np.sin(th)[:, None], np.cos(th)[:, None] * np.ones_like(ph)[None, :],
                  np.sin(ph)[None, :] * np.sin(th)[:, None]], -1)
    tris, nrm = [], []
    for i in range(stacks):
        for j in range(slices):
            a, b, c, d = P[i, j], P[i + 1, j], P[i + 1, j + 1], P[i, j + 1]
            if i != 0:
                tris.append([a, b, d])
            if i != stacks - 1:
                tris.append([b, c, d])
    n = np.asarray(tris, np.float64)
    return Mesh((n * radius).astype(np.float32), n.astype(np.float32))


def translate_rot_y(t, angle: float = 0.0, scale=1.0) -> np.ndarray:
    """A 3x4 world matrix: rotation about y, then translation."""
    c, s = math.cos(angle), math.sin(angle)
    sc = np.broadcast_to(np.asarray(scale, float), (3,))
    m = np.array([[c * sc[0], 0, s * sc[2], t[0]], [0, sc[1], 0, t[1]], [-s * sc[0], 0, c * sc[2], t[2]]], np.float32)
    return m


def rot_x(angle: float, t=(0, 0, 0)) -> np.ndarray:
    c, s = math.cos(angle), math.sin(angle)
    return np.array([[1, 0, 0, t[0]], [0, c, -s, t[1]], [0, s, c, t[2]]], np.float32)


def srgb_to_linear(c):
    c = np.asarray(c, np.float64)
    return np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)


# ---- config 0: the Cornell box ----------------------------------------------------------------------------------


def cornell(width: int = 256, height: int = 256, max_depth: int = 5, seed: int = 0x5EED) -> SceneDescription:
    """36 triangles: five walls (white 0.73, red (0.65, 0.05, 0.05), green (0.12, 0.45, 0.15)), a 0.13 x 0.105 ceiling
    light of radiance (17, 12, 4), a short box 0.6 high and a tall box 1.2 high rotated by -18 and +18 degrees; all
    Lambertian; black sky; the camera of scenes/cornell-box.ts."""
    white, red, green = lambert(0.73), lambert((0.65, 0.05, 0.05)), lambert((0.12, 0.45, 0.15))
    light = Material(base=(0.0, 0.0, 0.0), emissive=(17.0, 12.0, 4.0), roughness=1.0, metallic=0.0, specular=0.0,
                     card=True)
    materials = [white, red, green, light]
    meshes, instances = [], []

    def add(mesh, mat, world=None):
        meshes.append(mesh)
        instances.append(Instance(len(meshes) - 1, [mat], world if world is not None else translate_rot_y((0, 0, 0)),
                                  object=len(instances)))

    def wall(corners, normal, mat):
        t, n = quad(corners, normal)
        add(Mesh(t, n), mat)

    wall([(-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1)], (0, 1, 0), 0)       # floor
    wall([(-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)], (0, -1, 0), 0)      # ceiling
    wall([(-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)], (0, 0, 1), 0)     # back
    wall([(-1, 0, 1), (-1, 0, -1), (-1, 2, -1), (-1, 2, 1)], (1, 0, 0), 1)     # left, red
    wall([(1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)], (-1, 0, 0), 2)        # right, green
    lx, lz, ly = 0.13 / 2, 0.105 / 2, 1.995
    wall([(-lx, ly, -lz), (lx, ly, -lz), (lx, ly, lz), (-lx, ly, lz)], (0, -1, 0), 3)  # the light, facing down
    add(box_mesh(0.6, 1.2, 0.6), 0, translate_rot_y((-0.33, 0.6, -0.28), math.radians(18.0)))
    add(box_mesh(0.6, 0.6, 0.6), 0, translate_rot_y((0.35, 0.3, 0.32), math.radians(-18.0)))
    cam = Camera.look_at((0.0, 1.0, 3.9), (0.0, 1.0, 0.0), 39.0, width, height)
    return SceneDescription(meshes, materials, instances, cam, sky=Sky("none"),
                            preset=Preset(max_bounces=max_depth, rr_depth=3, clamp_indirect=1.0e9), seed=seed)


# ---- config 1: the procedural city ------------------------------------------------------------------------------


def catmull_rom(points: np.ndarray, t: float) -> np.ndarray:
    """A closed Catmull-Rom spline through `points` at t in [0, 1)."""
    n = len(points)
    x = (t % 1.0) * n
    i = int(math.floor(x))
    u = x - i
    p0, p1, p2, p3 = (points[(i - 1) % n], points[i % n], points[(i + 1) % n], points[(i + 2) % n])
    return 0.5 * ((2 * p1) + (-p0 + p2) * u + (2 * p0 - 5 * p1 + 4 * p2 - p3) * u * u + (-p0 + 3 * p1 - 3 * p2 + p3) * u ** 3)


def city_camera_path(seed: int, extent: float = 500.0, keys: int = 12) -> np.ndarray:
    """Key points of the camera's loop over the city: 0.25 to 0.75 of the way out, 3 to 9 % of the extent up."""
    rng = np.random.default_rng(seed ^ 0xC0FFEE)
    ang = np.sort(rng.uniform(0, 2 * math.pi, keys))
    rad = rng.uniform(0.25, 0.75, keys) * extent
    hgt = rng.uniform(0.03, 0.09, keys) * extent
    return np.stack([np.cos(ang) * rad, hgt, np.sin(ang) * rad], -1)


def city_camera(frame: int, frames: int, seed: int, width: int, height: int, extent: float = 500.0) -> Camera:
    pts = city_camera_path(seed, extent)
    t = frame / frames
    p = catmull_rom(pts, t)
    q = catmull_rom(pts, t + 0.5 / frames)
    look = q + (q - p) / max(np.linalg.norm(q - p), 1e-6) * (0.1 * extent)
    look[1] = p[1] - 0.024 * extent
    return Camera.look_at(tuple(p), tuple(look), 60.0, width, height)


def city(n_objects: int = 4000, width: int = 1280, height: int = 720, max_depth: int = 4, seed: int = 1,
         extent: float = 500.0, n_emitters: int = 200, box_segments: int = 4, sphere_slices: int = 20,
         sphere_stacks: int = 21, frame: int = 0, frames: int = 240, sky_size=(1024, 512),
         sky: str = "atmosphere", emitter_offset=(0.0, 0.0, 0.0)) -> SceneDescription:
    """Config 1: `n_objects` seeded boxes (faces split 4 x 4: 192 triangles) and UV spheres (20 x 21: 800 triangles),
    half each, on a 1 km grid: 1,984,000 triangles at 4,000, one mesh and one unit each. GGX materials with roughness
    U(0.05, 1), metallic Bernoulli(0.3) and base colour uniform in sRGB. 200 emissive quads (400 triangles, a light
    tree) of log-uniform 10-1000 nits, a 90,000-lux sun at 28 degrees elevation, and the sky: the physical atmosphere
    lit by that sun (sky.rs:643 bake_atmosphere, baked on the device at 1024 x 512; its sun light tinted by the
    atmosphere's transmittance), or with sky="gradient" a gradient sky (sky.rs:941) that the host prep bakes.
    emitter_offset moves every emissive quad (the same quads elsewhere: scenes whose emitters moved)."""
    rng = np.random.default_rng(seed)
    meshes, materials, instances = [], [], []
    side = int(math.ceil(math.sqrt(n_objects)))
    cell = 2.0 * extent / side
    order = rng.permutation(side * side)[:n_objects]
    for k, c in enumerate(order):
        gx, gz = c % side, c // side
        x = -extent + (gx + 0.5) * cell + rng.uniform(-0.2, 0.2) * cell
        z = -extent + (gz + 0.5) * cell + rng.uniform(-0.2, 0.2) * cell
        base = tuple(srgb_to_linear(rng.uniform(0.0, 1.0, 3)))
        mat = Material(base=base, roughness=float(rng.uniform(0.05, 1.0)), metallic=float(rng.random() < 0.3),
                       specular=0.5)
        materials.append(mat)
        if k % 2 == 0:
            fx, fz = rng.uniform(0.3, 0.8, 2) * cell
            hy = float(np.exp(rng.uniform(math.log(5.0), math.log(60.0))))
            meshes.append(box_mesh(fx, hy, fz, box_segments))
            world = translate_rot_y((x, hy / 2, z), rng.uniform(0, math.pi))
        else:
            r = rng.uniform(0.15, 0.45) * cell
            meshes.append(sphere_mesh(r, sphere_slices, sphere_stacks))
            world = translate_rot_y((x, r * rng.uniform(0.6, 1.4), z))
        instances.append(Instance(len(meshes) - 1, [len(materials) - 1], world, object=k))
    # The ground.
    materials.append(Material(base=(0.18, 0.18, 0.18), roughness=0.8, specular=0.5))
    meshes.append(plane_mesh(2.4 * extent))
    instances.append(Instance(len(meshes) - 1, [len(materials) - 1], object=n_objects))
    # Emissive quads: one mesh, a section (and an emissive material) each.
    if n_emitters:
        tris, nrm, sec = [], [], []
        first_mat = len(materials)
        for e in range(n_emitters):
            w_, h_ = rng.uniform(2.0, 6.0), rng.uniform(1.0, 3.0)
            cx, cz = rng.uniform(-extent, extent, 2)
            cy = rng.uniform(3.0, 20.0)
            a = rng.uniform(0, 2 * math.pi)
            u = np.array([math.cos(a), 0.0, math.sin(a)]) * w_ / 2
            v = np.array([0.0, h_ / 2, 0.0])
            c = np.array([cx, cy, cz]) + np.asarray(emitter_offset, np.float64)
            t, n = quad([c - u - v, c + u - v, c + u + v, c - u + v])
            tris.append(t)
            nrm.append(n)
            sec += [e, e]
            nits = float(np.exp(rng.uniform(math.log(10.0), math.log(1000.0))))
            tint = srgb_to_linear(rng.uniform(0.6, 1.0, 3))
            tint = tint / (0.2126 * tint[0] + 0.7152 * tint[1] + 0.0722 * tint[2])
            materials.append(Material(base=(0.05, 0.05, 0.05), emissive=tuple(tint * nits), roughness=0.5,
                                      specular=0.5))
        meshes.append(Mesh(np.concatenate(tris), np.concatenate(nrm), sections=np.asarray(sec, np.uint32),
                           n_sections=n_emitters))
        instances.append(Instance(len(meshes) - 1, list(range(first_mat, first_mat + n_emitters)), object=n_objects + 1))
    el, az = math.radians(28.0), math.radians(35.0)
    to_sun = (math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az))
    if sky == "atmosphere":
        sun = DirLight(direction=tuple(-np.asarray(to_sun)), color=(1.0, 1.0, 1.0), intensity=90000.0)
        sky_desc = Sky("atmosphere", sun_light=0, width=sky_size[0], height=sky_size[1])
    else:
        sun = DirLight(direction=tuple(-np.asarray(to_sun)), color=(1.0, 0.96, 0.9), intensity=90000.0)
        sky_desc = Sky("gradient", zenith=(1200.0, 2000.0, 4000.0), horizon=(5250.0, 5950.0, 7000.0),
                       ground=(600.0, 600.0, 600.0), width=sky_size[0], height=sky_size[1])
    cam = city_camera(frame, frames, seed, width, height, extent)
    return SceneDescription(meshes, materials, instances, cam, lights=[sun], sky=sky_desc,
                            preset=Preset(max_bounces=max_depth, rr_depth=3, clamp_indirect=1.0e9), seed=0x5EED)


# ---- the reference's analytic render tests (tests/render/*.ts: 160 x 90, 64 spp, cinematic, no compensation) ------

TEST_SIZE = (160, 90)
CENTER = (0.45, 0.45, 0.55, 0.55)


def _test_camera(position, target, fov=30.0, size=TEST_SIZE):
    return Camera.look_at(position, target, fov, size[0], size[1])


def _test_preset(energy=0.0):
    # presets/cinematic.json "native": maxBounces 8, russianRouletteDepth 3; tests run with clamps as the preset's
    # (the analytic scenes have no indirect light the clamp reaches), energyCompensation as the test says.
    return Preset(max_bounces=8, rr_depth=3, clamp_indirect=1.0e9, energy_compensation=energy)


def furnace_diffuse(size=TEST_SIZE) -> tuple[SceneDescription, float]:
    """tests/render/furnace-diffuse.ts: an albedo-1 Lambert sphere in a uniform 1-nit sky reads 1 (+-2 %)."""
    m = sphere_mesh(0.5, 64, 48)
    d = SceneDescription([m], [lambert(1.0)], [Instance(0, [0])], _test_camera((0, 0, 3), (0, 0, 0), size=size),
                         sky=Sky("color", color=(1.0, 1.0, 1.0)), preset=_test_preset())
    return d, 1.0


def directional_lambert(size=TEST_SIZE) -> tuple[SceneDescription, float]:
    """tests/render/light-directional-lambert.ts: 10,000 lux at 60 degrees on albedo 0.5: 0.5 E sin60 / pi (+-2 %)."""
    pos = np.array([0.0, math.sin(math.pi / 3), math.cos(math.pi / 3)])
    sun = DirLight(direction=tuple(-pos / np.linalg.norm(pos)), intensity=10000.0)
    d = SceneDescription([plane_mesh(20.0)], [lambert(0.5)], [Instance(0, [0])],
                         _test_camera((2, 2, 0), (0, 0, 0), size=size), lights=[sun], sky=Sky("none"),
                         preset=_test_preset())
    return d, 0.5 * 10000.0 * math.sin(math.pi / 3) / math.pi


def emissive_nits(size=TEST_SIZE) -> tuple[SceneDescription, float]:
    """tests/render/material-emissive-nits.ts: a 500-nit emissive plane shows 500 (+-1 %)."""
    t, n = quad([(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)], (0, 0, 1))
    mat = Material(base=(0, 0, 0), emissive=(500.0, 500.0, 500.0), roughness=1.0, specular=0.5)
    d = SceneDescription([Mesh(t, n)], [mat], [Instance(0, [0])], _test_camera((0, 0, 3), (0, 0, 0), size=size),
                         sky=Sky("none"), preset=_test_preset())
    return d, 500.0


def metal_f0(size=TEST_SIZE) -> tuple[SceneDescription, tuple]:
    """tests/render/material-metal-f0.ts: a smooth metal plane under a 1-nit sky shows its F0 (0.9, 0.5, 0.2) (+-3 %)."""
    mat = Material(base=(0.9, 0.5, 0.2), metallic=1.0, roughness=0.0, specular=0.5)
    d = SceneDescription([plane_mesh(50.0)], [mat], [Instance(0, [0])],
                         _test_camera((0, 3, 0.001), (0, 0, 0), 20.0, size=size), sky=Sky("color", color=(1.0, 1.0, 1.0)),
                         preset=_test_preset())
    return d, (0.9, 0.5, 0.2)


def emitter_grid(n=12, step=0.5, height=2.0, side=0.05, nits=20000.0, size=TEST_SIZE) -> tuple[SceneDescription, float]:
    """tests/render/light-emitter-tree.ts (and light-emitter-far.ts with step 2, height 150, side 1, 10,000 nits):
    n x n emissive squares facing down over an albedo-0.5 plane, a light tree past 256 triangles; the centre reads
    0.5 / pi x the sum of L A cos^2 / d^2 (+-2 %)."""
    at = lambda k: (k - (n - 1) / 2) * step
    cells = [(at(k % n), at(k // n)) for k in range(n * n)]
    expected = (0.5 / math.pi) * nits * side * side * sum(height * height / (x * x + z * z + height * height) ** 2
                                                          for x, z in cells)
    s = side / 2
    t, nn = quad([(-s, 0, -s), (s, 0, -s), (s, 0, s), (-s, 0, s)], (0, -1, 0))
    glow = Material(base=(0, 0, 0), emissive=(nits, nits, nits), roughness=1.0, specular=0.5)
    meshes = [plane_mesh(400.0), Mesh(t, nn)]
    insts = [Instance(0, [0], object=0)]
    for k, (x, z) in enumerate(cells):
        insts.append(Instance(1, [1], translate_rot_y((x, height, z)), object=1 + k))
    d = SceneDescription(meshes, [lambert(0.5), glow], insts, _test_camera((0, 0.5, 0.001), (0, 0, 0), 40.0, size=size),
                         sky=Sky("none"), preset=_test_preset())
    return d, expected


def shadow_directional(size=TEST_SIZE):
    """tests/render/shadow-directional.ts: under an overhead sun a black occluder's shadow reads 0 against the lit
    ground (ratio 0 +- 0.005). Returns the regions a (shadow) and b (lit)."""
    sun = DirLight(direction=(0.0, -1.0, 0.0), intensity=10000.0)
    box = box_mesh(2.0, 0.2, 2.0)
    d = SceneDescription([box, plane_mesh(40.0)], [lambert(0.0), lambert(0.5)],
                         [Instance(0, [0], translate_rot_y((0, 1.5, 0)), object=0), Instance(1, [1], object=1)],
                         _test_camera((4, 2.2, 0.001), (0, 0, 0), 30.0, size=size), lights=[sun], sky=Sky("none"),
                         preset=_test_preset())
    return d, (0.47, 0.47, 0.53, 0.53), (0.02, 0.85, 0.12, 0.95)


def furnace_metal(size=TEST_SIZE) -> tuple[SceneDescription, float]:
    """tests/render/furnace-metal.ts: an F0 = 1, roughness 0.5 metal sphere in a 1-nit sky with energy
    compensation 1 reads 1 (+-3 %)."""
    mat = Material(base=(1.0, 1.0, 1.0), metallic=1.0, roughness=0.5, specular=0.5)
    d = SceneDescription([sphere_mesh(0.5, 64, 48)], [mat], [Instance(0, [0])],
                         _test_camera((0, 0, 3), (0, 0, 0), size=size), sky=Sky("color", color=(1.0, 1.0, 1.0)),
                         preset=_test_preset(energy=1.0))
    return d, 1.0


def region_pixels(width: int, height: int, region) -> np.ndarray:
    """Pixel indices of a region [u0, v0, u1, v1] (0..1, v down), as the render tests' metrics read them."""
    u0, v0, u1, v1 = region
    x0, x1 = int(math.floor(u0 * width)), int(math.ceil(u1 * width))
    y0, y1 = int(math.floor(v0 * height)), int(math.ceil(v1 * height))
    xs, ys = np.meshgrid(np.arange(x0, x1), np.arange(y0, y1))
    return (ys * width + xs).ravel().astype(np.uint32)
