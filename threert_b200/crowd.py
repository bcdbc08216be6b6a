"""Config 2, the instanced dynamic crowd: a procedural humanoid (capsules joined into one mesh, 30 bones, two bone
weights a vertex), placed `n` times on a 50k-triangle ground, walking, in K pose groups (K skinned copies of the
mesh, instance i posed by group i % K), under config 1's lights. Each frame the host computes the groups' palettes
(forward kinematics of seeded sinusoidal joint angles) and the instances' records; the device skins, gathers the
leaves, refits the K mesh trees and builds the top tree again (trt_deform), then renders.

Everything is generated from a seed; no asset is read.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import prep
from .prep import Camera, DirLight, Instance, Material, Mesh, Preset, SceneDescription, Sky
from .scenes import plane_mesh, quad, srgb_to_linear

# The skeleton: (parent, head in the rest pose, direction, length, radius). Bind pose: every bone unrotated at its
# head, so a bone's inverse bind matrix is a translation by minus its head.
_UP, _DOWN, _FWD = (0.0, 1.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.0, 1.0)
BONES = [
    (-1, (0.0, 0.95, 0.0), _UP, 0.12, 0.14),       # 0 pelvis
    (0, (0.0, 1.05, 0.0), _UP, 0.15, 0.13),        # 1 spine
    (1, (0.0, 1.20, 0.0), _UP, 0.15, 0.14),        # 2 spine
    (2, (0.0, 1.35, 0.0), _UP, 0.12, 0.15),        # 3 chest
    (3, (0.0, 1.50, 0.0), _UP, 0.08, 0.05),        # 4 neck
    (4, (0.0, 1.62, 0.0), _UP, 0.14, 0.10),        # 5 head
    (3, (0.05, 1.45, 0.0), (1.0, 0.0, 0.0), 0.13, 0.05),   # 6 clavicle L
    (6, (0.20, 1.45, 0.0), _DOWN, 0.27, 0.05),     # 7 upper arm L
    (7, (0.20, 1.16, 0.0), _DOWN, 0.24, 0.04),     # 8 forearm L
    (8, (0.20, 0.90, 0.0), _DOWN, 0.07, 0.035),    # 9 hand L
    (9, (0.20, 0.81, 0.0), _DOWN, 0.05, 0.02),     # 10 fingers L
    (3, (-0.05, 1.45, 0.0), (-1.0, 0.0, 0.0), 0.13, 0.05),  # 11 clavicle R
    (11, (-0.20, 1.45, 0.0), _DOWN, 0.27, 0.05),   # 12 upper arm R
    (12, (-0.20, 1.16, 0.0), _DOWN, 0.24, 0.04),   # 13 forearm R
    (13, (-0.20, 0.90, 0.0), _DOWN, 0.07, 0.035),  # 14 hand R
    (14, (-0.20, 0.81, 0.0), _DOWN, 0.05, 0.02),   # 15 fingers R
    (0, (0.09, 0.92, 0.0), _DOWN, 0.03, 0.07),     # 16 hip L
    (16, (0.09, 0.87, 0.0), _DOWN, 0.40, 0.075),   # 17 thigh L
    (17, (0.09, 0.46, 0.0), _DOWN, 0.37, 0.055),   # 18 shin L
    (18, (0.09, 0.06, 0.0), _FWD, 0.14, 0.04),     # 19 foot L
    (19, (0.09, 0.05, 0.16), _FWD, 0.04, 0.03),    # 20 toe L
    (0, (-0.09, 0.92, 0.0), _DOWN, 0.03, 0.07),    # 21 hip R
    (21, (-0.09, 0.87, 0.0), _DOWN, 0.40, 0.075),  # 22 thigh R
    (22, (-0.09, 0.46, 0.0), _DOWN, 0.37, 0.055),  # 23 shin R
    (23, (-0.09, 0.06, 0.0), _FWD, 0.14, 0.04),    # 24 foot R
    (24, (-0.09, 0.05, 0.16), _FWD, 0.04, 0.03),   # 25 toe R
    (9, (0.23, 0.88, 0.03), (0.3, -0.8, 0.5), 0.05, 0.015),   # 26 thumb L
    (14, (-0.23, 0.88, 0.03), (-0.3, -0.8, 0.5), 0.05, 0.015),  # 27 thumb R
    (5, (0.0, 1.63, 0.06), (0.0, -0.3, 1.0), 0.06, 0.04),     # 28 jaw
    (5, (0.0, 1.74, -0.08), (0.0, -0.6, -0.8), 0.14, 0.03),   # 29 hair
]
N_BONES = len(BONES)
PARENTS = np.array([b[0] for b in BONES])
HEADS = np.array([b[1] for b in BONES], np.float64)

# The walk cycle: per bone, amplitudes (radians) of its rotation about x and z and the phase shift of each.
_WALK = np.zeros((N_BONES, 4))
for _b, (_ax, _az, _px, _pz) in {
        0: (0.04, 0.05, 2.0, 0.0), 1: (0.04, 0.06, 0.0, 1.0), 2: (0.03, 0.05, 0.0, 1.0), 3: (0.03, 0.04, 0.0, 1.0),
        5: (0.10, 0.05, 2.0, 0.5), 7: (0.45, 0.08, math.pi, 0.0), 8: (0.30, 0.0, math.pi - 0.6, 0.0),
        12: (0.45, 0.08, 0.0, 0.0), 13: (0.30, 0.0, -0.6, 0.0), 17: (0.55, 0.04, 0.0, 0.0),
        18: (0.45, 0.0, -1.4, 0.0), 19: (0.25, 0.0, -0.8, 0.0), 22: (0.55, 0.04, math.pi, 0.0),
        23: (0.45, 0.0, math.pi - 1.4, 0.0), 24: (0.25, 0.0, math.pi - 0.8, 0.0), 28: (0.12, 0.0, 0.0, 0.0),
        29: (0.20, 0.15, 1.0, 2.0)}.items():
    _WALK[_b] = (_ax, _az, _px, _pz)


@dataclass
class Humanoid:
    mesh: Mesh
    positions: np.ndarray   # (V, 3) rest-pose model vertices
    normals: np.ndarray     # (V, 3)
    bones: np.ndarray       # (V, 2) palette indices
    weights: np.ndarray     # (V, 2)


def _basis(a):
    a = np.asarray(a, np.float64)
    a = a / np.linalg.norm(a)
    t = np.array([1.0, 0.0, 0.0]) if abs(a[0]) < 0.9 else np.array([0.0, 0.0, 1.0])
    u = np.cross(a, t)
    u /= np.linalg.norm(u)
    return a, u, np.cross(a, u)


def humanoid(segments: int = 16, hemi_rings: int = 5, body_rings: int = 12) -> Humanoid:
    """Capsules along the bones, joined into one mesh: 30 x 2 x segments x (2 x hemi_rings + body_rings - 1)
    triangles (16, 5, 12: 20,160). A vertex hangs on its bone and, near the bone's head, partly on the parent."""
    pos, nrm, bones, weights, tris = [], [], [], [], []
    for b, (parent, head, direction, length, radius) in enumerate(BONES):
        a, u, v = _basis(direction)
        head = np.asarray(head, np.float64)
        # The profile from pole to pole: (axial position, radial distance, axial normal, radial normal).
        prof = [(-radius, 0.0, -1.0, 0.0)]
        for j in range(1, hemi_rings + 1):
            phi = 0.5 * math.pi * j / hemi_rings
            prof.append((-radius * math.cos(phi), radius * math.sin(phi), -math.cos(phi), math.sin(phi)))
        for j in range(1, body_rings):
            prof.append((length * j / body_rings, radius, 0.0, 1.0))
        for j in range(hemi_rings, 0, -1):
            phi = 0.5 * math.pi * j / hemi_rings
            prof.append((length + radius * math.cos(phi), radius * math.sin(phi), math.cos(phi), math.sin(phi)))
        prof.append((length + radius, 0.0, 1.0, 0.0))
        ring_ids = []
        for k, (ax, rad, na, nr) in enumerate(prof):
            n_around = 1 if rad == 0.0 else segments
            ids = []
            for s in range(n_around):
                th = 2.0 * math.pi * s / segments
                radial = u * math.cos(th) + v * math.sin(th)
                pos.append(head + a * ax + radial * rad)
                nn = a * na + radial * nr
                nrm.append(nn / np.linalg.norm(nn))
                w_parent = 0.0 if parent < 0 else min(max(0.5 - ax / (0.5 * length), 0.0), 0.5)
                bones.append((b, max(parent, 0)))
                weights.append((1.0 - w_parent, w_parent))
                ids.append(len(pos) - 1)
            ring_ids.append(ids)
        for k in range(len(prof) - 1):
            r0, r1 = ring_ids[k], ring_ids[k + 1]
            for s in range(segments):
                s1 = (s + 1) % segments
                if len(r0) == 1:
                    tris.append((r0[0], r1[s1], r1[s]))
                elif len(r1) == 1:
                    tris.append((r0[s], r0[s1], r1[0]))
                else:
                    tris.append((r0[s], r0[s1], r1[s1]))
                    tris.append((r0[s], r1[s1], r1[s]))
    P = np.asarray(pos, np.float32)
    Nn = np.asarray(nrm, np.float32)
    T = np.asarray(tris, np.int64)
    mesh = Mesh(P[T], Nn[T])
    return Humanoid(mesh, P, Nn, np.asarray(bones, np.uint32), np.asarray(weights, np.float32))


def _rot_x(a):
    c, s = np.cos(a), np.sin(a)
    R = np.zeros(a.shape + (3, 3))
    R[..., 0, 0] = 1.0
    R[..., 1, 1], R[..., 1, 2], R[..., 2, 1], R[..., 2, 2] = c, -s, s, c
    return R


def _rot_z(a):
    c, s = np.cos(a), np.sin(a)
    R = np.zeros(a.shape + (3, 3))
    R[..., 2, 2] = 1.0
    R[..., 0, 0], R[..., 0, 1], R[..., 1, 0], R[..., 1, 1] = c, -s, s, c
    return R


def group_params(k: int, seed: int = 7) -> tuple[np.ndarray, np.ndarray]:
    """Each pose group's seeded phase and per-bone amplitude scale."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 2.0 * math.pi, k), rng.uniform(0.8, 1.2, (k, N_BONES))


def palettes(t: float, phase: np.ndarray, scale: np.ndarray, freq: float = 0.9) -> np.ndarray:
    """The K groups' palettes at time t: (K, 30, 3, 4) float32, bone world matrix times inverse bind (skin.rs
    PaletteRows: three rows a matrix). Joint angles: amplitude x sin(2 pi f t + group phase + bone shift)."""
    k = len(phase)
    ang = 2.0 * math.pi * freq * t + phase[:, None]
    rx = _WALK[None, :, 0] * scale * np.sin(ang + _WALK[None, :, 2])
    rz = _WALK[None, :, 1] * scale * np.sin(ang + _WALK[None, :, 3])
    local = _rot_x(rx) @ _rot_z(rz)                      # (K, 30, 3, 3)
    wr = np.zeros((k, N_BONES, 3, 3))
    wt = np.zeros((k, N_BONES, 3))
    bob = 0.03 * np.abs(np.sin(ang[:, 0]))               # the pelvis rises twice a cycle
    for b in range(N_BONES):
        p = PARENTS[b]
        if p < 0:
            wr[:, b] = local[:, b]
            wt[:, b] = HEADS[b] + np.stack([np.zeros(k), bob, np.zeros(k)], 1)
        else:
            wr[:, b] = wr[:, p] @ local[:, b]
            wt[:, b] = wt[:, p] + np.einsum("kij,j->ki", wr[:, p], HEADS[b] - HEADS[p])
    out = np.zeros((k, N_BONES, 3, 4))
    out[..., :3] = wr
    out[..., 3] = wt - np.einsum("kbij,bj->kbi", wr, HEADS)
    return out.astype(np.float32)


def walkers(n: int, extent: float, seed: int = 3):
    """Each instance's walk: a circle (centre, radius, angular speed, start angle)."""
    rng = np.random.default_rng(seed)
    side = int(math.ceil(math.sqrt(n)))
    cell = 2.0 * extent / side
    idx = rng.permutation(side * side)[:n]
    cx = -extent + (idx % side + 0.5) * cell + rng.uniform(-0.3, 0.3, n) * cell
    cz = -extent + (idx // side + 0.5) * cell + rng.uniform(-0.3, 0.3, n) * cell
    radius = rng.uniform(1.0, 6.0, n)
    omega = 1.4 / radius * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    a0 = rng.uniform(0.0, 2.0 * math.pi, n)
    return cx, cz, radius, omega, a0


def instance_worlds(t: float, walk) -> np.ndarray:
    """(n, 3, 4) float32 world matrices at time t: on its circle, facing along it."""
    cx, cz, radius, omega, a0 = walk
    a = a0 + omega * t
    x, z = cx + radius * np.cos(a), cz + radius * np.sin(a)
    # the tangent of travel, and the yaw that turns model +z onto it
    tx, tz = -np.sin(a) * np.sign(omega), np.cos(a) * np.sign(omega)
    yaw = np.arctan2(tx, tz)
    c, s = np.cos(yaw), np.sin(yaw)
    w = np.zeros((len(x), 3, 4))
    w[:, 0, 0], w[:, 0, 2], w[:, 0, 3] = c, s, x
    w[:, 1, 1], w[:, 1, 3] = 1.0, 0.0
    w[:, 2, 0], w[:, 2, 2], w[:, 2, 3] = -s, c, z
    return w.astype(np.float32)


FPS = 30.0


def crowd_camera(frame: int, width: int, height: int, extent: float) -> Camera:
    a = 0.6 + 0.004 * frame
    r = 0.75 * extent
    return Camera.look_at((r * math.sin(a), 0.28 * extent, r * math.cos(a)), (0.0, 0.0, 0.0), 45.0, width, height)


@dataclass
class Crowd:
    desc: SceneDescription
    body: Humanoid
    groups: int
    n: int
    walk: tuple
    phase: np.ndarray
    scale: np.ndarray
    extent: float


def crowd(n: int = 5000, groups: int = 1, width: int = 1280, height: int = 720, max_depth: int = 3,
          extent: float = 75.0, ground_segments: int = 158, n_emitters: int = 200, seed: int = 11,
          body: Humanoid | None = None, sky_size=(1024, 512), sky: str = "atmosphere") -> Crowd:
    """Config 2 at frame 0: n walkers (meshes 0 .. groups - 1: the humanoid and its repeats, instance i on mesh
    i % groups), the ground (158 x 158 quads: 49,928 triangles) and config 1's light set: 200 emissive quads of
    log-uniform 10-1000 nits (here lamps 4-6 m up, facing down), the 90,000-lux sun at 28 degrees and config 1's sky
    (the atmosphere baked on the device, or with sky="gradient" the gradient sky)."""
    rng = np.random.default_rng(seed)
    body = body or humanoid()
    meshes = [body.mesh] + [Mesh(body.mesh.positions, like=0) for _ in range(groups - 1)]
    materials = [Material(base=tuple(srgb_to_linear(rng.uniform(0.1, 0.9, 3))), roughness=float(rng.uniform(0.3, 0.9)),
                          specular=0.5) for _ in range(16)]
    walk = walkers(n, extent, seed + 1)
    worlds = instance_worlds(0.0, walk)
    cloth = rng.integers(0, 16, n)
    instances = [Instance(i % groups, [int(cloth[i])], worlds[i], object=i) for i in range(n)]
    materials.append(Material(base=(0.25, 0.25, 0.22), roughness=0.85, specular=0.5))
    meshes.append(plane_mesh(4.0 * extent, ground_segments))
    instances.append(Instance(len(meshes) - 1, [len(materials) - 1], object=n))
    if n_emitters:
        tris, nrm, sec = [], [], []
        first_mat = len(materials)
        for e in range(n_emitters):
            sx, sz = rng.uniform(0.8, 2.0, 2)
            cx, cz = rng.uniform(-1.5 * extent, 1.5 * extent, 2)
            cy = rng.uniform(4.0, 6.0)
            c = np.array([cx, cy, cz])
            t, nn = quad([c + (-sx, 0, -sz), c + (sx, 0, -sz), c + (sx, 0, sz), c + (-sx, 0, sz)], (0, -1, 0))
            tris.append(t)
            nrm.append(nn)
            sec += [e, e]
            nits = float(np.exp(rng.uniform(math.log(10.0), math.log(1000.0))))
            tint = srgb_to_linear(rng.uniform(0.6, 1.0, 3))
            tint = tint / (0.2126 * tint[0] + 0.7152 * tint[1] + 0.0722 * tint[2])
            materials.append(Material(base=(0.05, 0.05, 0.05), emissive=tuple(tint * nits), roughness=0.5,
                                      specular=0.5))
        meshes.append(Mesh(np.concatenate(tris), np.concatenate(nrm), sections=np.asarray(sec, np.uint32),
                           n_sections=n_emitters))
        instances.append(Instance(len(meshes) - 1, list(range(first_mat, first_mat + n_emitters)), object=n + 1))
    el, az = math.radians(28.0), math.radians(35.0)
    to_sun = (math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az))
    if sky == "atmosphere":
        sun = DirLight(direction=tuple(-np.asarray(to_sun)), color=(1.0, 1.0, 1.0), intensity=90000.0)
        sky_desc = Sky("atmosphere", sun_light=0, width=sky_size[0], height=sky_size[1])
    else:
        sun = DirLight(direction=tuple(-np.asarray(to_sun)), color=(1.0, 0.96, 0.9), intensity=90000.0)
        sky_desc = Sky("gradient", zenith=(1200.0, 2000.0, 4000.0), horizon=(5250.0, 5950.0, 7000.0),
                       ground=(600.0, 600.0, 600.0), width=sky_size[0], height=sky_size[1])
    cam = crowd_camera(0, width, height, extent)
    desc = SceneDescription(meshes, materials, instances, cam, lights=[sun], sky=sky_desc,
                            preset=Preset(max_bounces=max_depth, rr_depth=3, clamp_indirect=1.0e9), seed=0x5EED)
    phase, scale = group_params(groups, seed + 2)
    return Crowd(desc, body, groups, n, walk, phase, scale, extent)


# ---- from the prepared buffers: what trt_deform_setup and each frame take ------------------------------------------

RECORD_WORDS = 40


def records(P: prep.Prepared) -> tuple[int, np.ndarray]:
    """The instance section's first vec4 and the records as (units, 40) uint32."""
    t_inst = int(P.params[124 + 7])
    units = int(P.params[68 + 3])
    rec = P.tables[4 * t_inst: 4 * t_inst + RECORD_WORDS * units].reshape(units, RECORD_WORDS)
    return t_inst, rec


def deform_jobs(P: prep.Prepared, c: Crowd) -> tuple[np.ndarray, np.ndarray]:
    """trt_deform_setup's input: the corners (one a vertex of the humanoid, in the prepared vertices' order, which
    every repeat shares) and a job a pose group (its vertices, corner 0, palette group x 30, triangles, tree)."""
    _, rec = records(P)
    info = rec[:, 24:28]
    roots = rec[:, 15]
    top = int(P.params[68 + 2])
    all_roots = np.unique(np.append(roots, top))
    first_tri, first_vertex = info[:c.groups, 0], info[:c.groups, 2]
    n_tris = len(c.body.mesh.positions)
    # The humanoid's vertices as prepared (deduplicated, in its tree's order): each back to its model vertex by
    # (position, normal), which no two model vertices share.
    rows = P.vertices.reshape(-1, 3, 4)
    key = {c.body.positions[i].tobytes() + c.body.normals[i].tobytes(): i for i in range(len(c.body.positions))}
    if len(key) != len(c.body.positions):
        raise ValueError("two model vertices share a position and a normal")
    order = []
    v = int(first_vertex[0])
    while v < len(rows) and len(order) < len(c.body.positions):
        kk = rows[v, 0, :3].astype(np.float32).tobytes() + rows[v, 1, :3].astype(np.float32).tobytes()
        if kk not in key:
            break
        order.append(key[kk])
        v += 1
    order = np.asarray(order)
    if len(order) != len(c.body.positions):
        raise ValueError("the prepared humanoid's vertices are not the model's")
    corners = np.zeros((len(order), 16), np.float32)
    corners[:, 0:3] = c.body.positions[order]
    corners[:, 4:7] = c.body.normals[order]
    b = c.body.bones[order].astype(np.uint32)
    corners[:, 3] = (b[:, 0] | (b[:, 1] << 16)).view(np.float32)
    corners[:, 7] = np.zeros(len(order), np.uint32).view(np.float32)
    corners[:, 11] = np.full(len(order), 1, np.uint32).view(np.float32)  # TRT_CORNER_NORMAL
    corners[:, 12:14] = c.body.weights[order]
    jobs = np.zeros((c.groups, 8), np.uint32)
    for g in range(c.groups):
        r = int(roots[g])
        nxt = all_roots[np.searchsorted(all_roots, r, side="right")]
        jobs[g] = (first_vertex[g], len(order), 0, g * N_BONES, first_tri[g], n_tris, r, nxt - r)
    return corners, jobs


def frame_records(P: prep.Prepared, c: Crowd, t: float) -> np.ndarray:
    """The walkers' records at time t (trt_prep_unit_records over their new worlds, info and roots unchanged)."""
    _, rec = records(P)
    worlds = instance_worlds(t, c.walk)
    return prep.unit_records(worlds, rec[:c.n, 24:28], rec[:c.n, 15], np.ones(c.n, np.uint32))
