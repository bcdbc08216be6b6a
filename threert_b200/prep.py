"""Scene descriptions and the host prep (include/threert_prep.h) from Python.

A `SceneDescription` holds what ThreeRT's scene build hands `prepare_as` (renderer/src/lib.rs:530): meshes in model
space, metal-rough materials, instances placing meshes with a material per section, directional lights, a sky, a
camera and the render preset. `prepare` runs the native prep and returns the packed buffers the pass takes
(`Prepared`, the counterpart of lib.rs:66-88 `Prepared`).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

SUN_ANGULAR_DIAMETER = 0.5357  # degrees (packages/scene/src/core.ts:2134, the default sun)
DEFAULT_SEED = 0x5EED          # lib.rs:312-315 rng_seed


@dataclass
class Mesh:
    positions: np.ndarray                 # (n, 3, 3) model-space corners
    normals: np.ndarray | None = None     # (n, 3, 3) corner normals, None: the triangle's own
    uvs: np.ndarray | None = None         # (n, 3, 2)
    sections: np.ndarray | None = None    # (n,) section of each triangle
    n_sections: int = 1
    like: int | None = None               # an earlier mesh this one repeats (own vertices, leaves and tree)


@dataclass
class Material:
    base: tuple = (0.8, 0.8, 0.8)
    emissive: tuple = (0.0, 0.0, 0.0)
    metallic: float = 0.0
    roughness: float = 1.0
    specular: float = 0.5
    card: bool = False
    opacity: float = 1.0


def lambert(albedo) -> Material:
    """tests/render/lib.ts:49-50 `lambert`: roughness 1, metalness 0, specularIntensity 0."""
    a = (albedo, albedo, albedo) if np.isscalar(albedo) else tuple(albedo)
    return Material(base=a, roughness=1.0, metallic=0.0, specular=0.0)


@dataclass
class Instance:
    mesh: int
    materials: list
    world: np.ndarray = field(default_factory=lambda: np.hstack([np.eye(3), np.zeros((3, 1))]).astype(np.float32))
    object: int = 0
    cast_shadow: bool = True


@dataclass
class DirLight:
    direction: tuple                      # the way the light travels
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0                # lux
    angular_diameter: float = SUN_ANGULAR_DIAMETER
    cast_shadow: bool = True
    specular_scale: float = 1.0


@dataclass
class Sky:
    kind: str = "none"                    # none | color | gradient | atmosphere
    color: tuple = (0.0, 0.0, 0.0)
    zenith: tuple = (0.0, 0.0, 0.0)
    horizon: tuple = (0.0, 0.0, 0.0)
    ground: tuple = (0.0, 0.0, 0.0)
    width: int = 1024
    height: int = 512
    # The atmosphere (packages/scene/src/core.ts:2319-2359 SkyAtmosphere; scene.rs:1397-1414): its sun is directional
    # light `sun_light` (its direction and colour x intensity); baked on the device (sky.rs:643) at width x height.
    sun_light: int = 0
    rayleigh_scale: float = 1.0
    mie_scale: float = 1.0
    mie_anisotropy: float = 0.8
    ground_albedo: tuple = (0.401978, 0.401978, 0.401978)
    altitude: float | None = None         # a planet's viewer altitude (m); None: the camera's height, a flat world
    glow: tuple = (0.0, 0.0, 0.0)         # nits
    horizon_glow: tuple = (0.0, 0.0, 0.0)
    horizon_glow_height: float = 0.06
    cloud_cover: float = 0.0


@dataclass
class Camera:
    position: tuple
    forward: tuple
    right: tuple
    up: tuple
    tan_half_fov: float
    width: int
    height: int

    @staticmethod
    def look_at(position, target, fov_deg, width, height, world_up=(0.0, 1.0, 0.0)) -> "Camera":
        """A pinhole camera at `position` looking at `target`; fov_deg is the vertical field of view."""
        p = np.asarray(position, np.float64)
        f = np.asarray(target, np.float64) - p
        f /= np.linalg.norm(f)
        r = np.cross(f, np.asarray(world_up, np.float64))
        r /= np.linalg.norm(r)
        u = np.cross(r, f)
        return Camera(tuple(p), tuple(f), tuple(r), tuple(u), math.tan(math.radians(fov_deg) * 0.5), width, height)


@dataclass
class Preset:
    max_bounces: int = 8
    rr_depth: int = 3
    clamp_indirect: float = 1.0e9
    energy_compensation: float = 0.0


@dataclass
class SceneDescription:
    meshes: list
    materials: list
    instances: list
    camera: Camera
    lights: list = field(default_factory=list)
    sky: Sky = field(default_factory=Sky)
    preset: Preset = field(default_factory=Preset)
    object_power: list | None = None
    seed: int = DEFAULT_SEED
    light_tree: bool = True


@dataclass
class Prepared:
    """The packed buffers and the base Params of a scene (what trt_scene_upload and trt_render take)."""
    vertices: np.ndarray   # float32 (n, 4), 3 rows a vertex
    leaves: np.ndarray     # float32 (n, 4), 3 rows a triangle
    nodes: np.ndarray      # uint32 (n, 8)
    tables: np.ndarray     # uint32
    words: np.ndarray      # uint32
    env_half: np.ndarray   # uint16 (env_w * env_h * 4)
    env_w: int
    env_h: int
    params: np.ndarray     # uint32 (156,)
    info: dict
    # An atmosphere sky still to bake on a device (Gpu.upload bakes it): (its trt_atmosphere, the sun light's index).
    sky_pending: tuple | None = None

    def with_size(self, width: int, height: int) -> np.ndarray:
        p = self.params.copy()
        aspect = np.float32(width / height)
        p[7] = aspect.view(np.uint32)
        p[16], p[17] = width, height
        return p

    @property
    def width(self):
        return int(self.params[16])

    @property
    def height(self):
        return int(self.params[17])


def _f32(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if shape is not None:
        a = a.reshape(shape)
    return a


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


def prepare(desc: SceneDescription) -> Prepared:
    L = N.lib()
    keep = []
    meshes = (N.MeshSpec * len(desc.meshes))()
    for k, m in enumerate(desc.meshes):
        if m.like is not None:
            src = desc.meshes[m.like]
            meshes[k] = N.MeshSpec(len(np.asarray(src.positions).reshape(-1, 9)), None, None, None, None,
                                   src.n_sections, m.like + 1)
            continue
        pos = _f32(m.positions, (-1, 9))
        nrm = _f32(m.normals, (-1, 9)) if m.normals is not None else None
        uvs = _f32(m.uvs, (-1, 6)) if m.uvs is not None else None
        sec = np.ascontiguousarray(m.sections, dtype=np.uint32) if m.sections is not None else None
        keep += [pos, nrm, uvs, sec]
        meshes[k] = N.MeshSpec(pos.shape[0], _ptr(pos, C.c_float), _ptr(nrm, C.c_float), _ptr(uvs, C.c_float),
                               _ptr(sec, C.c_uint32), m.n_sections, 0)
    mats = (N.MaterialSpec * max(1, len(desc.materials)))()
    for k, m in enumerate(desc.materials):
        mats[k] = N.MaterialSpec((C.c_float * 4)(*m.base[:3], m.opacity), (C.c_float * 3)(*m.emissive), m.metallic,
                                 m.roughness, m.specular, 1 if m.card else 0)
    insts = (N.InstanceSpec * len(desc.instances))()
    for k, i in enumerate(desc.instances):
        sm = np.ascontiguousarray(i.materials, dtype=np.uint32)
        keep.append(sm)
        w = _f32(i.world, (12,))
        insts[k] = N.InstanceSpec(i.mesh, i.object, (C.c_float * 12)(*w), _ptr(sm, C.c_uint32),
                                  1 if i.cast_shadow else 0)
    lights = (N.DirLightSpec * max(1, len(desc.lights)))()
    for k, l in enumerate(desc.lights):
        lights[k] = N.DirLightSpec((C.c_float * 3)(*l.direction), (C.c_float * 3)(*l.color), l.intensity,
                                   l.angular_diameter, 1 if l.cast_shadow else 0, l.specular_scale)
    kinds = {"none": 0, "color": 1, "gradient": 2, "atmosphere": 3}
    s = desc.sky
    sky = N.SkySpec(kinds[s.kind], (C.c_float * 3)(*s.color), (C.c_float * 3)(*s.zenith), (C.c_float * 3)(*s.horizon),
                    (C.c_float * 3)(*s.ground), s.width, s.height)
    c = desc.camera
    cam = N.CameraSpec((C.c_float * 3)(*c.position), (C.c_float * 3)(*c.forward), (C.c_float * 3)(*c.right),
                       (C.c_float * 3)(*c.up), c.tan_half_fov, c.width, c.height, 0.0, 1.0)
    pr = desc.preset
    preset = N.PresetSpec(pr.max_bounces, pr.rr_depth, pr.clamp_indirect, pr.energy_compensation)
    power = _f32(desc.object_power) if desc.object_power is not None else None
    spec = N.SceneSpec(len(desc.meshes), meshes, len(desc.materials), mats, len(desc.instances), insts,
                       0 if power is None else len(power), _ptr(power, C.c_float), len(desc.lights), lights, sky, cam,
                       preset, desc.seed, 1 if desc.light_tree else 0)
    h = C.c_void_p()
    if L.trt_prep_build(C.byref(spec), C.byref(h)) != 0:
        raise ValueError("prep: " + L.trt_prep_last_error().decode())
    try:
        b = N.PreparedBuffers()
        L.trt_prep_buffers(h, C.byref(b))

        def take(ptr, nbytes, dtype, cols=None):
            a = np.frombuffer((C.c_char * nbytes).from_address(ptr), dtype=dtype).copy()
            return a.reshape(-1, cols) if cols else a

        params = np.zeros(N.PARAMS_WORDS, np.uint32)
        L.trt_prep_params(h, params.ctypes.data_as(C.POINTER(C.c_uint32)))
        info = N.PrepInfo()
        L.trt_prep_get_info(h, C.byref(info))
        n_lt = L.trt_prep_light_tree(h, None, None, 0)
        lt_order = np.zeros(max(1, n_lt), np.uint32)
        lt_code = np.zeros(max(1, n_lt), np.uint32)
        L.trt_prep_light_tree(h, lt_order.ctypes.data_as(C.POINTER(C.c_uint32)),
                              lt_code.ctypes.data_as(C.POINTER(C.c_uint32)), n_lt)
        d = {f[0]: getattr(info, f[0]) for f in N.PrepInfo._fields_}
        d["light_tree_order"] = lt_order[:n_lt]
        d["light_tree_codes"] = lt_code[:n_lt]
        return Prepared(
            vertices=take(b.vertices, b.vertices_bytes, np.float32, 4),
            leaves=take(b.leaves, b.leaves_bytes, np.float32, 4),
            nodes=take(b.nodes, b.nodes_bytes, np.uint32, 8),
            tables=take(b.tables, b.tables_bytes, np.uint32),
            words=take(b.words, b.words_bytes, np.uint32),
            env_half=take(b.env_half, b.env_w * b.env_h * 8, np.uint16),
            env_w=b.env_w, env_h=b.env_h, params=params, info=d,
            sky_pending=(atmosphere_of(desc), desc.sky.sun_light if desc.lights else -1)
            if s.kind == "atmosphere" else None)
    finally:
        L.trt_prep_free(h)


def atmosphere_of(desc: SceneDescription) -> N.Atmosphere:
    """The trt_atmosphere of a scene's atmosphere sky (lib.rs:958-982 bake_sky; scene.rs:1397-1414): toward its sun
    light, that light's colour x intensity above the atmosphere, the camera's height unless a planet's altitude."""
    s = desc.sky
    if desc.lights and 0 <= s.sun_light < len(desc.lights):
        l = desc.lights[s.sun_light]
        sun_dir = tuple(-float(v) for v in l.direction)
        sun_lux = tuple(float(c) * float(l.intensity) for c in l.color)
    else:
        sun_dir, sun_lux = (0.0, 1.0, 0.0), (0.0, 0.0, 0.0)
    planet = s.altitude is not None
    altitude = max(float(s.altitude), 0.0) if planet else max(float(desc.camera.position[1]), 0.0)
    return N.Atmosphere((C.c_float * 3)(*sun_dir), (C.c_float * 3)(*sun_lux), s.rayleigh_scale, s.mie_scale,
                        s.mie_anisotropy, (C.c_float * 3)(*s.ground_albedo), altitude, 1 if planet else 0,
                        (C.c_float * 3)(*s.glow), (C.c_float * 3)(*s.horizon_glow), s.horizon_glow_height,
                        s.cloud_cover, s.width, s.height)


def apply_sky(P: Prepared, texels: np.ndarray, result, sun_light: int) -> None:
    """Writes a sky bake into a prepared scene as lib.rs:680-684 and 1005-1010 do: the RGBA16F texels, the CDF (the
    words' first section), the sun light's colour (the illuminance the atmosphere leaves it), Params' env, sky_color.w
    and counts2.y (the sky light-sampled when its brightest luminance reaches the emitters' floor)."""
    L = N.lib()
    h, w = texels.shape[:2]
    if (w, h) != (P.env_w, P.env_h):
        raise ValueError(f"apply_sky: the bake is {w} x {h}, the scene's map {P.env_w} x {P.env_h}")
    tex = np.ascontiguousarray(texels, np.float32)
    env = np.zeros(w * h * 4, np.uint16)
    cdf = np.zeros(h + w * h, np.float32)
    bright = C.c_float()
    if L.trt_prep_env(tex.ctypes.data_as(C.POINTER(C.c_float)), w, h, env.ctypes.data_as(C.POINTER(C.c_uint16)),
                      cdf.ctypes.data_as(C.POINTER(C.c_float)), C.byref(bright)) != 0:
        raise ValueError("trt_prep_env: " + L.trt_prep_last_error().decode())
    P.env_half = env
    at = int(P.params[136])
    P.words[at:at + cdf.size] = cdf.view(np.uint32)
    if sun_light >= 0:
        lt = (int(P.params[126]) + sun_light * 5 + 2) * 4
        P.tables[lt:lt + 4] = np.array([*result.sun_illuminance, 0.0], np.float32).view(np.uint32)
    pf = P.params.view(np.float32)
    pf[24], pf[25], pf[26] = 1.0, float(w), float(h)
    pf[35] = result.horizon_v
    sampled = float(bright.value) >= float(P.info["env_nee_floor"])
    P.params[37] = 1 if sampled else 0
    P.info["env_sampled"] = 1 if sampled else 0
    P.sky_pending = None


def unit_records(worlds: np.ndarray, info: np.ndarray, roots: np.ndarray, cast_shadow: np.ndarray) -> np.ndarray:
    """trt_prep_unit_records: (n, 40) uint32 instance records for worlds (n, 3, 4), info (n, 4), roots (n,)."""
    w = _f32(worlds, (-1, 12))
    n = len(w)
    inf = np.ascontiguousarray(info, np.uint32).reshape(n, 4)
    r = np.ascontiguousarray(roots, np.uint32).reshape(n)
    cs = np.ascontiguousarray(cast_shadow, np.uint32).reshape(n)
    out = np.zeros((n, 40), np.uint32)
    if N.lib().trt_prep_unit_records(n, _ptr(w, C.c_float), _ptr(inf, C.c_uint32), _ptr(r, C.c_uint32),
                                     _ptr(cs, C.c_uint32), _ptr(out, C.c_uint32)) != 0:
        raise ValueError("trt_prep_unit_records failed")
    return out


def units_top(worlds: np.ndarray, local_boxes: np.ndarray) -> tuple[np.ndarray, int]:
    """trt_prep_units_top: the top tree's (2n - 1, 8) uint32 nodes over units with these worlds and model boxes."""
    w = _f32(worlds, (-1, 12))
    n = len(w)
    b = _f32(local_boxes, (n, 6))
    nodes = np.zeros((2 * n - 1, 8), np.uint32)
    depth = C.c_uint32()
    if N.lib().trt_prep_units_top(n, _ptr(w, C.c_float), _ptr(b, C.c_float), _ptr(nodes, C.c_uint32),
                                  C.byref(depth)) != 0:
        raise ValueError("trt_prep_units_top failed")
    return nodes, depth.value


def params_with(params: np.ndarray, **kw) -> np.ndarray:
    """A copy of a Params block with named fields changed: sample, seed, max_bounces, rr_depth, clamp, width, height."""
    p = params.copy()
    f32 = lambda v: np.float32(v).view(np.uint32)
    for k, v in kw.items():
        if k == "sample":
            p[18] = v
        elif k == "seed":
            p[19] = v
        elif k == "max_bounces":
            p[22] = v
        elif k == "rr_depth":
            p[23] = v
        elif k == "clamp":
            p[28] = f32(v)
        elif k == "energy_compensation":
            p[30] = f32(v)
        elif k == "width":
            p[16] = v
            p[7] = f32(v / p[17])
        elif k == "height":
            p[17] = v
            p[7] = f32(p[16] / v)
        else:
            raise KeyError(k)
    return p


def set_camera(params: np.ndarray, cam: Camera) -> np.ndarray:
    """A copy of a Params block with another camera (position, forward, right, up, tan(fov/2))."""
    p = params.copy()
    f = np.zeros(16, np.float32)
    f[0:3], f[3] = cam.position, cam.tan_half_fov
    f[4:7], f[7] = cam.forward, p[7:8].view(np.float32)[0]
    f[8:11], f[11] = cam.right, p[11:12].view(np.float32)[0]
    f[12:15], f[15] = cam.up, p[15:16].view(np.float32)[0]
    p[0:16] = f.view(np.uint32)
    return p
