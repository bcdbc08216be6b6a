"""ctypes bindings of the native library (include/threert_cuda.h, include/threert_prep.h).

The library is built in-tree (threert_b200/build.py). Loading fails loudly when it is missing: there is no other
implementation of the pass to fall back to.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libthreert_b200.so"

u32, u64, f32, i32 = C.c_uint32, C.c_uint64, C.c_float, C.c_int32
P = C.POINTER

PARAMS_WORDS = 156
PIXEL_FLOATS = 20

TRT_RENDER_ACCUMULATE = 1
TRT_RENDER_COUNT = 2
TRT_RENDER_WIDE = 4
TRT_RENDER_SORT_RAYS = 8
TRT_RENDER_UNSORTED_HITS = 16
TRT_RENDER_SORT_SHADOWS = 32
TRT_RENDER_DEPTH = 64
TRT_RENDER_ASYNC_READBACK = 128

TRT_OK, TRT_EINVAL, TRT_ECUDA, TRT_EGUARD = 0, 1, 2, 3
TRT_MATH_COS, TRT_MATH_SIN, TRT_MATH_ACOS, TRT_MATH_ATAN2 = 0, 1, 2, 3
ERRORS = {1: "TRT_EINVAL", 2: "TRT_ECUDA", 3: "TRT_EGUARD"}


class MeshSpec(C.Structure):
    _fields_ = [("n_tris", u32), ("positions", P(f32)), ("normals", P(f32)), ("uvs", P(f32)),
                ("sections", P(u32)), ("n_sections", u32), ("like", u32)]


class MaterialSpec(C.Structure):
    _fields_ = [("base_color", f32 * 4), ("emissive", f32 * 3), ("metallic", f32), ("roughness", f32),
                ("specular", f32), ("card", i32)]


class InstanceSpec(C.Structure):
    _fields_ = [("mesh", u32), ("object", u32), ("world", f32 * 12), ("section_materials", P(u32)),
                ("cast_shadow", u32)]


class DirLightSpec(C.Structure):
    _fields_ = [("dir", f32 * 3), ("color", f32 * 3), ("intensity", f32), ("angular_diameter_deg", f32),
                ("cast_shadow", u32), ("specular_scale", f32)]


class SkySpec(C.Structure):
    _fields_ = [("kind", u32), ("color", f32 * 3), ("zenith", f32 * 3), ("horizon", f32 * 3), ("ground", f32 * 3),
                ("width", u32), ("height", u32)]


class CameraSpec(C.Structure):
    _fields_ = [("position", f32 * 3), ("forward", f32 * 3), ("right", f32 * 3), ("up", f32 * 3),
                ("tan_half_fov", f32), ("width", u32), ("height", u32), ("lens_radius", f32),
                ("focus_distance", f32)]


class PresetSpec(C.Structure):
    _fields_ = [("max_bounces", u32), ("rr_depth", u32), ("clamp_indirect", f32), ("energy_compensation", f32)]


class SceneSpec(C.Structure):
    _fields_ = [("n_meshes", u32), ("meshes", P(MeshSpec)), ("n_materials", u32), ("materials", P(MaterialSpec)),
                ("n_instances", u32), ("instances", P(InstanceSpec)), ("n_objects", u32),
                ("object_power", P(f32)), ("n_lights", u32), ("lights", P(DirLightSpec)), ("sky", SkySpec),
                ("camera", CameraSpec), ("preset", PresetSpec), ("seed", u32), ("use_light_tree", u32)]


class PreparedBuffers(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertices_bytes", u64), ("leaves", C.c_void_p), ("leaves_bytes", u64),
                ("nodes", C.c_void_p), ("nodes_bytes", u64), ("tables", C.c_void_p), ("tables_bytes", u64),
                ("words", C.c_void_p), ("words_bytes", u64), ("env_half", C.c_void_p), ("env_w", u32),
                ("env_h", u32)]


class PrepInfo(C.Structure):
    _fields_ = [("n_units", u32), ("top_first", u32), ("n_nodes", u32), ("n_tris", u32), ("n_vertices", u32),
                ("n_emitters", u32), ("light_tree_nodes", u32), ("env_sampled", u32), ("max_mesh_depth", u32),
                ("top_depth", u32), ("emitter_total", f32), ("env_nee_floor", f32)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("flags", u32)]


class SceneDesc(C.Structure):
    _fields_ = PreparedBuffers._fields_


class Stats(C.Structure):
    _fields_ = [("closest_rays", u64), ("shadow_rays", u64), ("paths", u64), ("device_ms", f32),
                ("launches", u32), ("guard_trips", u32)]


class Totals(C.Structure):
    _fields_ = [("closest_rays", u64), ("shadow_rays", u64), ("paths", u64), ("renders", u64), ("launches", u64),
                ("node_visits", u64), ("tri_tests", u64), ("unit_entries", u64), ("shadow_node_visits", u64),
                ("shadow_tri_tests", u64), ("shadow_unit_entries", u64), ("extend_ms", C.c_double),
                ("shadow_ms", C.c_double), ("shade_ms", C.c_double), ("extend_launches", u64),
                ("shadow_launches", u64), ("guard_trips", u64), ("sort_ms", C.c_double)]


class Ray(C.Structure):
    _fields_ = [("o", f32 * 3), ("tmax", f32), ("d", f32 * 3), ("mode", u32)]


class Hit(C.Structure):
    _fields_ = [("t", f32), ("tri", u32), ("u", f32), ("v", f32), ("inst", u32), ("part", u32)]


class Corner(C.Structure):
    _fields_ = [("p", f32 * 4), ("n", f32 * 4), ("t", f32 * 4), ("w", f32 * 4)]


class DeformMesh(C.Structure):
    _fields_ = [("first_vertex", u32), ("n_vertices", u32), ("first_corner", u32), ("palette", u32),
                ("first_tri", u32), ("n_tris", u32), ("root", u32), ("n_nodes", u32)]


class DeformDesc(C.Structure):
    _fields_ = [("corners", C.c_void_p), ("n_corners", u64), ("meshes", P(DeformMesh)), ("n_meshes", u32)]


class DeformStats(C.Structure):
    _fields_ = [("device_ms", f32), ("skin_ms", f32), ("gather_ms", f32), ("refit_ms", f32), ("top_ms", f32),
                ("wide_ms", f32), ("errors", u32)]


TRT_CORNER_NORMAL = 1
TRT_CORNER_TANGENT = 2

class ServerOptions(C.Structure):
    _fields_ = [("wave_slots", u32), ("max_active", u32), ("hbm_reserve", u64), ("flags", u32), ("launch_mode", u32),
                ("denoiser", C.c_void_p), ("denoise_max_spp", u32)]


class RequestDone(C.Structure):
    _fields_ = [("id", u64), ("status", C.c_int32), ("steps", u32), ("submit_ms", C.c_double),
                ("start_ms", C.c_double), ("done_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("steps", u64), ("requests_done", u64), ("paths", u64), ("closest_rays", u64), ("shadow_rays", u64),
                ("busy_ms", C.c_double), ("active", u32), ("pending", u32)]


class Atmosphere(C.Structure):
    _fields_ = [("sun_dir", f32 * 3), ("sun_lux", f32 * 3), ("rayleigh_scale", f32), ("mie_scale", f32),
                ("mie_g", f32), ("ground_albedo", f32 * 3), ("altitude_m", f32), ("planet", u32),
                ("glow_uniform", f32 * 3), ("glow_horizon", f32 * 3), ("glow_height", f32), ("cloud_cover", f32),
                ("width", u32), ("height", u32)]


class SkyResult(C.Structure):
    _fields_ = [("sun_illuminance", f32 * 3), ("horizon_v", f32), ("brightest", f32), ("tables_ms", f32),
                ("bake_ms", f32)]


SKY_TABLE_FLOATS = 3 * (257 * 128 + 64 * 32 + 64)

# Every function the C headers declare, with its signature: (name, restype, argtypes).
SIGNATURES = [
    # threert_prep.h
    ("trt_prep_build", C.c_int, [P(SceneSpec), P(C.c_void_p)]),
    ("trt_prep_free", None, [C.c_void_p]),
    ("trt_prep_env", C.c_int, [P(f32), u32, u32, P(C.c_uint16), P(f32), P(f32)]),
    ("trt_prep_buffers", None, [C.c_void_p, P(PreparedBuffers)]),
    ("trt_prep_params", None, [C.c_void_p, P(u32)]),
    ("trt_prep_get_info", None, [C.c_void_p, P(PrepInfo)]),
    ("trt_prep_light_tree", u32, [C.c_void_p, P(u32), P(u32), u32]),
    ("trt_prep_last_error", C.c_char_p, []),
    ("trt_prep_bvh", u32, [P(f32), u32, u32, P(u32), u32, P(u32), P(u32)]),
    ("trt_prep_check_tree", C.c_int, [P(u32), u32, u32, u32, u32, P(u32)]),
    ("trt_prep_specular_albedo", None, [C.c_double, C.c_double, u32, u32, P(C.c_double)]),
    ("trt_prep_unit_records", C.c_int, [u32, P(f32), P(u32), P(u32), P(u32), P(u32)]),
    ("trt_prep_units_top", C.c_int, [u32, P(f32), P(f32), P(u32), P(u32)]),
    # threert_cuda.h
    ("trt_create", C.c_int, [P(Options), P(C.c_void_p)]),
    ("trt_destroy", None, [C.c_void_p]),
    ("trt_last_error", C.c_char_p, [C.c_void_p]),
    ("trt_device_info", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, P(C.c_int)]),
    ("trt_scene_upload", C.c_int, [C.c_void_p, P(SceneDesc), P(C.c_void_p)]),
    ("trt_scene_free", None, [C.c_void_p]),
    ("trt_scene_update", C.c_int, [C.c_void_p, u32, u64, C.c_void_p, u64]),
    ("trt_scene_read", C.c_int, [C.c_void_p, u32, u64, C.c_void_p, u64]),
    ("trt_denoise_atrous", C.c_int, [C.c_void_p, u32, P(f32), P(f32)]),
    ("trt_sky_bake", C.c_int, [C.c_void_p, P(Atmosphere), P(f32), P(f32), P(SkyResult)]),
    ("trt_scene_weigh_emitters", C.c_int, [C.c_void_p, P(u32), u32, P(f32), P(f32), P(f32)]),
    ("trt_scene_build_light_tree", C.c_int, [C.c_void_p, P(u32), P(u32), P(f32)]),
    ("trt_scene_set_sky", C.c_int, [C.c_void_p, P(Atmosphere), C.c_int32, f32, P(u32), P(SkyResult)]),
    ("trt_deform_setup", C.c_int, [C.c_void_p, P(DeformDesc)]),
    ("trt_deform", C.c_int, [C.c_void_p, P(u32), P(f32), u32, u32, P(DeformStats)]),
    ("trt_render", C.c_int, [C.c_void_p, P(u32), u32, u32, u32, P(f32), P(Stats)]),
    ("trt_accum_device_ptr", C.c_int, [C.c_void_p, P(C.c_void_p), P(u64)]),
    ("trt_accum_read", C.c_int, [C.c_void_p, P(f32), u64]),
    ("trt_accum_copy", C.c_int, [C.c_void_p, C.c_void_p, u64]),
    ("trt_trace", C.c_int, [C.c_void_p, P(u32), P(Ray), u64, u32, P(Hit)]),
    ("trt_render_noalloc", C.c_int, [P(SceneDesc), P(u32), u32, u32, u32, C.c_void_p, C.c_void_p, C.c_char_p,
                                     C.c_size_t]),
    ("trt_server_create", C.c_int, [C.c_void_p, P(ServerOptions), P(C.c_void_p)]),
    ("trt_server_destroy", None, [C.c_void_p]),
    ("trt_server_submit", C.c_int, [C.c_void_p, C.c_void_p, P(u32), u32, P(f32), P(u64)]),
    ("trt_server_submit_rgb", C.c_int, [C.c_void_p, C.c_void_p, P(u32), u32, P(f32), P(f32), P(u64)]),
    ("trt_server_clock", C.c_int, [C.c_void_p, P(C.c_double)]),
    ("trt_server_submit_at", C.c_int, [C.c_void_p, C.c_void_p, P(u32), u32, P(f32), P(f32), C.c_double, P(u64)]),
    ("trt_server_poll", C.c_int, [C.c_void_p, P(RequestDone), u32, P(u32), u32]),
    ("trt_server_stats_get", C.c_int, [C.c_void_p, P(ServerStats)]),
    ("trt_unet_create", C.c_int, [C.c_int, u32, u32, u32, P(C.c_void_p)]),
    ("trt_unet_destroy", None, [C.c_void_p]),
    ("trt_unet_last_error", C.c_char_p, [C.c_void_p]),
    ("trt_unet_param_count", u64, []),
    ("trt_unet_set_params", C.c_int, [C.c_void_p, P(f32)]),
    ("trt_unet_get_params", C.c_int, [C.c_void_p, P(f32)]),
    ("trt_unet_forward", C.c_int, [C.c_void_p, P(f32), u32, u32, u32, P(f32), P(f32)]),
    ("trt_unet_train_step", C.c_int, [C.c_void_p, P(f32), P(f32), u32, u32, u32, f32, C.c_int, P(f32), P(f32), P(f32)]),
    ("trt_unet_denoise_accum", C.c_int, [C.c_void_p, C.c_void_p, u32, u32, P(f32), P(f32)]),
    ("trt_unet_hold_next_load", C.c_int, [C.c_void_p]),
    ("trt_math_eval", C.c_int, [C.c_void_p, u32, P(f32), P(f32), u64, P(f32)]),
    ("trt_scene_totals", C.c_int, [C.c_void_p, P(Totals)]),
    ("trt_scene_reset_totals", None, [C.c_void_p]),
    ("trt_scene_set_profiling", None, [C.c_void_p, C.c_int]),
    ("trt_timer_start", C.c_int, [C.c_void_p]),
    ("trt_timer_stop", C.c_int, [C.c_void_p, P(f32)]),
    ("trt_synchronize", C.c_int, [C.c_void_p]),
]

_lib = None


def lib() -> C.CDLL:
    """The loaded library, with every signature set. Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it first (python -m threert_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return [s[0] for s in SIGNATURES]
