"""Test infrastructure, not product code: the CPU oracle of the path-trace pass.

A C++ restatement of the reference's offline kernel (oracle.cpp, built by the Makefile beside it into
liboracle.so) with ctypes bindings. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as
the checker or as the timed CPU baseline; the product never calls it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"


class _Scene(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("n_vertex_vec4", C.c_uint64), ("leaves", C.c_void_p),
                ("n_leaf_vec4", C.c_uint64), ("nodes", C.c_void_p), ("n_nodes", C.c_uint64), ("tables", C.c_void_p),
                ("n_table_vec4", C.c_uint64), ("words", C.c_void_p), ("n_words", C.c_uint64),
                ("env_half", C.c_void_p), ("env_w", C.c_uint32), ("env_h", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("node_visits", C.c_uint64),
                ("tri_tests", C.c_uint64), ("unit_entries", C.c_uint64)]


def build(force: bool = False) -> Path:
    """Builds liboracle.so with make (g++)."""
    if force or not LIB_PATH.exists() or any(
            p.stat().st_mtime > LIB_PATH.stat().st_mtime for p in (HERE / "oracle.cpp", HERE / "deform.cpp", HERE / "denoise.cpp", HERE / "sky.cpp", HERE / "emitters.cpp", HERE / "oracle.h")):
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "liboracle.so"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER
        L.orc_render.argtypes = [P(_Scene), P(C.c_uint32), C.c_uint32, C.c_uint32, P(C.c_float), C.c_int, P(Stats)]
        L.orc_render_pixels.argtypes = [P(_Scene), P(C.c_uint32), C.c_uint32, C.c_uint32, P(C.c_uint32), C.c_uint64,
                                        P(C.c_float), C.c_int, P(Stats)]
        L.orc_trace.argtypes = [P(_Scene), P(C.c_uint32), C.c_void_p, C.c_uint64, C.c_void_p, C.c_int, P(Stats)]
        L.orc_trace_brute.argtypes = [P(_Scene), P(C.c_uint32), C.c_void_p, C.c_uint64, C.c_void_p, C.c_int]
        L.orc_intersect.argtypes = [P(_Scene), P(C.c_uint32), C.c_void_p, C.c_void_p, C.c_uint64, P(C.c_float)]
        L.orc_rng4.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, P(C.c_float)]
        L.orc_rng4.restype = None
        L.orc_sobol_directions.argtypes = [P(C.c_uint32)]
        L.orc_sobol_directions.restype = None
        L.orc_hash_hp.argtypes = [C.c_uint32]
        L.orc_hash_hp.restype = C.c_uint32
        L.orc_hardware_threads.restype = C.c_int
        L.orc_skin.argtypes = [P(C.c_uint32), C.c_uint32, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.orc_leaf_gather.argtypes = [P(C.c_uint32), C.c_uint32, P(C.c_float), P(C.c_uint32), C.c_uint32, P(C.c_float)]
        L.orc_refit.argtypes = [P(C.c_uint32), C.c_uint32, P(C.c_float), P(C.c_uint32), C.c_uint32, P(C.c_uint32)]
        L.orc_denoise.argtypes = [P(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32, P(C.c_float)]
        L.orc_sky_exp4.argtypes = [P(C.c_double), P(C.c_double)]
        L.orc_sky_exp4.restype = None
        L.orc_sky_columns.argtypes = [C.c_double, C.c_double, P(C.c_double)]
        L.orc_sky_columns.restype = None
        L.orc_sky_sun_transmittance.argtypes = [C.c_float, C.c_float, C.c_float, P(C.c_float), P(C.c_float),
                                                P(C.c_float)]
        L.orc_sky_sun_transmittance.restype = None
        L.orc_sky_horizon_elevation.argtypes = [C.c_float]
        L.orc_sky_horizon_elevation.restype = C.c_float
        L.orc_sky_tables.argtypes = [C.c_float, C.c_float, C.c_float, P(C.c_float)]
        L.orc_sky_tables.restype = C.c_void_p
        L.orc_sky_tables_free.argtypes = [C.c_void_p]
        L.orc_sky_tables_free.restype = None
        L.orc_sky_tables_get.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.orc_sky_tables_get.restype = None
        L.orc_sky_transmittances.argtypes = [C.c_void_p, C.c_double, C.c_double, P(C.c_double), P(C.c_double)]
        L.orc_sky_transmittances.restype = None
        L.orc_sky_radiance.argtypes = [C.c_void_p, C.c_float, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.orc_sky_radiance.restype = None
        L.orc_sky_bake.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float), C.c_float, C.c_uint32, C.c_uint32,
                                   P(C.c_float), C.c_float, C.c_int, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.orc_sky_bake.restype = None
        L.orc_weigh_emitters.argtypes = [P(C.c_uint32), C.c_uint64, P(C.c_uint32), C.c_uint64, P(C.c_uint32),
                                         C.c_uint32, P(C.c_float), P(C.c_float)]
        L.orc_weigh_emitters.restype = None
        _lib = L
    return _lib


class Oracle:
    """The oracle over one prepared scene (threert_b200.prep.Prepared: the buffers the GPU pass takes)."""

    def __init__(self, prepared):
        self.p = prepared
        self._keep = [np.ascontiguousarray(a) for a in (prepared.vertices, prepared.leaves, prepared.nodes,
                                                         prepared.tables, prepared.words, prepared.env_half)]
        v, l, n, t, w, e = self._keep
        self.scene = _Scene(v.ctypes.data, v.size // 4, l.ctypes.data, l.size // 4, n.ctypes.data, n.size // 8,
                            t.ctypes.data, t.size // 4, w.ctypes.data, w.size, e.ctypes.data, prepared.env_w,
                            prepared.env_h)

    def render(self, params, spp: int, first_sample: int = 0, pixels=None, threads: int = 0, accum=None):
        """accum (w * h, 20) float32 after `spp` samples (added to `accum` if given), and the walk's counts."""
        L = lib()
        p = np.ascontiguousarray(params, dtype=np.uint32)
        w, h = int(p[16]), int(p[17])
        acc = np.zeros((w * h, 20), np.float32) if accum is None else accum
        st = Stats()
        if pixels is None:
            L.orc_render(C.byref(self.scene), p.ctypes.data_as(C.POINTER(C.c_uint32)), first_sample, spp,
                         acc.ctypes.data_as(C.POINTER(C.c_float)), threads, C.byref(st))
        else:
            px = np.ascontiguousarray(pixels, dtype=np.uint32)
            L.orc_render_pixels(C.byref(self.scene), p.ctypes.data_as(C.POINTER(C.c_uint32)), first_sample, spp,
                                px.ctypes.data_as(C.POINTER(C.c_uint32)), len(px),
                                acc.ctypes.data_as(C.POINTER(C.c_float)), threads, C.byref(st))
        return acc, {f[0]: getattr(st, f[0]) for f in Stats._fields_}

    def trace(self, params, rays, brute: bool = False, threads: int = 0):
        from threert_b200.gpu import HIT_DTYPE, RAY_DTYPE
        L = lib()
        r = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.zeros(len(r), HIT_DTYPE)
        p = np.ascontiguousarray(params, dtype=np.uint32)
        st = Stats()
        if brute:
            L.orc_trace_brute(C.byref(self.scene), p.ctypes.data_as(C.POINTER(C.c_uint32)), r.ctypes.data, len(r),
                              hits.ctypes.data, threads)
        else:
            L.orc_trace(C.byref(self.scene), p.ctypes.data_as(C.POINTER(C.c_uint32)), r.ctypes.data, len(r),
                        hits.ctypes.data, threads, C.byref(st))
        return hits, {f[0]: getattr(st, f[0]) for f in Stats._fields_}


    def intersect(self, params, rays, hits):
        """The t of each hit's own triangle along its ray (inf where it misses or names none)."""
        from threert_b200.gpu import HIT_DTYPE, RAY_DTYPE
        r = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        h = np.ascontiguousarray(hits, dtype=HIT_DTYPE)
        t = np.zeros(len(r), np.float32)
        p = np.ascontiguousarray(params, dtype=np.uint32)
        lib().orc_intersect(C.byref(self.scene), p.ctypes.data_as(C.POINTER(C.c_uint32)), r.ctypes.data, h.ctypes.data,
                            len(r), t.ctypes.data_as(C.POINTER(C.c_float)))
        return t


def rng4(pixel_seed: int, index: int, dim: int) -> np.ndarray:
    out = (C.c_float * 4)()
    lib().orc_rng4(pixel_seed, index, dim, out)
    return np.array(out[:], np.float32)


def sobol_directions() -> np.ndarray:
    out = (C.c_uint32 * 96)()
    lib().orc_sobol_directions(out)
    return np.array(out[:], np.uint32).reshape(3, 32)


def hash_hp(x: int) -> int:
    return int(lib().orc_hash_hp(x))


def hardware_threads() -> int:
    return int(lib().orc_hardware_threads())


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def deform(jobs, corners, palette, vertices, leaves, nodes, words, w_indices: int):
    """skin.wgsl, leaf_gather.wgsl and units.rs refit over the jobs: new (vertices, leaves, nodes) arrays."""
    j = np.ascontiguousarray(jobs, np.uint32).reshape(-1, 8)
    c = np.ascontiguousarray(corners, np.float32).reshape(-1, 16)
    pal = np.ascontiguousarray(palette, np.float32).reshape(-1, 12)
    v = np.array(vertices, np.float32, copy=True, order="C")
    lv = np.array(leaves, np.float32, copy=True, order="C")
    nd = np.array(nodes, np.uint32, copy=True, order="C")
    w = np.ascontiguousarray(words, np.uint32)
    L = lib()
    L.orc_skin(_p(j, C.c_uint32), len(j), _p(c, C.c_float), _p(pal, C.c_float), _p(v, C.c_float))
    L.orc_leaf_gather(_p(j, C.c_uint32), len(j), _p(v, C.c_float), _p(w, C.c_uint32), w_indices, _p(lv, C.c_float))
    L.orc_refit(_p(j, C.c_uint32), len(j), _p(v, C.c_float), _p(w, C.c_uint32), w_indices, _p(nd, C.c_uint32))
    return v, lv, nd


def denoise(accum, width: int, height: int, iterations: int = 4) -> np.ndarray:
    """denoise.rs over the Frame of the accum: (height, width, 3) float32."""
    a = np.ascontiguousarray(accum, np.float32).reshape(-1, 20)
    out = np.zeros((height, width, 3), np.float32)
    lib().orc_denoise(_p(a, C.c_float), width, height, iterations, _p(out, C.c_float))
    return out


def _f32(v, n=None):
    a = np.ascontiguousarray(v, np.float32).ravel()
    assert n is None or a.size == n
    return a


class Sky:
    """renderer/src/sky.rs's atmosphere on the CPU: Atmosphere::earth(rayleigh, mie, g, ground) and its Luts::build
    tables (built once, in the constructor), the sky's radiance and the equirectangular bake."""

    SUN_TABLE = (257, 128)
    SCATTER_TABLE = (64, 32)

    def __init__(self, rayleigh: float = 1.0, mie: float = 1.0, g: float = 0.8, ground=(0.401978,) * 3):
        self.args = (float(rayleigh), float(mie), float(g), _f32(ground, 3))
        self.h = lib().orc_sky_tables(*self.args[:3], _p(self.args[3], C.c_float))

    def close(self):
        if self.h:
            lib().orc_sky_tables_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        """(sun (128, 257, 3), scattered (32, 64, 3), ground (64, 3)) float32."""
        (sc, sr), (gc, gr) = self.SUN_TABLE, self.SCATTER_TABLE
        sun = np.zeros((sr, sc, 3), np.float32)
        scat = np.zeros((gr, gc, 3), np.float32)
        ground = np.zeros((gc, 3), np.float32)
        lib().orc_sky_tables_get(self.h, _p(sun, C.c_float), _p(scat, C.c_float), _p(ground, C.c_float))
        return sun, scat, ground

    def transmittances(self, r: float, mu: float):
        """(exp(-optical_depth(r, mu)), the sun table's transmittance at (mu, r)), each 3 float64."""
        a, b = np.zeros(3), np.zeros(3)
        lib().orc_sky_transmittances(self.h, r, mu, _p(a, C.c_double), _p(b, C.c_double))
        return a, b

    def radiance(self, altitude_km: float, direction, sun) -> np.ndarray:
        """Luts::sky: radiance per unit of the sun's illuminance, planet frame (Z up)."""
        d, s, out = _f32(direction, 3), _f32(sun, 3), np.zeros(3, np.float32)
        lib().orc_sky_radiance(self.h, altitude_km, _p(d, C.c_float), _p(s, C.c_float), _p(out, C.c_float))
        return out

    def bake(self, sun_dir, sun_lux, altitude_m: float, width: int, height: int, glow=(0.0,) * 7,
             cover: float = 0.0, planet: bool = False):
        """bake_atmosphere_with: (texels (height, width, 4) float32, sun illuminance (3,), horizon_v)."""
        tex = np.zeros((height, width, 4), np.float32)
        sd, sl, gl = _f32(sun_dir, 3), _f32(sun_lux, 3), _f32(glow, 7)
        sun = np.zeros(3, np.float32)
        hv = C.c_float()
        lib().orc_sky_bake(self.h, _p(sd, C.c_float), _p(sl, C.c_float), altitude_m, width, height,
                           _p(gl, C.c_float), cover, 1 if planet else 0, _p(tex, C.c_float), _p(sun, C.c_float),
                           C.byref(hv))
        return tex, sun, hv.value


def sky_exp4(x) -> np.ndarray:
    a = np.ascontiguousarray(x, np.float64)
    out = np.zeros(4)
    lib().orc_sky_exp4(_p(a, C.c_double), _p(out, C.c_double))
    return out


def sky_columns(r: float, mu: float) -> np.ndarray:
    out = np.zeros(3)
    lib().orc_sky_columns(r, mu, _p(out, C.c_double))
    return out


def sky_sun_transmittance(direction, rayleigh=1.0, mie=1.0, g=0.8, ground=(0.0,) * 3) -> np.ndarray:
    out = np.zeros(3, np.float32)
    gr, d = _f32(ground, 3), _f32(direction, 3)
    lib().orc_sky_sun_transmittance(rayleigh, mie, g, _p(gr, C.c_float), _p(d, C.c_float), _p(out, C.c_float))
    return out


def sky_horizon_elevation(altitude_km: float) -> float:
    return float(lib().orc_sky_horizon_elevation(altitude_km))


def weigh_emitters(tables, words, params, tree_nodes: int, lod=None, cull=None) -> np.ndarray:
    """emitter_weights.wgsl over a copy of the scene's tables: the tables with the emitters' entries, guide, header
    and the light tree's powers made again."""
    t = np.array(tables, np.uint32, copy=True, order="C")
    w = np.ascontiguousarray(words, np.uint32)
    p = np.ascontiguousarray(params, np.uint32)
    lo = _f32(lod, 4) if lod is not None else None
    cu = _f32(cull, 6) if cull is not None else None
    lib().orc_weigh_emitters(_p(t, C.c_uint32), t.size // 4, _p(w, C.c_uint32), w.size, _p(p, C.c_uint32), tree_nodes,
                             _p(lo, C.c_float) if lo is not None else None,
                             _p(cu, C.c_float) if cu is not None else None)
    return t
