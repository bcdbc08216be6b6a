"""The C ABI: the library loads without a GPU and exports every function include/*.h declares, with the bindings'
signatures in step (no compute calls here)."""
import ctypes as C
import re
from pathlib import Path

from threert_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(trt_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_function_is_exported():
    declared = declared_functions()
    assert len(declared) >= 25
    lib = N.lib()
    for name in sorted(declared):
        assert hasattr(lib, name), name


def test_the_bindings_cover_the_headers():
    assert declared_functions() == set(N.exported_symbols())


def test_record_sizes():
    assert C.sizeof(N.Ray) == 32 and C.sizeof(N.Hit) == 24
    assert C.sizeof(N.MaterialSpec) == 44


def test_no_alloc_render_refuses_bad_sizes_before_any_cuda_call():
    """trt_render_noalloc checks its arguments on the host first, so these refusals need no GPU: a size past its
    array, and one whose 32-bit path-slot count would wrap to zero (2^20 x 2^14 pixels)."""
    import numpy as np
    from threert_b200 import prep, scenes
    P = prep.prepare(scenes.cornell(8, 8))
    fake = 1 << 40  # device addresses that are never touched: the call returns before its first CUDA call
    d = N.SceneDesc(fake, P.vertices.nbytes, fake, P.leaves.nbytes, fake, P.nodes.nbytes, fake, P.tables.nbytes,
                    fake, P.words.nbytes, fake, P.env_w, P.env_h)
    err = C.create_string_buffer(256)
    L = N.lib()
    for w, h in ((512, 512), (1 << 20, 1 << 14), (0xFFFFFFF9, 1)):
        p = np.ascontiguousarray(prep.params_with(P.params, width=w, height=h), np.uint32)
        rc = L.trt_render_noalloc(C.byref(d), p.ctypes.data_as(C.POINTER(C.c_uint32)), 0, 1, 0, fake, None, err, 256)
        assert rc == N.TRT_EINVAL and b"too large" in err.value, (w, h, rc, err.value)
    p = np.ascontiguousarray(P.params, np.uint32)
    rc = L.trt_render_noalloc(C.byref(d), p.ctypes.data_as(C.POINTER(C.c_uint32)), 0, 1, N.TRT_RENDER_WIDE, fake,
                              None, err, 256)
    assert rc == N.TRT_EINVAL and b"flags" in err.value
