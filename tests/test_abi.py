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
