"""The C-ABI libraries load and export every entry point their headers declare (no GPU needed:
nothing here calls into the device)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(clay_\w+|orc_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def clay_lib():
    from clay_engine_b200 import build

    build.build()
    return ctypes.CDLL(build.LIB)


def test_library_exports_every_declared_symbol(clay_lib):
    names = declared(os.path.join(ROOT, "include", "clay_fluid.h"))
    assert len(names) > 40
    missing = [n for n in names if not hasattr(clay_lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from clay_engine_b200 import _native

    names = declared(os.path.join(ROOT, "include", "clay_fluid.h"))
    assert sorted(_native.SIGNATURES) == names


def test_oracle_exports_every_declared_symbol(oracle):
    names = declared(os.path.join(ROOT, "oracle", "clay_oracle.h"))
    L = oracle.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_the_reference():
    """FluidParticle is 48 B (fluid.ts:20-26), FluidParams 80 B (fluid.ts:28-51), Brush 80 B
    (brush.ts:52-78), ContactList 528 B (fluid.ts:55-58)."""
    from clay_engine_b200 import _native as N
    from clay_engine_b200.core import PARTICLE_DTYPE

    assert PARTICLE_DTYPE.itemsize == 48
    assert ctypes.sizeof(N.FluidParams) == 80
    assert ctypes.sizeof(N.Brush) == 80
    assert ctypes.sizeof(N.ContactList) == 16 + 32 * 16


def test_no_cpu_fallback_when_library_missing(tmp_path, monkeypatch):
    """The host API raises rather than computing anything without the CUDA library."""
    from clay_engine_b200 import _native

    monkeypatch.setattr(_native, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_native, "_lib", None)
    with pytest.raises(ImportError, match="no CPU fallback"):
        _native.lib()
