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


def _static_args(**kw):
    """A cloud descriptor and splat options for clay_splat_bake_static with host-side values only:
    every case below is refused by the argument checks before any CUDA call."""
    from clay_engine_b200 import _native as N

    desc = N.CloudDesc()
    desc.capacity, desc.positions, desc.position_stride = 4, kw.get("positions", 0x10000), 12
    opts = N.SplatOpts()
    opts.set = N.SPLAT["resolution"] | N.SPLAT["mipLevels"]
    opts.radius = kw.get("radius", 0.1)
    opts.resolution = kw.get("resolution", 64)
    opts.mip_levels = kw.get("mips", 1)
    return desc, opts


@pytest.mark.parametrize("case,message", [
    (dict(resolution=1 << 21), "outside 1..128"),  # its cube would overflow the voxel count
    (dict(resolution=2048), "outside 1..128"),
    (dict(resolution=0), "outside 1..128"),
    (dict(resolution=-64), "outside 1..128"),
    (dict(radius=-0.5), "radius must be a non-negative number"),
    (dict(radius=float("nan")), "radius must be a non-negative number"),
    (dict(dist=0x10002), "dist_out_f16 must be 4-byte aligned"),
    (dict(material=0x20001), "material_out_f16 must be 2-byte aligned"),
    (dict(positions=0x10002), "positions must be 4-byte aligned"),
])
def test_static_bake_refuses_bad_arguments_before_any_launch(clay_lib, case, message):
    """The allocation-free bake checks its arguments on the host: a size its scratch cannot
    hold, a negative radius or a misaligned output is refused with CLAY_EINVAL, never
    launched (the pointers here are not device memory, so nothing may touch them)."""
    import ctypes as C

    from clay_engine_b200 import _native as N

    desc, opts = _static_args(**case)
    rc = N.lib().clay_splat_bake_static(C.byref(desc), C.byref(opts), case.get("dist", 0x30000),
                                        case.get("material", None), None)
    assert rc == N.CLAY_EINVAL
    assert message in N.lib().clay_last_error().decode()
