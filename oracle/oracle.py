"""ctypes wrapper of the CPU restatement in ``oracle/clay_oracle.cpp``.

TEST INFRASTRUCTURE. Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` import this module; the product path never does. Every function here
forwards to the C++ restatement of the reference WGSL (see the header of
``clay_oracle.h`` for the rounding rules and the reference lines each function follows).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libclay_oracle.so")


def build() -> str:
    """Compiles the restatement with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")


class Volume(C.Structure):
    _fields_ = [
        ("res", C.c_int32), ("mips", C.c_int32), ("origin", C.c_double * 3),
        ("world_size", C.c_double), ("band", C.c_double), ("gradient_voxels", C.c_double),
        ("dist", C.c_void_p), ("mat", C.c_void_p),
    ]


class Field(C.Structure):
    _fields_ = [("n", C.c_int32), ("pad", C.c_int32), ("vol", Volume * 8),
                ("offset", (C.c_double * 3) * 8)]


class FluidCfg(C.Structure):
    _fields_ = [
        ("capacity", C.c_uint32), ("bucket", C.c_uint32), ("spacing", C.c_double),
        ("h", C.c_double), ("radius", C.c_double), ("surface_radius", C.c_double),
        ("material", C.c_double), ("bake_res", C.c_int32), ("bake_mips", C.c_int32),
        ("bake_band", C.c_double), ("origin", C.c_double * 3), ("world_size", C.c_double),
        ("substeps", C.c_int32), ("pad", C.c_int32),
    ]


class Params(C.Structure):
    _fields_ = [
        ("gravity", C.c_float * 3), ("dt", C.c_float), ("emit_pos", C.c_float * 3),
        ("emit_radius", C.c_float), ("emit_vel", C.c_float * 3), ("max_speed", C.c_float),
        ("stiffness", C.c_float), ("viscosity", C.c_float), ("damping", C.c_float),
        ("count", C.c_uint32), ("emit_base", C.c_uint32), ("emit_count", C.c_uint32),
        ("emit_seed", C.c_uint32), ("contact_depth", C.c_float),
    ]


class FluidDerived(C.Structure):
    _fields_ = [
        ("h", C.c_double), ("poly6", C.c_double), ("spiky_grad", C.c_double),
        ("mass", C.c_double), ("rest_density", C.c_double), ("grid_res", C.c_int32),
        ("pad", C.c_int32), ("grid_origin", C.c_double * 3), ("wall_lo", C.c_double * 3),
        ("wall_hi", C.c_double * 3),
    ]


class Cloud(C.Structure):
    _fields_ = [
        ("capacity", C.c_uint32), ("pos_stride", C.c_uint32), ("pos", C.c_void_p),
        ("live_mode", C.c_uint32), ("live_a", C.c_uint32), ("live_b", C.c_uint32),
        ("nrm_stride", C.c_uint32), ("nrm", C.c_void_p), ("quat", C.c_void_p),
    ]


class SplatCfg(C.Structure):
    _fields_ = [
        ("res", C.c_int32), ("mips", C.c_int32), ("band", C.c_double), ("radius", C.c_double),
        ("world_size", C.c_double), ("material", C.c_double), ("origin", C.c_double * 3),
    ]


class ExtractCfg(C.Structure):
    _fields_ = [
        ("res", C.c_int32), ("body", C.c_int32), ("base", C.c_int32), ("capacity", C.c_int32),
        ("quad_cap", C.c_int32), ("has_motion", C.c_int32), ("origin", C.c_float * 3), ("cell", C.c_float),
        ("vel", C.c_float * 3), ("preserve", C.c_uint32), ("offset_by_motion", C.c_int32), ("pad", C.c_int32),
    ]


class SolveCfg(C.Structure):
    _fields_ = [
        ("gravity", C.c_float * 3), ("h", C.c_float), ("radius", C.c_float), ("friction", C.c_float),
        ("damping", C.c_float), ("max_speed", C.c_float), ("push", C.c_float * 3), ("push_body", C.c_uint32),
        ("kick", C.c_float * 3), ("capacity", C.c_int32), ("max_bodies", C.c_int32), ("rot_iters", C.c_int32),
        ("substeps", C.c_int32), ("kicking", C.c_int32),
    ]


BRUSH_DTYPE = np.dtype([
    ("pos", np.float32, 3), ("scale", np.float32), ("rot", np.float32, 4),
    ("size", np.float32, 3), ("radius", np.float32), ("material", np.float32),
    ("blend", np.float32), ("bound", np.float32), ("mask", np.float32),
    ("kind", np.uint32), ("op", np.uint32), ("slot", np.uint32), ("pad", np.uint32),
])
assert BRUSH_DTYPE.itemsize == 80

PARTICLE_DTYPE = np.dtype([
    ("pos", np.float32, 3), ("density", np.float32), ("vel", np.float32, 3),
    ("pressure", np.float32), ("nvel", np.float32, 3), ("pad", np.float32),
])
assert PARTICLE_DTYPE.itemsize == 48
PARTICLE_DTYPE_F64 = np.dtype([
    ("pos", np.float64, 3), ("density", np.float64), ("vel", np.float64, 3),
    ("pressure", np.float64), ("nvel", np.float64, 3), ("pad", np.float64),
])


def _declare(L):
    L.orc_hash1.argtypes = [C.c_uint32]
    L.orc_hash1.restype = C.c_float
    L.orc_hash3.argtypes = [C.c_uint32, f32p]
    L.orc_f32_to_f16.argtypes = [C.c_float]
    L.orc_f32_to_f16.restype = C.c_uint16
    L.orc_f16_to_f32.argtypes = [C.c_uint16]
    L.orc_f16_to_f32.restype = C.c_float
    L.orc_volume_mip_levels.argtypes = [C.c_int32, C.c_int32, C.c_char_p, C.c_int32]
    L.orc_volume_mip_levels.restype = C.c_int32
    L.orc_volume_total_voxels.argtypes = [C.c_int32, C.c_int32]
    L.orc_volume_total_voxels.restype = C.c_int64
    L.orc_field_query_f32.argtypes = [C.POINTER(Field), f32p, f32p, f32p]
    L.orc_field_query_f64.argtypes = [C.POINTER(Field), f64p, f64p, f64p]
    L.orc_rest_density.argtypes = [C.c_double, C.c_double]
    L.orc_rest_density.restype = C.c_double
    L.orc_fluid_derive.argtypes = [C.POINTER(FluidCfg), C.POINTER(FluidDerived)]
    L.orc_fluid_cells.argtypes = [C.POINTER(FluidCfg), C.c_void_p, C.c_uint32, u32p]
    L.orc_fluid_emit.argtypes = [C.POINTER(FluidCfg), C.POINTER(Params), C.c_void_p]
    L.orc_fluid_substep_f32.argtypes = [
        C.POINTER(FluidCfg), C.POINTER(Params), C.POINTER(Field), C.c_void_p,
        C.POINTER(C.c_uint32), f32p, u32p, C.c_uint32, C.c_int32]
    L.orc_fluid_substep_f64.argtypes = [
        C.POINTER(FluidCfg), C.POINTER(Params), C.POINTER(Field), C.c_void_p, C.c_int32]
    L.orc_fluid_density_f64.argtypes = [
        C.POINTER(FluidCfg), C.POINTER(Params), C.c_void_p, f64p, C.c_int32]
    L.orc_splat_encode.argtypes = [C.c_float, C.c_float]
    L.orc_splat_encode.restype = C.c_uint32
    L.orc_splat_decode.argtypes = [C.c_uint32]
    L.orc_splat_decode.restype = C.c_float
    L.orc_splat_keys.argtypes = [C.POINTER(SplatCfg), C.POINTER(Cloud), u32p, C.c_int32]
    L.orc_splat_resolve.argtypes = [C.POINTER(SplatCfg), u32p, u16p, u16p]
    L.orc_splat_values_f64.argtypes = [C.POINTER(SplatCfg), C.POINTER(Cloud), f64p, C.c_int32]
    L.orc_build_brushes.argtypes = [C.POINTER(Volume), C.c_void_p, C.c_int32, u16p, u16p, C.c_int32]
    L.orc_eval_brush.argtypes = [C.c_void_p, f32p, C.c_int32, f32p]
    L.orc_field_query_mip_f32.argtypes = [C.POINTER(Field), f32p, C.c_int32, f32p, f32p]
    L.orc_field_query_mip_batch.argtypes = [C.POINTER(Field), f32p, C.c_int64, C.c_int32, f32p, f32p, C.c_int32]
    L.orc_solver_step.argtypes = [C.POINTER(SolveCfg), C.POINTER(Field), C.c_void_p, C.c_void_p, C.c_int32]
    L.orc_sincos_f32.argtypes = [C.c_float, f32p]
    L.orc_extract.argtypes = [C.POINTER(ExtractCfg), C.POINTER(Field), C.c_void_p, C.c_void_p, C.c_void_p, u32p,
                              u32p, u32p, u32p]


# ---------------------------------------------------------------------------------------
# Thin Python helpers over the C entry points.

def hash1(seed: int) -> float:
    return float(lib().orc_hash1(seed & 0xFFFFFFFF))


def hash3(seed: int) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().orc_hash3(seed & 0xFFFFFFFF, out)
    return out


def f32_to_f16(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a, np.float32).ravel()
    return np.array([lib().orc_f32_to_f16(float(x)) for x in a], np.uint16)


def mip_levels(resolution: int, requested: int | None = None):
    err = C.create_string_buffer(256)
    m = lib().orc_volume_mip_levels(resolution, -1 if requested is None else requested, err, 256)
    if m < 0:
        raise ValueError(err.value.decode())
    return m


def total_voxels(res: int, mips: int) -> int:
    return int(lib().orc_volume_total_voxels(res, mips))


class VolumeData:
    """A volume as f16 planes plus its geometry, the oracle's view of an SdfVolume."""

    def __init__(self, res, mips, origin, world_size, band=4.0, gradient_voxels=1.0,
                 dist=None, mat=None):
        self.res, self.mips = int(res), int(mips)
        self.origin = tuple(float(x) for x in origin)
        self.world_size, self.band = float(world_size), float(band)
        self.gradient_voxels = float(gradient_voxels)
        n = total_voxels(self.res, self.mips)
        self.dist = np.ascontiguousarray(dist if dist is not None else np.full(n, 0x3C00, np.uint16), np.uint16)
        self.mat = np.ascontiguousarray(mat if mat is not None else np.zeros(n, np.uint16), np.uint16)

    def c(self) -> Volume:
        v = Volume()
        v.res, v.mips = self.res, self.mips
        v.origin[:] = self.origin
        v.world_size, v.band, v.gradient_voxels = self.world_size, self.band, self.gradient_voxels
        v.dist = self.dist.ctypes.data
        v.mat = self.mat.ctypes.data
        return v


def make_field(volumes, offsets=None) -> Field:
    """A union of volumes as the oracle's field. The field holds raw pointers into the volumes'
    planes, so it keeps the volumes alive for as long as it exists."""
    f = Field()
    f.n = len(volumes)
    for i, v in enumerate(volumes):
        f.vol[i] = v.c()
        off = offsets[i] if offsets is not None else (0.0, 0.0, 0.0)
        f.offset[i][:] = off
    f._volumes = list(volumes)
    return f


def field_query_f32(field: Field, pts: np.ndarray):
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    s = np.zeros((len(pts), 2), np.float32)
    n = np.zeros((len(pts), 3), np.float32)
    o2, o3 = np.zeros(2, np.float32), np.zeros(3, np.float32)
    for i, p in enumerate(pts):
        lib().orc_field_query_f32(C.byref(field), np.ascontiguousarray(p), o2, o3)
        s[i], n[i] = o2, o3
    return s, n


def field_query_mip_f32(field: Field, pts: np.ndarray, mip: int):
    """sample(p, mip) and field(p, mip) at each point: two (n, 2) float32 arrays."""
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    s = np.zeros((len(pts), 2), np.float32)
    f = np.zeros((len(pts), 2), np.float32)
    o2, o2b = np.zeros(2, np.float32), np.zeros(2, np.float32)
    for i, p in enumerate(pts):
        lib().orc_field_query_mip_f32(C.byref(field), np.ascontiguousarray(p), int(mip), o2, o2b)
        s[i], f[i] = o2, o2b
    return s, f


def field_query_mip_batch(field: Field, pts: np.ndarray, mip: int, threads=1):
    """field_query_mip_f32 over all points in one call (OpenMP over points)."""
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    s = np.zeros((len(pts), 2), np.float32)
    f = np.zeros((len(pts), 2), np.float32)
    lib().orc_field_query_mip_batch(C.byref(field), pts, len(pts), int(mip), s, f, int(threads))
    return s, f


def fluid_cfg(**kw) -> FluidCfg:
    c = FluidCfg()
    for k, v in kw.items():
        if k == "origin":
            c.origin[:] = v
        else:
            setattr(c, k, v)
    return c


def derive(cfg: FluidCfg) -> FluidDerived:
    d = FluidDerived()
    lib().orc_fluid_derive(C.byref(cfg), C.byref(d))
    return d


def params_from(d: dict) -> Params:
    p = Params()
    for k, v in d.items():
        if isinstance(v, (list, tuple, np.ndarray)):
            getattr(p, k)[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


def fluid_cells(cfg: FluidCfg, parts: np.ndarray) -> np.ndarray:
    parts = np.ascontiguousarray(parts, PARTICLE_DTYPE)
    keys = np.zeros(len(parts), np.uint32)
    lib().orc_fluid_cells(C.byref(cfg), parts.ctypes.data, len(parts), keys)
    return keys


def fluid_emit(cfg: FluidCfg, prm: Params, parts: np.ndarray) -> None:
    assert parts.dtype == PARTICLE_DTYPE and parts.flags["C_CONTIGUOUS"]
    lib().orc_fluid_emit(C.byref(cfg), C.byref(prm), parts.ctypes.data)


def fluid_substep_f32(cfg, prm, field, parts, threads=1, max_ids=1 << 20):
    """One substep in place on an f32 particle array. Returns (count, points[32,4], ids)."""
    assert parts.dtype == PARTICLE_DTYPE and parts.flags["C_CONTIGUOUS"]
    cnt = C.c_uint32(0)
    pts = np.zeros(32 * 4, np.float32)
    ids = np.zeros(max(max_ids, 1), np.uint32)
    lib().orc_fluid_substep_f32(C.byref(cfg), C.byref(prm), C.byref(field) if field else None,
                                parts.ctypes.data, C.byref(cnt), pts, ids, max_ids, threads)
    n = cnt.value
    return n, pts.reshape(32, 4), ids[: min(n, max_ids)].copy()


def fluid_substep_f64(cfg, prm, field, parts_d, threads=1):
    assert parts_d.dtype == PARTICLE_DTYPE_F64 and parts_d.flags["C_CONTIGUOUS"]
    lib().orc_fluid_substep_f64(C.byref(cfg), C.byref(prm), C.byref(field) if field else None,
                                parts_d.ctypes.data, threads)


def fluid_density_f64(cfg, prm, parts, threads=1) -> np.ndarray:
    parts = np.ascontiguousarray(parts, PARTICLE_DTYPE)
    out = np.zeros(2 * len(parts), np.float64)
    lib().orc_fluid_density_f64(C.byref(cfg), C.byref(prm), parts.ctypes.data, out, threads)
    return out.reshape(-1, 2)


def to_f64(parts: np.ndarray) -> np.ndarray:
    out = np.zeros(len(parts), PARTICLE_DTYPE_F64)
    for name in PARTICLE_DTYPE.names:
        out[name] = parts[name]
    return out


def splat_cfg(res, mips, band, radius, world_size=24.0, material=0.0, origin=(-12.0, -4.0, -12.0)):
    c = SplatCfg()
    c.res, c.mips, c.band, c.radius = res, mips, band, radius
    c.world_size, c.material = world_size, material
    c.origin[:] = origin
    return c


class CloudData:
    """A ParticleCloud as arrays (positions, optional normals, liveness rule)."""

    def __init__(self, pos, normals=None, quat=None, live_mode=0, live_a=0, live_b=0):
        self.pos = np.ascontiguousarray(pos, np.float32)
        self.pos_stride = self.pos.shape[1] if self.pos.ndim == 2 else 3
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32)
        self.quat = None if quat is None else np.ascontiguousarray(quat, np.float32)
        self.live_mode, self.live_a, self.live_b = live_mode, live_a, live_b

    def c(self) -> Cloud:
        c = Cloud()
        c.capacity = self.pos.shape[0]
        c.pos_stride = self.pos_stride
        c.pos = self.pos.ctypes.data
        c.live_mode, c.live_a, c.live_b = self.live_mode, self.live_a, self.live_b
        if self.normals is not None:
            c.nrm = self.normals.ctypes.data
            c.nrm_stride = self.normals.shape[1]
        if self.quat is not None:
            c.quat = self.quat.ctypes.data
        return c


def enc(sd: float, bw: float = 1.0) -> int:
    return int(lib().orc_splat_encode(sd, bw))


def dec(key: int) -> float:
    return float(lib().orc_splat_decode(key))


def splat_keys(cfg: SplatCfg, cloud: CloudData, threads=1) -> np.ndarray:
    keys = np.zeros(total_voxels(cfg.res, cfg.mips), np.uint32)
    cc = cloud.c()
    lib().orc_splat_keys(C.byref(cfg), C.byref(cc), keys, threads)
    return keys


def splat_resolve(cfg: SplatCfg, keys: np.ndarray):
    n = total_voxels(cfg.res, cfg.mips)
    d = np.zeros(n, np.uint16)
    m = np.zeros(n, np.uint16)
    lib().orc_splat_resolve(C.byref(cfg), np.ascontiguousarray(keys, np.uint32), d, m)
    return d, m


def splat_values_f64(cfg: SplatCfg, cloud: CloudData, threads=1) -> np.ndarray:
    vals = np.zeros(total_voxels(cfg.res, cfg.mips), np.float64)
    cc = cloud.c()
    lib().orc_splat_values_f64(C.byref(cfg), C.byref(cc), vals, threads)
    return vals


def build_brushes(vol: VolumeData, brushes: np.ndarray, threads=1):
    brushes = np.ascontiguousarray(brushes, BRUSH_DTYPE)
    n = total_voxels(vol.res, vol.mips)
    d = np.zeros(n, np.uint16)
    m = np.zeros(n, np.uint16)
    v = vol.c()
    lib().orc_build_brushes(C.byref(v), brushes.ctypes.data, len(brushes), d, m, threads)
    return d, m


def eval_brush(brush: np.ndarray, pts) -> np.ndarray:
    b = np.ascontiguousarray(np.asarray(brush, BRUSH_DTYPE).reshape(1))
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    out = np.zeros(len(pts), np.float32)
    lib().orc_eval_brush(b.ctypes.data, pts.ravel(), len(pts), out)
    return out


def extract(field: Field, particles: np.ndarray, bodies: np.ndarray, res: int, body: int, base: int, capacity: int,
            origin, size: float, vel=(0.0, 0.0, 0.0), motion: np.ndarray | None = None, preserve: bool = False,
            offset_by_motion: bool = False):
    """SurfaceExtractor.extract (sim/extract.ts:194-436) on the host, in place on the
    ParticleSet records `particles` (96-byte) and `bodies` (64-byte); `motion` (8 float32,
    in/out) with a motion-relative region. Returns (indices, draw_args, counters)."""
    cfg = ExtractCfg(res=res, body=body, base=base, capacity=capacity, quad_cap=int(math.ceil(capacity * 1.5)),
                     has_motion=1 if motion is not None else 0, cell=float(np.float32(size / res)),
                     preserve=1 if preserve else 0, offset_by_motion=1 if offset_by_motion else 0)
    cfg.origin[:] = [float(np.float32(x)) for x in origin]
    cfg.vel[:] = [float(np.float32(x)) for x in vel]
    assert particles.flags["C_CONTIGUOUS"] and bodies.flags["C_CONTIGUOUS"]
    idx = np.zeros(cfg.quad_cap * 6, np.uint32)
    draw = np.zeros(4, np.uint32)
    cnt = np.zeros(2, np.uint32)
    grid = np.zeros(res ** 3, np.uint32)
    lib().orc_extract(C.byref(cfg), C.byref(field), None if motion is None else motion.ctypes.data,
                      particles.ctypes.data, bodies.ctypes.data, idx, draw, cnt, grid)
    return idx, draw, cnt


def solver_cfg(capacity, max_bodies, gravity=(0.0, -9.81, 0.0), dt=1 / 60, substeps=2, radius=0.1, friction=0.35,
               damping=0.995, max_speed=40.0, rotation_iterations=2) -> SolveCfg:
    """ClaySolverOptions after defaults (sim/pbd.ts:101-118) as the f32 SolveParams uniform."""
    c = SolveCfg(h=float(np.float32(dt / substeps)), radius=float(np.float32(radius)),
                 friction=float(np.float32(friction)), damping=float(np.float32(damping)),
                 max_speed=float(np.float32(max_speed)), push_body=0xFFFFFFFF, capacity=capacity,
                 max_bodies=max_bodies, rot_iters=rotation_iterations, substeps=substeps, kicking=0)
    c.gravity[:] = [float(np.float32(g)) for g in gravity]
    return c


def solver_set_force(cfg: SolveCfg, body, accel, impulse=(0.0, 0.0, 0.0)):
    cfg.push[:] = [float(np.float32(a)) for a in accel]
    cfg.kick[:] = [float(np.float32(a)) for a in impulse]
    cfg.push_body = int(body) & 0xFFFFFFFF
    cfg.kicking = 1 if any(x != 0 for x in impulse) else 0


def solver_step(cfg: SolveCfg, field: Field, particles: np.ndarray, bodies: np.ndarray, body_count: int):
    """ClaySolver.step (sim/pbd.ts:396-416) in place on the ParticleSet records; the kick is
    applied once (the flag is cleared, as the reference's `kicking`)."""
    assert particles.flags["C_CONTIGUOUS"] and bodies.flags["C_CONTIGUOUS"]
    lib().orc_solver_step(C.byref(cfg), C.byref(field), particles.ctypes.data, bodies.ctypes.data, int(body_count))
    if body_count > 0:
        cfg.kicking = 0


def sincos(x: float):
    out = np.zeros(2, np.float32)
    lib().orc_sincos_f32(float(x), out)
    return float(out[0]), float(out[1])
