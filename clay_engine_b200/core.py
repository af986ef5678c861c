"""Host API mirroring the reference's `SdfVolume`, `TracedField`, `ParticleCloud`,
`SplatField` and `FluidSim` (lib/src/field/volume.ts, lib/src/trace/field.ts,
lib/src/sim/splat.ts, lib/src/sim/fluid.ts) over the C ABI of ``include/clay_fluid.h``.

Names and option keys follow the reference (camelCase options, the same defaults, the same
error messages); a "pass" is a CUDA stream (None = the legacy default stream, an int
handle, or a ``torch.cuda.Stream``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import ClayError, check, lib, stream_handle

PARTICLE_DTYPE = np.dtype([
    ("pos", np.float32, 3), ("density", np.float32), ("vel", np.float32, 3),
    ("pressure", np.float32), ("nvel", np.float32, 3), ("pad", np.float32),
])
assert PARTICLE_DTYPE.itemsize == 48


class Root:
    """The device context every constructor takes (the reference's `TgpuRoot`)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().clay_ctx_create(device, C.byref(h)))
        self.handle = h.value
        self.device = device

    def bytes_in_use(self) -> int:
        v = C.c_uint64()
        check(lib().clay_ctx_bytes_in_use(self.handle, C.byref(v)))
        return int(v.value)

    def destroy(self):
        if self.handle:
            lib().clay_ctx_destroy(self.handle)
            self.handle = None


def init(device: int = 0) -> Root:
    return Root(device)


def _f16_from_f32(a: np.ndarray) -> np.ndarray:
    return np.asarray(a, np.float32).astype(np.float16).view(np.uint16)


class SdfVolume:
    """`SdfVolume` (volume.ts:91-343)."""

    def __init__(self, root: Root, resolution=None, worldSize=None, origin=None, mipLevels=None,
                 band=None, gradientVoxels=None, label=None, _handle=None):
        self.root = root
        if _handle is None:
            o = N.VolumeOpts()
            for key, val in (("resolution", resolution), ("worldSize", worldSize), ("origin", origin),
                             ("mipLevels", mipLevels), ("band", band), ("gradientVoxels", gradientVoxels)):
                if val is None:
                    continue
                o.set |= N.VOL[key]
                if key == "origin":
                    o.origin[:] = [float(x) for x in val]
                elif key == "worldSize":
                    o.world_size = float(val)
                elif key == "mipLevels":
                    o.mip_levels = int(val)
                elif key == "gradientVoxels":
                    o.gradient_voxels = float(val)
                else:
                    setattr(o, key, val)
            h = C.c_void_p()
            check(lib().clay_volume_create(root.handle, C.byref(o), C.byref(h)))
            self.handle = h.value
            self._owned = True
        else:
            self.handle = _handle
            self._owned = False
        self._load_info()

    def _load_info(self):
        info = N.VolumeInfo()
        check(lib().clay_volume_get_info(self.handle, C.byref(info)))
        self.resolution = info.resolution
        self.mipLevels = info.mip_levels
        self.worldSize = info.world_size
        self.voxelSize = info.voxel_size
        self.band = info.band
        self.origin = tuple(info.origin)
        self.tileRes = self.resolution // 8
        self.tileResPerMip = [info.tile_res_per_mip[m] for m in range(self.mipLevels)]
        self.levelOffsets = [int(info.level_offset[m]) for m in range(self.mipLevels)]
        self.totalVoxels = int(info.total_voxels)
        self.totalCells = int(info.total_cells)
        off, self.cellOffsets = 0, []
        for t in self.tileResPerMip:
            self.cellOffsets.append(off)
            off += t ** 3

    def voxelSizeAt(self, mip: int) -> float:
        return self.voxelSize * 2 ** mip

    def setOrigin(self, origin):
        check(lib().clay_volume_set_origin(self.handle, *[float(x) for x in origin]))
        self.origin = tuple(float(x) for x in origin)

    def upload(self, dist_f16: np.ndarray | None = None, material_f16: np.ndarray | None = None, stream=None):
        """Writes whole planes (all levels) from host f16 arrays (uint16 bit patterns)."""
        d = None if dist_f16 is None else np.ascontiguousarray(dist_f16, np.uint16)
        m = None if material_f16 is None else np.ascontiguousarray(material_f16, np.uint16)
        for a in (d, m):
            if a is not None and a.size != self.totalVoxels:
                raise ValueError(f"plane has {a.size} values, the volume {self.totalVoxels}")
        check(lib().clay_volume_upload(self.handle, None if d is None else d.ctypes.data,
                                       None if m is None else m.ctypes.data, stream_handle(stream)))
        _sync(stream)

    def download(self, stream=None):
        d = np.zeros(self.totalVoxels, np.uint16)
        m = np.zeros(self.totalVoxels, np.uint16)
        check(lib().clay_volume_download(self.handle, d.ctypes.data, m.ctypes.data, stream_handle(stream)))
        _sync(stream)
        return d, m

    def level(self, plane: np.ndarray, mip: int) -> np.ndarray:
        r = self.resolution >> mip
        o = self.levelOffsets[mip]
        return plane[o:o + r ** 3].reshape(r, r, r)  # [z][y][x]

    def download_rgba16f(self, mip: int = 0) -> np.ndarray:
        r = self.resolution >> mip
        out = np.zeros(r ** 3 * 4, np.uint16)
        check(lib().clay_volume_download_rgba16f(self.handle, mip, out.ctypes.data, None))
        return out.reshape(r, r, r, 4)

    def build(self, brushes: np.ndarray, stream=None):
        """SdfBuilder.setBrushes + rebuild (builder.ts:147-172)."""
        b = np.ascontiguousarray(brushes)
        check(lib().clay_volume_build_brushes(self.handle, b.ctypes.data if len(b) else None, len(b),
                                              stream_handle(stream)))

    def destroy(self):
        if self._owned and self.handle:
            lib().clay_volume_destroy(self.handle)
        self.handle = None


def _sync(stream):
    import torch  # device plumbing only

    if stream is None or isinstance(stream, int):
        torch.cuda.synchronize()
    else:
        stream.synchronize()


class TracedField:
    """A collider (trace/field.ts:20-73): `volumeField`, `unionField`, `offsetField`."""

    def __init__(self, handle, owned=True, parts=()):
        self.handle = handle
        self._owned = owned
        self._parts = parts  # keep the volumes alive

    def query(self, points: np.ndarray):
        """(sample(p,0) as (x,y) pairs, normal(p)) at host points, evaluated on the device."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        s = np.zeros((len(pts), 2), np.float32)
        n = np.zeros((len(pts), 3), np.float32)
        check(lib().clay_field_query(self.handle, pts.ctypes.data, len(pts), s.ctypes.data, n.ctypes.data, None))
        return s, n

    def query_mip(self, points: np.ndarray, mip: int):
        """(sample(p, mip), field(p, mip)) as (x, y) pairs at host points, on the device."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        s = np.zeros((len(pts), 2), np.float32)
        f = np.zeros((len(pts), 2), np.float32)
        check(lib().clay_field_query_mip(self.handle, pts.ctypes.data, len(pts), int(mip), s.ctypes.data,
                                         f.ctypes.data, None))
        return s, f

    def query_mip_device(self, points, sample_xy, field_xy, mip: int, stream=None):
        """sample(p, mip) and field(p, mip) at device points into device (x, y) pairs: CUDA
        tensors (n x 3 and n x 2 float32), asynchronous on `stream`, nothing allocated."""
        import torch

        n = int(points.shape[0])
        for t, w in ((points, 3), (sample_xy, 2), (field_xy, 2)):
            if not t.is_cuda or t.dtype != torch.float32 or tuple(t.shape) != (n, w) or not t.is_contiguous():
                raise ValueError("query_mip_device: contiguous float32 CUDA tensors of n x 3, n x 2, n x 2")
        check(lib().clay_field_query_mip_device(self.handle, points.data_ptr(), n, int(mip), sample_xy.data_ptr(),
                                                field_xy.data_ptr(), stream_handle(stream)))

    def bandWorld(self, mip: int) -> float:
        return self._band_voxel(mip)[0]

    def voxelWorld(self, mip: int) -> float:
        return self._band_voxel(mip)[1]

    def _band_voxel(self, mip):
        b, v = C.c_float(), C.c_float()
        check(lib().clay_field_band_voxel(self.handle, int(mip), C.byref(b), C.byref(v)))
        return float(b.value), float(v.value)

    def setOffset(self, offset):
        check(lib().clay_field_set_offset(self.handle, *[float(x) for x in offset]))

    def destroy(self):
        if self._owned and self.handle:
            lib().clay_field_destroy(self.handle)
        self.handle = None


def volumeField(volume: SdfVolume) -> TracedField:
    h = C.c_void_p()
    check(lib().clay_field_from_volume(volume.handle, C.byref(h)))
    return TracedField(h.value, True, (volume,))


def unionField(a: TracedField, b: TracedField) -> TracedField:
    h = C.c_void_p()
    check(lib().clay_field_union(a.handle, b.handle, C.byref(h)))
    return TracedField(h.value, True, (a, b))


def offsetField(f: TracedField, offset) -> TracedField:
    h = C.c_void_p()
    check(lib().clay_field_offset(f.handle, *[float(x) for x in offset], C.byref(h)))
    return TracedField(h.value, True, (f,))


def motion_buffer(center=(0.0, 0.0, 0.0), velocity=(0.0, 0.0, 0.0)):
    """An ExtractMotion (extract.ts:30-45) as an 8-float CUDA tensor: centre, pad, velocity, pad."""
    import torch

    return torch.tensor([*center, 0.0, *velocity, 0.0], dtype=torch.float32, device="cuda")


def offsetFieldDevice(f: TracedField, device_offset) -> TracedField:
    """offsetField(f, () => offset) with the offset read on the device at every sample (3 floats
    at `device_offset`, a CUDA tensor or pointer that must outlive the field), e.g. the centre
    of an ExtractMotion."""
    h = C.c_void_p()
    check(lib().clay_field_offset_device(f.handle, _dev_ptr(device_offset), C.byref(h)))
    return TracedField(h.value, True, (f, device_offset))


def _dev_ptr(x) -> int:
    """A device pointer from a CUDA tensor or an int."""
    return int(x) if isinstance(x, int) else int(x.data_ptr())


class SurfaceExtractor:
    """`SurfaceExtractor` (sim/extract.ts:84-484): naive surface nets of `field`'s zero level
    set into a ParticleSet held by the caller as device memory: `particles` (96-byte Particle
    records, `set_capacity` of them) and `bodies` (64-byte Body records, `max_bodies`).
    `motion`: an optional caller-owned ExtractMotion (8 device floats: centre, pad, velocity,
    pad, e.g. a CUDA tensor made by `motion_buffer`)."""

    def __init__(self, root: Root, particles, set_capacity: int, bodies, max_bodies: int, field: TracedField,
                 body: int, base: int, capacity: int, resolution: int | None = None, motion=None):
        o = N.ExtractorOpts(body=int(body), base=int(base), capacity=int(capacity),
                            motion=None if motion is None else _dev_ptr(motion))
        if resolution is not None:
            o.set |= N.CLAY_EXTRACT_RESOLUTION
            o.resolution = int(resolution)
        h = C.c_void_p()
        check(lib().clay_extractor_create(root.handle, field.handle, _dev_ptr(particles), int(set_capacity),
                                          _dev_ptr(bodies), int(max_bodies), C.byref(o), C.byref(h)))
        self.handle = h.value
        self.root = root
        self.field = field
        self.resolution = 32 if resolution is None else int(resolution)
        self._keep = (particles, bodies, motion)
        idx, draw, qc = C.c_void_p(), C.c_void_p(), C.c_int64()
        check(lib().clay_extractor_views(self.handle, C.byref(idx), C.byref(draw), C.byref(qc)))
        self.indices_ptr, self.draw_args_ptr, self.quadCapacity = idx.value, draw.value, int(qc.value)

    def setRegion(self, origin, size: float, vel=(0.0, 0.0, 0.0), preserveMotion: bool = False):
        o = (C.c_double * 3)(*[float(x) for x in origin])
        v = (C.c_double * 3)(*[float(x) for x in vel])
        check(lib().clay_extractor_set_region(self.handle, o, float(size), v, 1 if preserveMotion else 0))

    def extract(self, pass_=None):
        check(lib().clay_extractor_extract(self.handle, stream_handle(pass_)))

    def counts(self, stream=None):
        """(dual vertices, quads) of the last extraction, before the capacity clamps."""
        out = np.zeros(2, np.uint32)
        check(lib().clay_extractor_read_counts_async(self.handle, out.ctypes.data, stream_handle(stream)))
        _sync(stream)
        return int(out[0]), int(out[1])

    def indices(self, stream=None):
        """(triangles as an (n, 3) uint32 array, draw arguments) of the last extraction."""
        idx = np.zeros(self.quadCapacity * 6, np.uint32)
        draw = np.zeros(4, np.uint32)
        check(lib().clay_extractor_read_indices_async(self.handle, idx.ctypes.data, draw.ctypes.data,
                                                      stream_handle(stream)))
        _sync(stream)
        return idx[: int(draw[0])].reshape(-1, 3), draw

    def destroy(self):
        if self.handle:
            lib().clay_extractor_destroy(self.handle)
        self.handle = None


class ClaySolver:
    """`ClaySolver` (sim/pbd.ts:78-424) over a ParticleSet held by the caller as device memory
    (96-byte Particle records and 64-byte Body records), colliding against `world`. Options by
    the reference's names: gravity, dt, substeps, radius, friction, damping, maxSpeed,
    rotationIterations."""

    def __init__(self, root: Root, particles, capacity: int, bodies, max_bodies: int, world: TracedField,
                 options: dict | None = None):
        o = N.SolverOpts()
        for key, val in (options or {}).items():
            if key not in N.SOLVER:
                raise ClayError(N.CLAY_EINVAL, f"ClaySolver: unknown option '{key}'")
            o.set |= N.SOLVER[key]
            if key == "gravity":
                o.gravity[:] = [float(x) for x in val]
            elif key in ("substeps", "rotationIterations"):
                setattr(o, "substeps" if key == "substeps" else "rotation_iterations", int(val))
            else:
                setattr(o, {"maxSpeed": "max_speed"}.get(key, key), float(val))
        h = C.c_void_p()
        check(lib().clay_solver_create(root.handle, world.handle, _dev_ptr(particles), int(capacity),
                                       _dev_ptr(bodies), int(max_bodies), C.byref(o), C.byref(h)))
        self.handle = h.value
        self.world = world
        self._keep = (particles, bodies)

    def setForce(self, body: int, accel, impulse=(0.0, 0.0, 0.0)):
        a = (C.c_double * 3)(*[float(x) for x in accel])
        i = (C.c_double * 3)(*[float(x) for x in impulse])
        check(lib().clay_solver_set_force(self.handle, int(body) & 0xFFFFFFFF, a, i))

    def step(self, body_count: int, pass_=None):
        check(lib().clay_solver_step(self.handle, int(body_count), stream_handle(pass_)))

    def destroy(self):
        if self.handle:
            lib().clay_solver_destroy(self.handle)
        self.handle = None


@dataclass
class ParticleCloud:
    """`ParticleCloud` (splat.ts:15-38) as device arrays.

    positions: CUDA tensor (or device pointer with ``stride``) holding float xyz at the start of
    each record. live: "all", ("count", u32 device tensor) or ("range", first, count tensors).
    normals: optional device float xyz per record; rotation: optional device xyzw quaternion
    applied to the normals (bodyCloud's `quatRotate(body.rot, restNormal)`).
    """

    capacity: int
    positions: object
    stride: int | None = None
    live: object = "all"
    normals: object = None
    normal_stride: int | None = None
    rotation: object = None

    def desc(self) -> N.CloudDesc:
        d = N.CloudDesc()
        d.capacity = int(self.capacity)
        d.positions, d.position_stride = _ptr_stride(self.positions, self.stride)
        if self.live == "all":
            d.live_mode = N.LIVE_ALL
        elif self.live[0] == "count":
            d.live_mode = N.LIVE_COUNT
            d.live_count = _ptr(self.live[1])
        elif self.live[0] == "range":
            d.live_mode = N.LIVE_RANGE
            d.live_first = _ptr(self.live[1])
            d.live_range_count = _ptr(self.live[2])
        else:
            raise ValueError(f"unknown live rule {self.live!r}")
        if self.normals is not None:
            d.normals, d.normal_stride = _ptr_stride(self.normals, self.normal_stride)
        if self.rotation is not None:
            d.rotation = _ptr(self.rotation)
        return d


def _ptr(t) -> int:
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise ValueError("cloud arrays must live on the device")
    return int(t.data_ptr())


def _ptr_stride(t, stride):
    if isinstance(t, int):
        if stride is None:
            raise ValueError("a raw pointer needs an explicit stride")
        return t, int(stride)
    p = _ptr(t)
    if stride is None:
        stride = t.stride(0) * t.element_size() if t.dim() >= 2 else 12
    return p, int(stride)


PARTICLE_RECORD_BYTES = 96  # `Particle` (lib/src/sim/particles.ts:18-34)
BODY_RECORD_BYTES = 64      # `Body` (particles.ts:52-68)


def bodyCloud(particles, bodies, body: int) -> ParticleCloud:
    """`bodyCloud(set, body)` (splat.ts:47-72) over device buffers laid out as the reference's
    `Particle` (96 B: pos@0, restNormal@80) and `Body` (64 B: first@12, rot@16, count@44)
    records: live = first <= i < first + count, normal = quatRotate(body.rot, restNormal)."""
    pbase = _ptr(particles)
    bbase = _ptr(bodies) + body * BODY_RECORD_BYTES
    cap = particles.numel() * particles.element_size() // PARTICLE_RECORD_BYTES
    return ParticleCloud(capacity=cap, positions=pbase, stride=PARTICLE_RECORD_BYTES,
                         live=("range", bbase + 12, bbase + 44), normals=pbase + 80,
                         normal_stride=PARTICLE_RECORD_BYTES, rotation=bbase + 16)


class SplatField:
    """`SplatField` (splat.ts:136-309)."""

    def __init__(self, root: Root, cloud: ParticleCloud | None, radius=None, material=None, resolution=None,
                 mipLevels=None, band=None, origin=None, worldSize=None, label=None, _handle=None):
        self.root = root
        self.cloud = cloud
        if _handle is None:
            if radius is None:
                raise ClayError(N.CLAY_EINVAL, "SplatField: `radius` is required")
            o = N.SplatOpts()
            o.radius = float(radius)
            for key, val in (("material", material), ("resolution", resolution), ("mipLevels", mipLevels),
                             ("band", band), ("origin", origin), ("worldSize", worldSize)):
                if val is None:
                    continue
                o.set |= N.SPLAT[key]
                if key == "origin":
                    o.origin[:] = [float(x) for x in val]
                elif key == "mipLevels":
                    o.mip_levels = int(val)
                elif key == "worldSize":
                    o.world_size = float(val)
                else:
                    setattr(o, key, val)
            desc = cloud.desc()
            h = C.c_void_p()
            check(lib().clay_splat_create(root.handle, C.byref(desc), C.byref(o), C.byref(h)))
            self.handle = h.value
            self._owned = True
        else:
            self.handle = _handle
            self._owned = False
        self.volume = SdfVolume(root, _handle=lib().clay_splat_volume(self.handle))
        self.field = TracedField(lib().clay_splat_field(self.handle), owned=False, parts=(self,))

    def setCenter(self, center):
        check(lib().clay_splat_set_center(self.handle, *[float(x) for x in center]))
        half = self.volume.worldSize / 2
        self.volume.origin = tuple(float(c) - half for c in center)

    def bake(self, pass_=None):
        check(lib().clay_splat_bake(self.handle, stream_handle(pass_)))

    def census(self, pass_=None) -> int:
        """Measurement hook: the (particle, voxel) pairs a bake of the cloud as it is now lowers."""
        v = C.c_uint64()
        check(lib().clay_splat_census(self.handle, stream_handle(pass_), C.byref(v)))
        return int(v.value)

    def capture_keys(self, keys_device):
        """Test hook: subsequent bakes copy their 16-bit keys into `keys_device` (u32 tensor)."""
        check(lib().clay_splat_capture_keys(self.handle, None if keys_device is None else _ptr(keys_device)))

    def destroy(self):
        if self._owned and self.handle:
            lib().clay_splat_destroy(self.handle)
        self.handle = None


_FLUID_OPT_KEYS = ("capacity", "spacing", "smoothing", "bucket", "radius", "surfaceRadius", "material",
                   "bakeResolution", "bakeMipLevels", "bakeBand", "origin", "worldSize", "substeps",
                   "gravity", "stiffness", "viscosity", "damping", "maxSpeed")
_FLUID_FIELD = {"surfaceRadius": "surface_radius", "bakeResolution": "bake_resolution",
                "bakeMipLevels": "bake_mip_levels", "bakeBand": "bake_band", "worldSize": "world_size",
                "maxSpeed": "max_speed"}
_PARAM_FIELD = {"gravity": "gravity", "dt": "dt", "emitPos": "emit_pos", "emitRadius": "emit_radius",
                "emitVel": "emit_vel", "maxSpeed": "max_speed", "stiffness": "stiffness",
                "viscosity": "viscosity", "damping": "damping", "contactDepth": "contact_depth"}


class FluidSim:
    """`FluidSim` (fluid.ts:111-582)."""

    def __init__(self, root: Root, world: TracedField | None, options: dict | None = None, _handle=None, **kw):
        self.owned = _handle is None
        if _handle is None:
            o = fluid_options(options, **kw)
            h = C.c_void_p()
            check(lib().clay_fluid_create(root.handle, None if world is None else world.handle, C.byref(o),
                                          C.byref(h)))
            self.handle = h.value
        else:
            self.handle = _handle
        self.root = root
        self.world = world
        info = N.FluidInfo()
        check(lib().clay_fluid_get_info(self.handle, C.byref(info)))
        self.capacity = int(info.capacity)
        self.substeps = int(info.substeps)
        self.spacing = float(info.spacing)
        self.info = info
        self.surface = SplatField(root, None, _handle=lib().clay_fluid_surface(self.handle))
        self.field = self.surface.field
        self._contacts = N.ContactList()

    # -- the reference's surface ----------------------------------------------------------
    @property
    def particleCount(self) -> int:
        return int(lib().clay_fluid_particle_count(self.handle))

    def spawn(self, n: int, pos, vel, spread: float | None = None):
        p = (C.c_double * 3)(*[float(x) for x in pos])
        v = (C.c_double * 3)(*[float(x) for x in vel])
        sp = None if spread is None else C.byref(C.c_double(float(spread)))
        check(lib().clay_fluid_spawn(self.handle, int(n), p, v, sp))

    def configure(self, patch: dict):
        q = N.FluidParams()
        mask = 0
        for key, val in patch.items():
            if key in ("count", "emitBase", "emitCount", "emitSeed"):
                raise ClayError(N.CLAY_EINVAL, f"FluidSim.configure: '{key}' is not configurable")
            if key not in _PARAM_FIELD:
                raise ClayError(N.CLAY_EINVAL, f"FluidSim.configure: unknown parameter '{key}'")
            mask |= N.PARAM[key]
            name = _PARAM_FIELD[key]
            if key in ("gravity", "emitPos", "emitVel"):
                getattr(q, name)[:] = [float(x) for x in val]
            else:
                setattr(q, name, float(val))
        check(lib().clay_fluid_configure(self.handle, C.byref(q), mask))

    def step(self, pass_=None):
        check(lib().clay_fluid_step(self.handle, stream_handle(pass_)))

    @property
    def params(self) -> dict:
        q = N.FluidParams()
        check(lib().clay_fluid_get_params(self.handle, C.byref(q)))
        return {"gravity": tuple(q.gravity), "dt": q.dt, "emitPos": tuple(q.emit_pos),
                "emitRadius": q.emit_radius, "emitVel": tuple(q.emit_vel), "maxSpeed": q.max_speed,
                "stiffness": q.stiffness, "viscosity": q.viscosity, "damping": q.damping,
                "count": q.count, "emitBase": q.emit_base, "emitCount": q.emit_count,
                "emitSeed": q.emit_seed, "contactDepth": q.contact_depth}

    def readContacts(self, pass_=None):
        """`readContacts` (fluid.ts:565-569): [(x, y, z, speed)] of up to 32 contacts."""
        check(lib().clay_fluid_read_contacts_async(self.handle, C.byref(self._contacts), stream_handle(pass_)))
        _sync(pass_)
        n = min(int(self._contacts.count), 32)
        return [tuple(self._contacts.points[i]) for i in range(n)], int(self._contacts.count)

    def set_mode(self, mode: str):
        check(lib().clay_fluid_set_mode(self.handle, N.MODE_REFERENCE if mode == "reference" else N.MODE_FAST))

    # -- device data and test hooks ---------------------------------------------------------
    def particles_ptr(self):
        p = C.c_void_p()
        s = C.c_uint32()
        check(lib().clay_fluid_particles_device(self.handle, C.byref(p), C.byref(s)))
        return p.value, s.value

    def upload(self, parts: np.ndarray, stream=None):
        a = np.ascontiguousarray(parts, PARTICLE_DTYPE)
        check(lib().clay_fluid_upload(self.handle, a.ctypes.data if len(a) else None, len(a), stream_handle(stream)))
        _sync(stream)

    def download(self, count: int | None = None, stream=None) -> np.ndarray:
        n = self.particleCount if count is None else count
        out = np.zeros(n, PARTICLE_DTYPE)
        check(lib().clay_fluid_download(self.handle, out.ctypes.data if n else None, n, stream_handle(stream)))
        _sync(stream)
        return out

    def census(self, stream=None) -> dict:
        """Measurement hook: the algorithmic work of the last frame (neighbour candidates and
        accepted pairs of its last substep, the bake's in-band (particle, voxel) pairs)."""
        c = N.Census()
        check(lib().clay_fluid_census(self.handle, stream_handle(stream), C.byref(c)))
        return {k: int(getattr(c, k)) for k, _ in N.Census._fields_}

    def cell_indices(self) -> np.ndarray:
        """Test hook: the reference's cellIndex of every live particle (0xffffffff outside)."""
        out = np.zeros(max(self.particleCount, 1), np.uint32)
        check(lib().clay_fluid_cell_indices(self.handle, out.ctypes.data, None))
        return out[: self.particleCount]

    def destroy(self):
        if self.handle and self.owned:
            lib().clay_fluid_destroy(self.handle)
        self.handle = None


def fluid_options(options: dict | None = None, **kw) -> N.FluidOpts:
    """`FluidSimOptions` (fluid.ts:60-108) as the C ABI takes them: a field per option and a
    bit per option that is set, so unset ones resolve to the reference's defaults."""
    opts = dict(options or {})
    opts.update(kw)
    o = N.FluidOpts()
    for key, val in opts.items():
        if key == "label":
            continue
        if key not in _FLUID_OPT_KEYS:
            raise ClayError(N.CLAY_EINVAL, f"FluidSim: unknown option '{key}'")
        if val is None:
            continue
        o.set |= N.FLUID[key]
        name = _FLUID_FIELD.get(key, key)
        if key in ("origin", "gravity"):
            getattr(o, name)[:] = [float(x) for x in val]
        elif key in ("capacity", "bucket", "bakeResolution", "bakeMipLevels", "substeps"):
            setattr(o, name, int(val))
        else:
            setattr(o, name, float(val))
    return o


def fluid_estimate_bytes(options: dict | None = None, **kw) -> int:
    """Device bytes a FluidSim with these options allocates (its surface included)."""
    out = C.c_uint64()
    check(lib().clay_fluid_estimate_bytes(C.byref(fluid_options(options, **kw)), C.byref(out)))
    return int(out.value)


class Batch:
    """Independent FluidSims advanced one frame each per call, in one launch sequence captured
    into a CUDA graph (no reference counterpart)."""

    def __init__(self, root: Root, sims, extra_splats=(), sph_block=256, use_graph=True):
        arr = (C.c_void_p * len(sims))(*[s.handle for s in sims])
        h = C.c_void_p()
        check(lib().clay_batch_create(root.handle, arr, len(sims), C.byref(h)))
        self.handle = h.value
        self.sims = list(sims)
        self.extra = list(extra_splats)
        for s in self.extra:
            check(lib().clay_batch_add_splat(self.handle, s.handle))
        self.set_tuning(sph_block=sph_block, use_graph=use_graph)

    def set_tuning(self, sph_block=256, use_graph=True):
        t = N.BatchTuning(int(sph_block), 256, 1 if use_graph else 0)
        check(lib().clay_batch_set_tuning(self.handle, C.byref(t)))

    def set_bucket_blocks(self, uppers, blocks):
        """Thread-block size of the particle passes per scene-size bucket (capacity < upper)."""
        u = (C.c_int64 * len(uppers))(*[int(x) for x in uppers])
        b = (C.c_int32 * len(blocks))(*[int(x) for x in blocks])
        check(lib().clay_batch_set_bucket_blocks(self.handle, u, b, len(uppers)))

    def set_bucket_tuning(self, uppers, tunings):
        """Per scene-size bucket settings: `tunings` has len(uppers) + 1 dicts (the last for the
        scenes above every bound) with keys sph_block, density_variant, splat_tile_ratio,
        splat_walk_weight and forces_split."""
        u = (C.c_int64 * max(len(uppers), 1))(*[int(x) for x in uppers])
        t = (N.BucketTuning * len(tunings))()
        for i, d in enumerate(tunings):
            t[i] = N.BucketTuning(int(d["sph_block"]), int(d["density_variant"]), int(d["splat_tile_ratio"]),
                                  int(d["splat_walk_weight"]), int(d.get("forces_split", 0)))
        check(lib().clay_batch_set_bucket_tuning(self.handle, u, t, len(uppers)))

    def set_lanes(self, lanes: int):
        """Step the scenes as `lanes` groups whose passes run side by side (same results)."""
        check(lib().clay_batch_set_lanes(self.handle, int(lanes)))

    def step(self, pass_=None):
        check(lib().clay_batch_step(self.handle, stream_handle(pass_)))

    def step_subset(self, scenes, pass_=None):
        """One frame for the listed scenes only (indices into this batch, each at most once)."""
        arr = (C.c_int32 * len(scenes))(*[int(i) for i in scenes])
        check(lib().clay_batch_step_subset(self.handle, arr, len(scenes), stream_handle(pass_)))

    def read_contacts_async(self, host_ptr: int, pass_=None):
        """Every scene's ContactList into pinned host memory at `host_ptr` (528 B each)."""
        check(lib().clay_batch_read_contacts_async(self.handle, host_ptr, stream_handle(pass_)))

    def profile(self, pass_=None) -> dict:
        """One un-graphed frame with CUDA events around every kernel: {name: (ms, launches)}."""
        out = (N.PhaseTime * 64)()
        n = C.c_int()
        check(lib().clay_batch_profile(self.handle, stream_handle(pass_), out, 64, C.byref(n)))
        return {out[i].name.decode(): (float(out[i].ms), int(out[i].launches)) for i in range(n.value)}

    def launches_per_step(self) -> int:
        v = C.c_int64()
        check(lib().clay_batch_launches_per_step(self.handle, C.byref(v)))
        return int(v.value)

    def destroy(self):
        if self.handle:
            lib().clay_batch_destroy(self.handle)
        self.handle = None


def kernel_launch_count() -> int:
    return int(lib().clay_kernel_launch_count())
