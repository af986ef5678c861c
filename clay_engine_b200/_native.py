"""ctypes binding of ``libclayfluid.so`` (declared in ``include/clay_fluid.h``).

There is no fallback: if the library is missing or fails to load, importing the host API
raises, so nothing can silently run without the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libclayfluid.so")


class ClayError(RuntimeError):
    """An error reported by the library (the reference throws `Error` in these cases)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


CLAY_OK, CLAY_EINVAL, CLAY_ECUDA, CLAY_ENOMEM, CLAY_ESTATE, CLAY_ETIMEOUT = 0, -1, -2, -3, -4, -5

# option bits (include/clay_fluid.h)
VOL = dict(resolution=1 << 0, worldSize=1 << 1, origin=1 << 2, mipLevels=1 << 3, band=1 << 4,
           gradientVoxels=1 << 5)
SPLAT = dict(material=1 << 0, resolution=1 << 1, mipLevels=1 << 2, band=1 << 3, origin=1 << 4,
             worldSize=1 << 5)
FLUID = dict(capacity=1 << 0, spacing=1 << 1, smoothing=1 << 2, bucket=1 << 3, radius=1 << 4,
             surfaceRadius=1 << 5, material=1 << 6, bakeResolution=1 << 7, bakeMipLevels=1 << 8,
             bakeBand=1 << 9, origin=1 << 10, worldSize=1 << 11, substeps=1 << 12,
             gravity=1 << 13, stiffness=1 << 14, viscosity=1 << 15, damping=1 << 16,
             maxSpeed=1 << 17)
PARAM = dict(gravity=1 << 0, dt=1 << 1, emitPos=1 << 2, emitRadius=1 << 3, emitVel=1 << 4,
             maxSpeed=1 << 5, stiffness=1 << 6, viscosity=1 << 7, damping=1 << 8,
             contactDepth=1 << 9)
LIVE_ALL, LIVE_COUNT, LIVE_RANGE = 0, 1, 2
MODE_FAST, MODE_REFERENCE = 0, 1


class VolumeOpts(C.Structure):
    _fields_ = [("set", C.c_uint32), ("resolution", C.c_int32), ("world_size", C.c_double),
                ("origin", C.c_double * 3), ("mip_levels", C.c_int32), ("band", C.c_double),
                ("gradient_voxels", C.c_double)]


class VolumeInfo(C.Structure):
    _fields_ = [("resolution", C.c_int32), ("mip_levels", C.c_int32), ("world_size", C.c_double),
                ("voxel_size", C.c_double), ("band", C.c_double), ("origin", C.c_double * 3),
                ("tile_res_per_mip", C.c_int32 * 16), ("level_offset", C.c_int64 * 16),
                ("total_voxels", C.c_int64), ("total_cells", C.c_int32)]


class Brush(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("scale", C.c_float), ("rot", C.c_float * 4),
                ("size", C.c_float * 3), ("radius", C.c_float), ("material", C.c_float),
                ("blend", C.c_float), ("bound", C.c_float), ("mask", C.c_float),
                ("kind", C.c_uint32), ("op", C.c_uint32), ("slot", C.c_uint32), ("pad", C.c_uint32)]


class CloudDesc(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("positions", C.c_void_p), ("position_stride", C.c_uint32),
                ("live_mode", C.c_uint32), ("live_count", C.c_void_p), ("live_first", C.c_void_p),
                ("live_range_count", C.c_void_p), ("normals", C.c_void_p), ("normal_stride", C.c_uint32),
                ("rotation", C.c_void_p)]


class BucketTuning(C.Structure):
    _fields_ = [("sph_block", C.c_int32), ("density_variant", C.c_int32), ("splat_tile_ratio", C.c_int32),
                ("splat_walk_weight", C.c_int32), ("forces_split", C.c_int32)]


class Census(C.Structure):
    _fields_ = [("particles", C.c_uint64), ("candidates", C.c_uint64), ("accepted", C.c_uint64),
                ("splat_pairs", C.c_uint64)]


class SplatOpts(C.Structure):
    _fields_ = [("set", C.c_uint32), ("radius", C.c_double), ("material", C.c_double),
                ("resolution", C.c_int32), ("mip_levels", C.c_int32), ("band", C.c_double),
                ("origin", C.c_double * 3), ("world_size", C.c_double)]


class FluidOpts(C.Structure):
    _fields_ = [("set", C.c_uint32), ("capacity", C.c_int64), ("spacing", C.c_double),
                ("smoothing", C.c_double), ("bucket", C.c_int32), ("radius", C.c_double),
                ("surface_radius", C.c_double), ("material", C.c_double),
                ("bake_resolution", C.c_int32), ("bake_mip_levels", C.c_int32),
                ("bake_band", C.c_double), ("origin", C.c_double * 3), ("world_size", C.c_double),
                ("substeps", C.c_int32), ("gravity", C.c_double * 3), ("stiffness", C.c_double),
                ("viscosity", C.c_double), ("damping", C.c_double), ("max_speed", C.c_double)]


class FluidParams(C.Structure):
    _fields_ = [("gravity", C.c_float * 3), ("dt", C.c_float), ("emit_pos", C.c_float * 3),
                ("emit_radius", C.c_float), ("emit_vel", C.c_float * 3), ("max_speed", C.c_float),
                ("stiffness", C.c_float), ("viscosity", C.c_float), ("damping", C.c_float),
                ("count", C.c_uint32), ("emit_base", C.c_uint32), ("emit_count", C.c_uint32),
                ("emit_seed", C.c_uint32), ("contact_depth", C.c_float)]


class ContactList(C.Structure):
    _fields_ = [("count", C.c_uint32), ("pad", C.c_uint32 * 3), ("points", (C.c_float * 4) * 32)]


class FluidInfo(C.Structure):
    _fields_ = [("capacity", C.c_int64), ("substeps", C.c_int32), ("bucket", C.c_int32),
                ("grid_res", C.c_int32), ("smoothing", C.c_double), ("rest_density", C.c_double),
                ("grid_origin", C.c_double * 3), ("spacing", C.c_double), ("radius", C.c_double),
                ("device_bytes", C.c_uint64)]


class PhaseTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("ms", C.c_float), ("launches", C.c_int32)]


class BatchTuning(C.Structure):
    _fields_ = [("sph_block", C.c_int32), ("splat_block", C.c_int32), ("use_graph", C.c_int32)]


class ExtractorOpts(C.Structure):
    _fields_ = [("set", C.c_uint32), ("resolution", C.c_int32), ("body", C.c_int32), ("base", C.c_int32),
                ("capacity", C.c_int32), ("pad", C.c_int32), ("motion", C.c_void_p)]


CLAY_EXTRACT_RESOLUTION = 1


class SolverOpts(C.Structure):
    _fields_ = [("set", C.c_uint32), ("substeps", C.c_int32), ("gravity", C.c_double * 3), ("dt", C.c_double),
                ("radius", C.c_double), ("friction", C.c_double), ("damping", C.c_double), ("max_speed", C.c_double),
                ("rotation_iterations", C.c_int32), ("pad", C.c_int32)]


SOLVER = {"gravity": 1, "dt": 2, "substeps": 4, "radius": 8, "friction": 16, "damping": 32, "maxSpeed": 64,
          "rotationIterations": 128}


class ServerOpts(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("depth", C.c_int32), ("max_batch", C.c_int32),
                ("mode", C.c_int32), ("sph_block", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("frames", C.c_int64),
                ("scene_frames", C.c_int64), ("particle_steps", C.c_int64), ("admissions", C.c_int64),
                ("evictions", C.c_int64), ("resident_bytes", C.c_uint64), ("resident_scenes", C.c_int32),
                ("inflight", C.c_int32)]


P = C.c_void_p
I = C.c_int
D = C.c_double
# name -> (restype, argtypes); every function of include/clay_fluid.h.
SIGNATURES = {
    "clay_last_error": (C.c_char_p, []),
    "clay_version": (C.c_char_p, []),
    "clay_ctx_create": (I, [I, C.POINTER(P)]),
    "clay_ctx_destroy": (None, [P]),
    "clay_ctx_bytes_in_use": (I, [P, C.POINTER(C.c_uint64)]),
    "clay_volume_create": (I, [P, C.POINTER(VolumeOpts), C.POINTER(P)]),
    "clay_volume_destroy": (None, [P]),
    "clay_volume_get_info": (I, [P, C.POINTER(VolumeInfo)]),
    "clay_volume_set_origin": (I, [P, D, D, D]),
    "clay_volume_voxel_size_at": (D, [P, I]),
    "clay_volume_device_planes": (I, [P, C.POINTER(P), C.POINTER(P)]),
    "clay_volume_upload": (I, [P, P, P, P]),
    "clay_volume_download": (I, [P, P, P, P]),
    "clay_volume_download_rgba16f": (I, [P, I, P, P]),
    "clay_volume_build_brushes": (I, [P, P, I, P]),
    "clay_field_from_volume": (I, [P, C.POINTER(P)]),
    "clay_field_union": (I, [P, P, C.POINTER(P)]),
    "clay_field_offset": (I, [P, D, D, D, C.POINTER(P)]),
    "clay_field_set_offset": (I, [P, D, D, D]),
    "clay_field_destroy": (None, [P]),
    "clay_field_query": (I, [P, P, I, P, P, P]),
    "clay_field_query_mip": (I, [P, P, I, I, P, P, P]),
    "clay_field_query_mip_device": (I, [P, P, I, I, P, P, P]),
    "clay_field_band_voxel": (I, [P, I, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "clay_splat_create": (I, [P, C.POINTER(CloudDesc), C.POINTER(SplatOpts), C.POINTER(P)]),
    "clay_splat_destroy": (None, [P]),
    "clay_splat_set_center": (I, [P, D, D, D]),
    "clay_splat_bake": (I, [P, P]),
    "clay_splat_volume": (P, [P]),
    "clay_splat_field": (P, [P]),
    "clay_splat_capture_keys": (I, [P, P]),
    "clay_splat_bake_static": (I, [C.POINTER(CloudDesc), C.POINTER(SplatOpts), P, P, P]),
    "clay_fluid_create": (I, [P, P, C.POINTER(FluidOpts), C.POINTER(P)]),
    "clay_fluid_destroy": (None, [P]),
    "clay_fluid_set_mode": (I, [P, I]),
    "clay_fluid_spawn": (I, [P, C.c_int64, C.POINTER(D), C.POINTER(D), C.POINTER(D)]),
    "clay_fluid_configure": (I, [P, C.POINTER(FluidParams), C.c_uint32]),
    "clay_fluid_step": (I, [P, P]),
    "clay_fluid_particle_count": (C.c_int64, [P]),
    "clay_fluid_get_params": (I, [P, C.POINTER(FluidParams)]),
    "clay_fluid_read_contacts_async": (I, [P, P, P]),
    "clay_fluid_particles_device": (I, [P, C.POINTER(P), C.POINTER(C.c_uint32)]),
    "clay_fluid_upload": (I, [P, P, C.c_int64, P]),
    "clay_fluid_download": (I, [P, P, C.c_int64, P]),
    "clay_fluid_cell_indices": (I, [P, P, P]),
    "clay_fluid_census": (I, [P, P, C.POINTER(Census)]),
    "clay_splat_census": (I, [P, P, C.POINTER(C.c_uint64)]),
    "clay_fluid_surface": (P, [P]),
    "clay_fluid_field": (P, [P]),
    "clay_fluid_get_info": (I, [P, C.POINTER(FluidInfo)]),
    "clay_batch_create": (I, [P, P, I, C.POINTER(P)]),
    "clay_batch_destroy": (None, [P]),
    "clay_batch_add_splat": (I, [P, P]),
    "clay_batch_set_tuning": (I, [P, C.POINTER(BatchTuning)]),
    "clay_batch_get_tuning": (I, [P, C.POINTER(BatchTuning)]),
    "clay_batch_set_bucket_blocks": (I, [P, P, P, I]),
    "clay_batch_set_bucket_tuning": (I, [P, P, P, I]),
    "clay_batch_set_lanes": (I, [P, I]),
    "clay_batch_step": (I, [P, P]),
    "clay_batch_step_subset": (I, [P, P, I, P]),
    "clay_batch_read_contacts_async": (I, [P, P, P]),
    "clay_batch_profile": (I, [P, P, C.POINTER(PhaseTime), I, C.POINTER(C.c_int)]),
    "clay_batch_launches_per_step": (I, [P, C.POINTER(C.c_int64)]),
    "clay_server_create": (I, [P, C.POINTER(ServerOpts), P, C.POINTER(P)]),
    "clay_server_destroy": (None, [P]),
    "clay_server_add_scene": (I, [P, P, C.POINTER(FluidOpts), P, C.c_int64, C.POINTER(C.c_int32)]),
    "clay_server_submit": (I, [P, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    "clay_server_pump": (I, [P, C.POINTER(C.c_int32)]),
    "clay_server_wait": (I, [P, D]),
    "clay_server_drain": (I, [P]),
    "clay_server_poll": (I, [P, C.c_int64, C.POINTER(C.c_int32), C.POINTER(D)]),
    "clay_server_get_stats": (I, [P, C.POINTER(ServerStats)]),
    "clay_server_scene_sim": (I, [P, C.c_int32, C.POINTER(P)]),
    "clay_server_download": (I, [P, C.c_int32, P, C.c_int64, C.POINTER(C.c_int64)]),
    "clay_fluid_estimate_bytes": (I, [C.POINTER(FluidOpts), C.POINTER(C.c_uint64)]),
    "clay_extractor_create": (I, [P, P, P, C.c_int64, P, C.c_int32, C.POINTER(ExtractorOpts), C.POINTER(P)]),
    "clay_extractor_destroy": (None, [P]),
    "clay_extractor_set_region": (I, [P, C.POINTER(D), D, C.POINTER(D), I]),
    "clay_extractor_extract": (I, [P, P]),
    "clay_extractor_views": (I, [P, C.POINTER(P), C.POINTER(P), C.POINTER(C.c_int64)]),
    "clay_extractor_read_counts_async": (I, [P, P, P]),
    "clay_extractor_read_indices_async": (I, [P, P, P, P]),
    "clay_field_offset_device": (I, [P, P, C.POINTER(P)]),
    "clay_solver_create": (I, [P, P, P, C.c_int64, P, C.c_int32, C.POINTER(SolverOpts), C.POINTER(P)]),
    "clay_solver_destroy": (None, [P]),
    "clay_solver_set_force": (I, [P, C.c_uint32, C.POINTER(D), C.POINTER(D)]),
    "clay_solver_step": (I, [P, C.c_int32, P]),
    "clay_kernel_launch_count": (C.c_uint64, []),
}

_lib = None


def lib() -> C.CDLL:
    """Loads the library (raising if it is absent) and declares every entry point."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m clay_engine_b200.build` "
                "(the fluid path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != CLAY_OK:
        msg = lib().clay_last_error().decode(errors="replace")
        raise ClayError(rc, msg)


def stream_handle(s) -> int | None:
    """A CUDA stream as the library takes it: None / 0 (legacy default), an int handle, or a
    torch.cuda.Stream (its ``cuda_stream``)."""
    if s is None:
        return None
    if isinstance(s, int):
        return s or None
    h = getattr(s, "cuda_stream", None)
    if h is not None:
        return int(h) or None
    raise TypeError(f"not a CUDA stream: {s!r}")
