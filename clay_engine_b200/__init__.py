"""clay_engine_b200: a B200-native (sm_100a) implementation of clay-engine's per-frame fluid
hot path - the SPH step of `FluidSim` followed by the `SplatField` bake - behind the
reference's `FluidSim` / `SplatField` / `ParticleCloud` / `SdfVolume` surface.

The compute runs in ``_build/libclayfluid.so`` (C ABI: ``include/clay_fluid.h``); this
package is the host-side mirror of the reference's classes. There is no CPU fallback.
"""
from ._native import ClayError
from .core import (PARTICLE_DTYPE, Batch, ClaySolver, FluidSim, ParticleCloud, Root, SdfVolume, SplatField, SurfaceExtractor,
                   TracedField,
                   bodyCloud, init, kernel_launch_count, motion_buffer, offsetField, offsetFieldDevice, unionField,
                   volumeField)

__all__ = ["ClayError", "PARTICLE_DTYPE", "Batch", "ClaySolver", "FluidSim", "ParticleCloud", "Root", "SdfVolume",
           "SplatField", "SurfaceExtractor", "TracedField", "bodyCloud", "init", "kernel_launch_count", "motion_buffer", "offsetField", "offsetFieldDevice",
           "unionField", "volumeField"]
