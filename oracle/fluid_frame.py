"""`FluidSim` host bookkeeping (lib/src/sim/fluid.ts:140-558) driven over the oracle's f32
passes. TEST INFRASTRUCTURE: the CPU side of the parity tests that step a fluid, and the
CPU baseline of the benchmark."""
from __future__ import annotations

import math

import numpy as np


class OracleFluid:
    def __init__(self, oracle, world_volumes, capacity=8192, spacing=0.45, smoothing=None, bucket=64,
                 radius=None, surfaceRadius=None, material=0.0, bakeResolution=64, bakeMipLevels=None,
                 bakeBand=2.0, origin=(-12.0, -4.0, -12.0), worldSize=24.0, substeps=3,
                 gravity=(0.0, -9.81, 0.0), stiffness=220.0, viscosity=0.4, damping=0.995, maxSpeed=15.0,
                 offsets=None, threads=8):
        self.o = oracle
        self.threads = threads
        h = smoothing if smoothing is not None else spacing * 2.2
        self.radius = radius if radius is not None else spacing * 0.5
        surf = surfaceRadius if surfaceRadius is not None else spacing * 1.1
        mips = bakeMipLevels if bakeMipLevels is not None else max(1, int(math.log2(bakeResolution / 8)))
        self.capacity, self.spacing, self.substeps = capacity, spacing, substeps
        self.cfg = oracle.fluid_cfg(capacity=capacity, bucket=bucket, spacing=spacing, h=h, radius=self.radius,
                                    surface_radius=surf, material=material, bake_res=bakeResolution,
                                    bake_mips=mips, bake_band=bakeBand, origin=tuple(origin),
                                    world_size=worldSize, substeps=substeps)
        self.splat = oracle.splat_cfg(bakeResolution, mips, bakeBand, surf, world_size=worldSize,
                                      material=material, origin=tuple(origin))
        self.volumes = list(world_volumes)
        self.field = oracle.make_field(self.volumes, offsets) if self.volumes else None
        self.parts = np.zeros(capacity, oracle.PARTICLE_DTYPE)
        self.live = self.cursor = self.pending = 0
        self.seed = 1
        self.frozen = dict(gravity=[float(np.float32(g)) for g in gravity], dt=1 / 60 / substeps,
                           emit_pos=[0.0, 0.0, 0.0], emit_radius=spacing, emit_vel=[0.0, 0.0, 0.0],
                           max_speed=maxSpeed, stiffness=stiffness, viscosity=viscosity, damping=damping,
                           emit_seed=1, contact_depth=self.radius * 1.5)
        self.contacts = (0, np.zeros((32, 4), np.float32), np.zeros(0, np.uint32))
        self.keys = None

    def upload(self, parts):
        n = len(parts)
        self.parts[:n] = parts
        self.live, self.cursor, self.pending = n, n % self.capacity, 0

    def spawn(self, n, pos, vel, spread=None):
        if spread is None:
            spread = self.spacing * (max(n, 1) ** (1 / 3)) * 0.62
        self.pending = max(0, min(n, self.capacity))
        self.frozen.update(emit_pos=list(pos), emit_vel=list(vel), emit_radius=spread, emit_seed=self.seed)
        self.seed += 1

    def configure(self, **patch):
        self.frozen.update(patch)

    def step(self):
        ec, self.pending = self.pending, 0
        base = self.cursor
        if ec > 0:
            self.cursor = (base + ec) % self.capacity
            self.live = min(self.capacity, max(self.live, base + ec))
        prm = self.o.params_from(dict(self.frozen, count=self.live, emit_base=base, emit_count=ec))
        if ec > 0:
            self.o.fluid_emit(self.cfg, prm, self.parts)
        s = 0
        while s < self.substeps and self.live > 0:
            self.contacts = self.o.fluid_substep_f32(self.cfg, prm, self.field, self.parts, threads=self.threads)
            s += 1
        cloud = self.o.CloudData(self.parts["pos"].copy(), live_mode=1, live_a=self.live)
        self.keys = self.o.splat_keys(self.splat, cloud, threads=self.threads)
        self.prm = prm
        return self.keys
