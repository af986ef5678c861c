"""The census hooks the benchmark's compute roofline reads (clay_fluid_census,
clay_splat_census) count exactly the reference's work: checked against brute-force counts in
numpy with the same f32 arithmetic on a 4,096-particle blob.

- candidates: the particles in the 27 cells around each particle's cell (fluid.ts:346-364);
- accepted: of them, those with (dx*dx + dy*dy) + dz*dz < h^2 (fluid.ts:357), self included;
- splat pairs: (particle, voxel) pairs inside the particle's voxel box with
  length(c - p) - radius < bandWorld (splat.ts:238-249), over every level.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORIGIN = (-12.0, -4.0, -12.0)
f32 = np.float32


def brute_neighbours(pos, h, gorig):
    inv_h = f32(1.0 / h)
    h2 = f32(h * h)
    cell = np.floor((pos - gorig.astype(f32)) * inv_h).astype(np.int64)
    cand = acc = 0
    for i in range(len(pos)):
        near = (np.abs(cell - cell[i]) <= 1).all(1)
        d = pos[i] - pos[near]
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        cand += int(near.sum())
        acc += int((r2 < h2).sum())
    return cand, acc


def brute_splat_pairs(pos, res, mips, band, radius, world, origin):
    total = 0
    p = (pos - np.asarray(origin, f32)).astype(f32)
    for m in range(mips):
        voxel = (world / res) * 2.0 ** m
        bw = f32(band * voxel)
        reach = f32(radius + band * voxel)
        inv = f32(1 / voxel)
        v32 = f32(voxel)
        last = (res >> m) - 1
        lo = np.maximum(np.floor((p - reach) * inv).astype(np.int64), 0)
        hi = np.minimum(np.floor((p + reach) * inv).astype(np.int64), last)
        for i in range(len(p)):
            if (lo[i] > hi[i]).any():
                continue
            axes = [(np.arange(lo[i][k], hi[i][k] + 1).astype(f32) + f32(0.5)) * v32 - p[i][k] for k in range(3)]
            dz, dy, dx = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
            sd = np.sqrt((dx * dx + dy * dy) + dz * dz) - f32(radius)
            total += int((sd < bw).sum())
    return total


def test_fluid_census_counts_the_reference_work(root):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    opts = dict(capacity=4096, spacing=0.1, radius=0.05, substeps=1, gravity=(0, -9.8, 0), bakeResolution=64,
                bakeMipLevels=3, bakeBand=4.0, worldSize=24.0, origin=ORIGIN)
    sim = ce.FluidSim(root, None, opts)
    p = scenes.jittered_lattice(16, 0.1, (0.0, 3.0, 0.0), 1)
    p["vel"] = (0.3, -1.0, 0.1)
    sim.upload(p)
    sim.step()
    c = sim.census()
    info = sim.info
    cand, acc = brute_neighbours(p["pos"], info.smoothing, np.array(info.grid_origin[:]))
    assert c["particles"] == 4096
    assert c["candidates"] == cand
    assert c["accepted"] == acc
    # the bake of this frame read the stepped positions
    g = sim.download()
    pairs = brute_splat_pairs(g["pos"], 64, 3, 4.0, 0.11, 24.0, ORIGIN)
    assert c["splat_pairs"] == pairs
    assert pairs > 4096 * 100
    sim.destroy()


def test_splat_census_counts_the_bake_pairs(root):
    import torch

    import clay_engine_b200 as ce

    rng = np.random.default_rng(3)
    pos = (rng.normal(size=(3000, 3)) * 0.8 + (0.5, 1.0, -0.5)).astype(np.float32)
    cloud = ce.ParticleCloud(len(pos), torch.from_numpy(pos).cuda(), stride=12)
    s = ce.SplatField(root, cloud, radius=0.11, resolution=64, mipLevels=2, band=4.0, worldSize=24.0, origin=ORIGIN)
    assert s.census() == brute_splat_pairs(pos, 64, 2, 4.0, 0.11, 24.0, ORIGIN)
    s.destroy()


def test_fluid_census_after_batched_frames(root):
    """A sim stepped only through a Batch (whose frames read the batch's copy of every scene's
    uniform, not the sim's own) reports the census of the same sim stepped alone."""
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    opts = dict(capacity=4096, spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0), bakeResolution=64,
                bakeMipLevels=3, bakeBand=4.0, worldSize=24.0, origin=ORIGIN)
    p = scenes.jittered_lattice(16, 0.1, (0.0, 3.0, 0.0), 1)
    p["vel"] = (0.3, -1.0, 0.1)
    alone, batched = ce.FluidSim(root, None, opts), ce.FluidSim(root, None, opts)
    alone.upload(p)
    batched.upload(p)
    batch = ce.Batch(root, [batched])
    for _ in range(2):
        alone.step()
        batch.step()
    a, b = alone.census(), batched.census()
    assert a["candidates"] > 4096 * 20 and a["splat_pairs"] > 4096 * 100
    assert a == b
    batch.destroy()
    alone.destroy()
    batched.destroy()
