"""Seeded synthetic workloads for the fluid hot path.

Every input is generated from a seed with numpy's PCG64 (`np.random.default_rng`), so a
workload is reproducible from its config alone. The shapes and sizes are those of the five
benchmark configurations: a jittered lattice over a rounded-box collider (small), a tap
emitter over a 64-brush collider (at scale), hundreds of uneven scenes some of which carry a
clay-body shell (batched), one million particles (precision) and a resident scene pool
(serving).
"""
from __future__ import annotations

import math

import numpy as np

from .brushes import compile_shape, make_brush, sdf
from .core import PARTICLE_DTYPE

WORLD_ORIGIN = (-12.0, -4.0, -12.0)
WORLD_SIZE = 24.0


def jittered_lattice(n_side, spacing, center, seed, jitter_frac=0.1) -> np.ndarray:
    """n_side^3 particles on a lattice of `spacing` centred at `center`, each coordinate
    jittered by U(-jitter_frac, +jitter_frac) * spacing; zero velocity."""
    rng = np.random.default_rng(seed)
    idx = (np.arange(n_side) + 0.5 - n_side / 2) * spacing
    z, y, x = np.meshgrid(idx, idx, idx, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], 1) + np.asarray(center, np.float64)
    pos += rng.uniform(-jitter_frac, jitter_frac, pos.shape) * spacing
    out = np.zeros(len(pos), PARTICLE_DTYPE)
    out["pos"] = pos.astype(np.float32)
    return out


def lattice_block(n, spacing, center, seed) -> np.ndarray:
    """`n` particles from a jittered lattice block (sides ~ cbrt(n)), cut to exactly n."""
    side = int(math.ceil(n ** (1 / 3)))
    p = jittered_lattice(side, spacing, center, seed)
    return p[:n].copy()


def config1_collider_brushes() -> np.ndarray:
    """union(roundBox([11,1,11], 0.25).at([0,-1.4,0]),
    cut(box([9.5,1.4,0.9]), sphere(2).at([2.5,0.8,0]))) with the default 0.02 blend."""
    shape = sdf.union(sdf.roundBox((11, 1, 11), 0.25).at((0, -1.4, 0)),
                      sdf.cut(sdf.box((9.5, 1.4, 0.9)), sdf.sphere(2).at((2.5, 0.8, 0))))
    return compile_shape(shape)


def random_brushes(n, seed, lo=(-10, -3.5, -10), hi=(10, 2.0, 10), radius=(0.3, 2.5),
                   smooth=0.2, cut_frac=0.25, floor=True) -> np.ndarray:
    """`n` seeded brushes: spheres, boxes, capsules and tori with radii U(radius), ops add or
    cut, smooth blend `smooth`. The first is a floor slab so the fluid has somewhere to pool."""
    rng = np.random.default_rng(seed)
    recs = []
    if floor:
        recs.append(make_brush("box", "add", pos=(0.0, -3.0, 0.0), size=(10.0, 0.5, 10.0), smooth=smooth))
    kinds = ("sphere", "box", "capsule", "torus")
    while len(recs) < n:
        k = kinds[int(rng.integers(0, 4))]
        r = float(rng.uniform(*radius))
        pos = tuple(float(rng.uniform(lo[i], hi[i])) for i in range(3))
        op = "cut" if rng.random() < cut_frac else "add"
        euler = tuple(float(x) for x in rng.uniform(0, math.pi, 3))
        if k == "sphere":
            b = make_brush("sphere", op, pos=pos, size=r, smooth=smooth)
        elif k == "box":
            b = make_brush("box", op, pos=pos, euler=euler, size=tuple(r * rng.uniform(0.4, 1.0, 3)), smooth=smooth)
        elif k == "capsule":
            b = make_brush("capsule", op, pos=pos, euler=euler, size=(0.0, r, 0.0), radius=r * 0.4, smooth=smooth)
        else:
            b = make_brush("torus", op, pos=pos, euler=euler, size=r, radius=r * 0.3, smooth=smooth)
        recs.append(b)
    return np.concatenate(recs[:n])


def surface_net_sphere(radius, cell, center=(0.0, 0.0, 0.0)):
    """Clay-body shell particles of a sphere, as surface nets places them: one particle per
    grid cell whose corners straddle the surface, at the cell centre projected onto the
    surface along the field gradient (`p = v - n * dist(v)`, lib/src/sim/extract.ts:256-339,
    :305), with the gradient as its rest normal."""
    n = int(math.ceil(radius / cell)) + 2
    ax = (np.arange(-n, n + 1)) * cell
    zc, yc, xc = np.meshgrid(ax, ax, ax, indexing="ij")
    d = np.sqrt(xc ** 2 + yc ** 2 + zc ** 2) - radius
    s = d < 0
    # cell (i,j,k) spans corners i..i+1; it straddles when its 8 corners disagree in sign
    c = np.zeros(tuple(x - 1 for x in s.shape), np.int8)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                c = c + s[dz:dz + s.shape[0] - 1, dy:dy + s.shape[1] - 1, dx:dx + s.shape[2] - 1]
    straddle = (c > 0) & (c < 8)
    kz, ky, kx = np.nonzero(straddle)
    v = np.stack([ax[kx] + cell / 2, ax[ky] + cell / 2, ax[kz] + cell / 2], 1)
    r = np.linalg.norm(v, axis=1, keepdims=True)
    nrm = v / np.maximum(r, 1e-12)
    p = v - nrm * (r - radius)
    return (p + np.asarray(center)).astype(np.float32), nrm.astype(np.float32)


PARTICLE_RECORD = np.dtype([
    ("pos", np.float32, 3), ("body", np.uint32), ("prev", np.float32, 3), ("material", np.float32),
    ("vel", np.float32, 3), ("_padA", np.float32), ("velPrev", np.float32, 3), ("_padB", np.float32),
    ("rest", np.float32, 3), ("_padC", np.float32), ("restNormal", np.float32, 3), ("_padD", np.float32),
])
BODY_RECORD = np.dtype([
    ("com", np.float32, 3), ("first", np.uint32), ("rot", np.float32, 4), ("restCom", np.float32, 3),
    ("count", np.uint32), ("stiffness", np.float32), ("plasticity", np.float32), ("material", np.float32),
    ("flags", np.uint32),
])
assert PARTICLE_RECORD.itemsize == 96 and BODY_RECORD.itemsize == 64


def body_records(positions, normals, center, capacity=4096, rot=(0.0, 0.0, 0.0, 1.0)):
    """A `ParticleSet` (lib/src/sim/particles.ts:18-68) holding one body: particle records with
    `pos` and `restNormal`, and the body record with `first`, `count` and `rot`."""
    n = len(positions)
    parts = np.zeros(capacity, PARTICLE_RECORD)
    parts["pos"][:n] = positions
    parts["restNormal"][:n] = normals
    parts["rest"][:n] = positions - np.asarray(center, np.float32)
    body = np.zeros(1, BODY_RECORD)
    body["com"] = center
    body["first"] = 0
    body["count"] = n
    body["rot"] = rot
    body["restCom"] = 0.0
    return parts, body


def log_uniform_counts(n, lo, hi, seed) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), n)).astype(np.int64)


# ---- the five configurations ------------------------------------------------------------

CONFIG1 = dict(
    name="plain-small-4096",
    fluid=dict(capacity=4096, spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0),
               bakeResolution=64, bakeMipLevels=3, bakeBand=4, worldSize=24, origin=WORLD_ORIGIN),
    collider=dict(resolution=96, worldSize=24, origin=WORLD_ORIGIN),
)

CONFIG2 = dict(
    name="plain-scale-262144-tap",
    fluid=dict(capacity=262144, spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0),
               bakeResolution=128, bakeMipLevels=4, bakeBand=4, worldSize=24, origin=WORLD_ORIGIN),
    collider=dict(resolution=192, worldSize=24, origin=WORLD_ORIGIN),
    tap=dict(pos=(0.0, 6.0, 0.0), n=4096, speed=(2.0, 0.3)),
    steps=120,
)

CONFIG3 = dict(
    name="batched-256-scenes",
    scenes=256, n_lo=1024, n_hi=65536,
    fluid=dict(spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0), bakeResolution=64,
               bakeMipLevels=3, bakeBand=4, worldSize=24, origin=WORLD_ORIGIN),
    collider=dict(resolution=64, worldSize=24, origin=WORLD_ORIGIN),
    body=dict(radius=0.95, cell=0.067, bake_res=32, bake_box=32 * 0.083, band=4),
    body_every=3,
)

CONFIG4 = dict(
    name="precision-1m",
    fluid=dict(capacity=1 << 20, spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0),
               bakeResolution=128, bakeMipLevels=4, bakeBand=4, worldSize=24, origin=WORLD_ORIGIN),
    collider=dict(resolution=288, worldSize=24, origin=WORLD_ORIGIN),
    steps=240,
)

CONFIG5 = dict(
    name="serving-poisson",
    rate=2000.0, k_lo=1, k_hi=8, pool=1024, n_lo=2048, n_hi=262144, bakes=(32, 64, 128),
    budget_bytes=150 * 10 ** 9,
)


def config3_scene(root, i, n, seed, with_body=True, mode=None):
    """Scene `i` of the batched configuration: a FluidSim of capacity `n` over its own 64^3
    collider of 8 seeded brushes, its particles a jittered lattice block resting above the
    floor; every `body_every`-th scene also carries a clay-body shell (surface-net particles
    of a sphere, oriented discs) baked into a 32^3 x 2 SplatField that follows the body via
    setCenter, unioned into the scene's collider. Returns a dict: sim, body (the body's
    SplatField or None), collider (its SdfVolume), body_center, keep (objects the scene needs
    alive)."""
    import torch

    from .core import FluidSim, SdfVolume, SplatField, bodyCloud, unionField, volumeField

    cfg = CONFIG3
    bcfg = cfg["body"]
    vol = SdfVolume(root, resolution=cfg["collider"]["resolution"], worldSize=WORLD_SIZE, origin=WORLD_ORIGIN)
    vol.build(random_brushes(8, seed=seed * 100003 + i, lo=(-10, -3.5, -10), hi=(10, 1.0, 10)))
    world = volumeField(vol)
    keep = [vol, world]
    body = center = None
    if with_body and i % cfg["body_every"] == 0:
        center = (2.0, -1.4, 1.0)
        shell, shell_n = surface_net_sphere(bcfg["radius"], bcfg["cell"])
        parts, brec = body_records(shell + np.array(center, np.float32), shell_n, center)
        dp = torch.from_numpy(parts.view(np.uint8)).cuda()
        db = torch.from_numpy(brec.view(np.uint8)).cuda()
        box = bcfg["bake_box"]
        body = SplatField(root, bodyCloud(dp, db, 0), radius=(box / bcfg["bake_res"]) * 1.15,
                          resolution=bcfg["bake_res"], band=bcfg["band"], worldSize=box)
        body.setCenter(center)
        world = unionField(world, body.field)
        keep += [dp, db, body, world]
    o = dict(cfg["fluid"])
    o["capacity"] = int(n)
    sim = FluidSim(root, world, o)
    if mode:
        sim.set_mode(mode)
    side = math.ceil(n ** (1 / 3)) * 0.1
    sim.upload(lattice_block(int(n), 0.1, (0.0, -2.3 + side / 2, 0.0), seed * 7919 + i))
    return {"sim": sim, "body": body, "collider": vol, "body_center": center, "keep": keep, "options": o}
