"""The oracle pinned against the reference's own known-answer tests.

Ports of lib/test/fluid.test.mjs:30-145 (grid completeness, splat bounds, the fixed-point
encoding, rest density), lib/test/gpu/volume.gpu.ts:28-66 (mip chain and refusals) and
lib/test/gpu/brush.gpu.ts:34-209 (primitive distances worked out by hand), run against the
CPU restatement. Tolerances are the reference's: `near(.., eps=2e-3)` (evalbrush.ts:45-49),
1e-9 for the rest density, 1/32767.5 for the encoding round trip.
"""
import math

import numpy as np
import pytest


class Lcg:
    """The reference tests' generator (fluid.test.mjs:15-19), with JavaScript's binary64
    product and ToInt32 reproduced exactly."""

    def __init__(self, seed=12345):
        self.seed = seed

    def __call__(self):
        v = float(self.seed) * 1103515245.0 + 12345.0
        self.seed = (int(v) % (1 << 32)) & 0x7FFFFFFF
        return self.seed / 0x7FFFFFFF


def cloud(rnd, n, lo, hi):
    return [[lo + rnd() * (hi - lo) for _ in range(3)] for _ in range(n)]


def test_grid_scan_is_complete(oracle):
    """fluid.test.mjs:30-65 on the oracle's cellOf/cellIndex."""
    h = 1.0
    rnd = Lcg()
    pts = np.array(cloud(rnd, 400, -3, 3), np.float32)
    cfg = oracle.fluid_cfg(capacity=400, bucket=400, spacing=h / 2.2, h=h, radius=0.1,
                           origin=(-12, -4, -12), world_size=24.0, substeps=1)
    d = oracle.derive(cfg)
    assert d.grid_res == 26 and tuple(d.grid_origin) == (-13.0, -5.0, -13.0)
    parts = np.zeros(len(pts), oracle.PARTICLE_DTYPE)
    parts["pos"] = pts
    keys = oracle.fluid_cells(cfg, parts)
    assert (keys != 0xFFFFFFFF).all(), "grid must cover the volume"
    G = d.grid_res
    k64 = keys.astype(np.int64)
    cx, cy, cz = k64 % G, (k64 // G) % G, k64 // (G * G)
    buckets = {}
    for i, k in enumerate(keys):
        buckets.setdefault(int(k), []).append(i)
    p64 = pts.astype(np.float64)
    for i in range(len(pts)):
        found = set()
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    k = int(cx[i] + dx) + G * (int(cy[i] + dy) + G * int(cz[i] + dz))
                    for j in buckets.get(k, []):
                        if np.linalg.norm(p64[i] - p64[j]) < h:
                            found.add(j)
        brute = {j for j in range(len(pts)) if np.linalg.norm(p64[i] - p64[j]) < h}
        assert found == brute, f"particle {i}"


def test_splat_bounds_cover_every_voxel(oracle):
    """fluid.test.mjs:67-91, and the oracle's bake keeps every lowered voxel inside them."""
    res, world, surf_r = 32, 24.0, 0.5
    voxel = world / res
    rnd = Lcg()
    for band in (2, 4):
        bw = band * voxel
        reach = surf_r + bw
        for p in cloud(rnd, 60, 1, 22):
            lo = [math.floor((c - reach) / voxel) for c in p]
            hi = [math.floor((c + reach) / voxel) for c in p]
            ax = (np.arange(res) + 0.5) * voxel
            z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
            dist = np.sqrt((x - p[0]) ** 2 + (y - p[1]) ** 2 + (z - p[2]) ** 2) - surf_r
            zz, yy, xx = np.nonzero(dist < bw)
            assert (xx >= lo[0]).all() and (xx <= hi[0]).all()
            assert (yy >= lo[1]).all() and (yy <= hi[1]).all()
            assert (zz >= lo[2]).all() and (zz <= hi[2]).all()
            # the oracle's bake of this single particle (cloud origin at the volume corner)
            cfg = oracle.splat_cfg(res, 1, band, surf_r, world_size=world, origin=(0.0, 0.0, 0.0))
            keys = oracle.splat_keys(cfg, oracle.CloudData(np.array([p], np.float32))).reshape(res, res, res)
            kz, ky, kx = np.nonzero(keys < 65535)
            assert (kx >= lo[0]).all() and (kx <= hi[0]).all()
            assert (ky >= lo[1]).all() and (ky <= hi[1]).all()
            assert (kz >= lo[2]).all() and (kz <= hi[2]).all()
            inside = dist < bw - 1e-4
            assert (keys[inside] < 65535).all()


def test_encoding_turns_atomic_min_into_a_union(oracle):
    """fluid.test.mjs:93-113 on the oracle's encode/decode (f32, as the shader computes)."""
    enc = lambda v: oracle.enc(v, 1.0)
    assert enc(-1) == 0
    assert enc(1) == 65535
    prev = -1
    for i in range(401):
        e = enc(-1.5 + i * 0.0075)
        assert e >= prev, "encoding must be non-decreasing"
        prev = e
    rnd = Lcg()
    for _ in range(500):
        a = np.float32(rnd() * 4 - 2)
        b = np.float32(rnd() * 4 - 2)
        assert min(enc(a), enc(b)) == enc(min(a, b))
    for _ in range(500):
        v = np.float32(rnd() * 2 - 1)
        assert abs(oracle.dec(enc(v)) - v) <= 1 / 32767.5


def test_rest_density_is_the_lattice_density(oracle):
    """fluid.test.mjs:115-145."""
    spacing = 0.45
    h = spacing * 2.2
    rest = oracle.lib().orc_rest_density(spacing, h)
    poly6 = 315 / (64 * math.pi * h ** 9)
    mass = spacing ** 3
    measured = 0.0
    for z in range(-6, 7):
        for y in range(-6, 7):
            for x in range(-6, 7):
                r2 = (x * spacing) ** 2 + (y * spacing) ** 2 + (z * spacing) ** 2
                if r2 < h * h:
                    measured += mass * poly6 * (h * h - r2) ** 3
    assert abs(measured - rest) < 1e-9
    assert 0.5 < rest < 2


def test_mip_chain_rule(oracle):
    """volume.gpu.ts:28-52 (shape of the chain) and :54-66 (refusals)."""
    assert oracle.mip_levels(160) == 3
    assert [(160 // 8) >> m for m in range(3)] == [20, 10, 5]
    assert oracle.mip_levels(40) == 1
    for res, levels in ((64, 3), (128, 4), (256, 5)):
        assert oracle.mip_levels(res) == levels
    with pytest.raises(ValueError, match="must be a multiple of 64"):
        oracle.mip_levels(160, 4)
    with pytest.raises(ValueError, match="multiple of 8"):
        oracle.mip_levels(100)


def _brush(**kw):
    from clay_engine_b200.brushes import make_brush

    return make_brush(**kw)


def near(actual, expected, eps=2e-3):
    assert abs(actual - expected) < eps, f"expected ~{expected}, got {actual}"


def test_brush_known_answers(oracle):
    """brush.gpu.ts:34-120: primitives at hand-computed points."""
    ev = lambda b, pts: oracle.eval_brush(b, np.array(pts, np.float32))
    g = ev(_brush(kind="sphere", size=2, pos=(1, 0, 0)), [[1, 0, 0], [4, 0, 0], [3, 0, 0], [1, 0, 5]])
    for a, e in zip(g, (-2, 1, 0, 3)):
        near(a, e)
    g = ev(_brush(kind="sphere", size=1, scale=3), [[6, 0, 0], [0, 0, 0]])
    near(g[0], 3)
    near(g[1], -3)
    g = ev(_brush(kind="capsule", size=(0, 2, 0), radius=0.5, euler=(0, 0, math.pi / 2)),
           [[1, 0, 0], [0, 1, 0], [3, 0, 0]])
    for a, e in zip(g, (-0.5, 0.5, 0.5)):
        near(a, e)
    g = ev(_brush(kind="plane", radius=1.5), [[0, 3, 0], [9, 0, -9]])
    near(g[0], 1.5)
    near(g[1], -1.5)
    g = ev(_brush(kind="box", size=(1, 2, 3)), [[2, 0, 0], [0, 0, 0], [1, 2, 3]])
    for a, e in zip(g, (1, -1, 0)):
        near(a, e)
    g = ev(_brush(kind="cone", size=(1, 1, 0)), [[0, 0, 0], [0, 1, 0], [0, 2, 0], [2, -1, 0]])
    for a, e in zip(g, (-1 / math.sqrt(5), 0, 1, 1)):
        near(a, e)
    g = ev(_brush(kind="cone", size=(2, 1, 1)), [[0, 0, 0], [1.5, 0, 0], [0, 0, 1.5]])
    for a, e in zip(g, (-1, 0, 0)):
        near(a, e)


def test_platonic_known_answers(oracle):
    """brush.gpu.ts:138-209."""
    inr = math.sqrt((5 + 2 * math.sqrt(5)) / 15)
    phi = (1 + math.sqrt(5)) / 2

    def off_face(n, inradius, d):
        ln = math.hypot(*n)
        s = (inradius + d) / ln
        return [n[0] * s, n[1] * s, n[2] * s]

    ev = lambda kind, pts: oracle.eval_brush(_brush(kind=kind, size=1), np.array(pts, np.float32))
    g = ev("octahedron", [[0, 0, 0], [1, 0, 0], [0, 0, -1], [2, 0, 0], [0.5, 0.5, 0]])
    for a, e in zip(g, (-1 / math.sqrt(3), 0, 0, 1, 0)):
        near(a, e)
    s3 = 1 / math.sqrt(3)
    g = ev("tetrahedron", [[0, 0, 0], [s3, s3, s3], [-s3, -s3, s3], off_face([1, 1, -1], 1 / 3, 0.5)])
    for a, e in zip(g, (-1 / 3, 0, 0, 0.5)):
        near(a, e)
    g = ev("dodecahedron", [[0, 0, 0], [s3, s3, s3], [0, 1 / phi * s3, phi * s3], [phi * s3, 0, 1 / phi * s3],
                            off_face([0, phi, 1], inr, 0.5)])
    for a, e in zip(g, (-inr, 0, 0, 0, 0.5)):
        near(a, e)
    v = 1 / math.sqrt(1 + phi * phi)
    g = ev("icosahedron", [[0, 0, 0], [0, v, phi * v], [v, phi * v, 0], off_face([1, 1, 1], inr, 0.5),
                           [0, 1.5 * v, 1.5 * phi * v]])
    for a, e in zip(g, (-inr, 0, 0, 0.5, 0.5 * inr)):
        near(a, e)
    assert 0 < g[4] < 0.5


def test_brush_make_rule():
    """brush.ts:407-430 via the host rule: bound = reach * scale + smooth, unknown kinds refused."""
    from clay_engine_b200.brushes import make_brush

    b = make_brush("sphere", size=2, scale=1.5, smooth=0.05)
    near(float(b["bound"][0]), 2 * 1.5 + 0.05, 1e-6)
    b = make_brush("plane", radius=1)
    assert float(b["bound"][0]) == np.float32(1e9)
    with pytest.raises(ValueError, match="unknown primitive 'hexPrism'"):
        make_brush("hexPrism")


def test_f16_rounding_is_nearest_even(oracle):
    vals = np.array([0.0, 1.0, -1.0, 1 / 3, 65504.0, 1e-8, 2.0 ** -24, 0.1, -0.7, 1 + 2 ** -11, 1 + 3 * 2 ** -11],
                    np.float32)
    ours = oracle.f32_to_f16(vals)
    ref = vals.astype(np.float16).view(np.uint16)
    assert (ours == ref).all()


def test_hash_is_the_integer_avalanche(oracle):
    """gpu.ts:103-117 restated in Python integers."""
    def h(x):
        x &= 0xFFFFFFFF
        x ^= x >> 16
        x = (x * 0x7FEB352D) & 0xFFFFFFFF
        x ^= x >> 15
        x = (x * 0x846CA68B) & 0xFFFFFFFF
        x ^= x >> 16
        return (x & 0xFFFFFF) / 16777216
    for s in (0, 1, 9781, 123456789, 0xFFFFFFFF):
        assert oracle.hash1(s) == pytest.approx(h(s), abs=0)
