"""SplatField bake on the GPU against the oracle: the 16-bit keys (splat.ts:223-256) and the
resolved f16 volume (splat.ts:258-276) must match bit for bit."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def bake_both(root, oracle, pos, radius, res, mips, band, world=24.0, origin=(-12.0, -4.0, -12.0),
              normals=None, quat=None, live=("all",), center=None, stride_floats=3):
    import clay_engine_b200 as ce

    torch = _torch()
    n = len(pos)
    host = np.zeros((max(n, 1), stride_floats), np.float32)
    host[:n, :3] = pos
    dpos = torch.from_numpy(host).cuda()
    kw = {}
    dn = dq = None
    if normals is not None:
        dn = torch.from_numpy(np.ascontiguousarray(normals, np.float32)).cuda()
        kw.update(normals=dn, normal_stride=12)
    if quat is not None:
        dq = torch.from_numpy(np.asarray(quat, np.float32)).cuda()
        kw.update(rotation=dq)
    live_arg = "all"
    keep = []
    if live[0] == "count":
        t = torch.tensor([live[1]], dtype=torch.int32).cuda()
        keep.append(t)
        live_arg = ("count", t)
    elif live[0] == "range":
        a = torch.tensor([live[1]], dtype=torch.int32).cuda()
        b = torch.tensor([live[2]], dtype=torch.int32).cuda()
        keep += [a, b]
        live_arg = ("range", a, b)
    cloud = ce.ParticleCloud(capacity=n, positions=dpos, stride=stride_floats * 4, live=live_arg, **kw)
    s = ce.SplatField(root, cloud, radius=radius, resolution=res, mipLevels=mips, band=band, worldSize=world,
                      origin=origin, material=3.0)
    if center is not None:
        s.setCenter(center)
    keys = torch.zeros(s.volume.totalVoxels, dtype=torch.int32).cuda()
    s.capture_keys(keys)
    s.bake()
    torch.cuda.synchronize()
    gk = keys.cpu().numpy().view(np.uint32)
    gd, gm = s.volume.download()
    # oracle
    org = origin if center is None else tuple(c - world / 2 for c in center)
    cfg = oracle.splat_cfg(res, s.volume.mipLevels, band, radius, world_size=world, material=3.0, origin=org)
    mode = {"all": 0, "count": 1, "range": 2}[live[0]]
    la = live[1] if len(live) > 1 else 0
    lb = live[2] if len(live) > 2 else 0
    oc = oracle.CloudData(np.ascontiguousarray(pos, np.float32).reshape(-1, 3), normals=normals, quat=quat,
                          live_mode=mode, live_a=la, live_b=lb)
    ok = oracle.splat_keys(cfg, oc, threads=8)
    od, om = oracle.splat_resolve(cfg, ok)
    s.destroy()
    return gk, ok, gd, od, gm, om


def assert_bake_equal(res):
    gk, ok, gd, od, gm, om = res
    diff = np.nonzero(gk != ok)[0]
    assert diff.size == 0, f"{diff.size} keys differ, first at {diff[:5]}: gpu {gk[diff[:5]]} oracle {ok[diff[:5]]}"
    assert (gd == od).all()
    assert (gm == om).all()
    assert (ok < 65535).any(), "vacuous: nothing was baked"


def fluid_blob(n_side=16, spacing=0.1, center=(0.0, 3.0, 0.0), seed=1):
    rng = np.random.default_rng(seed)
    idx = (np.arange(n_side) + 0.5 - n_side / 2) * spacing
    z, y, x = np.meshgrid(idx, idx, idx, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], 1) + center
    p += rng.uniform(-0.1, 0.1, p.shape) * spacing
    return p.astype(np.float32)


def test_fluid_blob_bake_is_bit_exact(root, oracle):
    """Config-1 bake: 4096 particles, 64^3, 3 mips, band 4, radius 0.11."""
    assert_bake_equal(bake_both(root, oracle, fluid_blob(), 0.11, 64, 3, 4.0, stride_floats=4))


def test_scale_bake_is_bit_exact(root, oracle):
    """Config-2-style bake: 128^3, 4 mips, band 4, a spread-out sheet of 30k particles."""
    rng = np.random.default_rng(7)
    p = rng.uniform((-8, -3.5, -8), (8, 0.5, 8), (30000, 3)).astype(np.float32)
    assert_bake_equal(bake_both(root, oracle, p, 0.11, 128, 4, 4.0))


def test_sparse_incoherent_cloud(root, oracle):
    """Particles scattered across and beyond the volume: exercises the per-particle walk, the
    clipping at the volume's edges, and particles entirely outside it."""
    rng = np.random.default_rng(3)
    p = rng.uniform(-16, 24, (3000, 3)).astype(np.float32)
    assert_bake_equal(bake_both(root, oracle, p, 0.5, 32, 2, 2.0))


def test_blocks_whose_union_box_exceeds_the_shared_tile(root, oracle):
    """Consecutive particles alternate between small clusters far apart, so a block's union box
    at level 0 spans several shared tiles (up to the sub-box limit, and beyond it for the wider
    spacing): the walk goes through the box in sub-boxes of the tile, or falls back to the
    other walks, and the keys stay the oracle's."""
    rng = np.random.default_rng(21)
    for span in ((8.0, 0.0, 4.0), (10.0, 2.0, 6.0), (20.0, 6.0, 20.0)):
        n = 4096
        k = np.arange(n)
        corner = np.stack([(k % 2) * span[0], ((k // 2) % 2) * span[1], ((k // 4) % 2) * span[2]], 1)
        pos = (rng.normal(size=(n, 3)) * 0.3 + corner + (-8.0, -2.0, -8.0)).astype(np.float32)
        assert_bake_equal(bake_both(root, oracle, pos, 0.11, 64, 3, 4.0))


@pytest.mark.parametrize("band", [2.0, 4.0])
def test_band_and_radius(root, oracle, band):
    p = fluid_blob(8, 0.3, center=(1.0, 2.0, -1.0), seed=5)
    assert_bake_equal(bake_both(root, oracle, p, 0.35, 32, 2, band))


def test_live_rules(root, oracle):
    p = fluid_blob(10, 0.12, seed=9)
    assert_bake_equal(bake_both(root, oracle, p, 0.15, 32, 2, 4.0, live=("count", 600)))
    assert_bake_equal(bake_both(root, oracle, p, 0.15, 32, 2, 4.0, live=("range", 200, 300)))


def test_oriented_discs_with_rotation(root, oracle):
    """bodyCloud's contribution: max(dot(delta, n), |delta| - r) with n = quatRotate(rot, rest)."""
    rng = np.random.default_rng(11)
    v = rng.normal(size=(2000, 3))
    nrm = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    pos = (nrm * 0.95 + np.array([0.3, 1.1, -0.2])).astype(np.float32)
    ang = 0.7
    q = np.array([0.0, math.sin(ang / 2), 0.0, math.cos(ang / 2)], np.float32)
    assert_bake_equal(bake_both(root, oracle, pos, 0.0955, 32, 2, 4.0, world=2.656, normals=nrm, quat=q,
                                center=(0.3, 1.1, -0.2)))


def test_set_center_moves_the_bake(root, oracle):
    p = fluid_blob(8, 0.1, center=(5.0, 5.0, 5.0))
    assert_bake_equal(bake_both(root, oracle, p, 0.11, 32, 2, 4.0, world=4.0, center=(5.1, 4.9, 5.0)))


def test_empty_cloud_bakes_saturated(root, oracle):
    """The clear is unconditional (splat.ts:289-295): nothing live reads as +1 everywhere."""
    p = fluid_blob(4, 0.1)
    gk, ok, gd, od, _, _ = bake_both(root, oracle, p, 0.11, 32, 2, 4.0, live=("count", 0))
    assert (gk == 65535).all() and (ok == 65535).all()
    assert (gd == 0x3C00).all()


def test_repeated_bakes_clear_between(root):
    """A second bake of a moved cloud does not keep the first bake's minima."""
    import clay_engine_b200 as ce

    torch = _torch()
    p = np.zeros((1, 3), np.float32)
    dp = torch.from_numpy(p).cuda()
    s = ce.SplatField(root, ce.ParticleCloud(1, dp, stride=12), radius=0.5, resolution=32, band=2.0,
                      worldSize=24.0, origin=(-12, -12, -12))
    s.bake()
    d1, _ = s.volume.download()
    dp += 6.0
    s.bake()
    d2, _ = s.volume.download()
    assert (d1 != 0x3C00).sum() == (d2 != 0x3C00).sum() > 0
    assert not np.array_equal(d1, d2)
    s.destroy()
