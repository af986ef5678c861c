"""Reading a baked volume at a level: volumeField.sample(p, mip) / field(p, mip), the level
capped at each volume's top level, through unionField and offsetField, and bandWorld /
voxelWorld of a union (trace/field.ts:102-180, 246-315, 396-429). The GPU matches the CPU
restatement bit for bit. The reference has no test of level sampling, so the restatement is
pinned here by properties instead: level 0 is the collider sampler already pinned, levels past
the top read the top, and a coarse level's surface lies within its own voxel of the fine one."""
import numpy as np
import pytest

from clay_engine_b200 import brushes

pytestmark = pytest.mark.gpu


def test_levels_capped_union_offset(root, oracle):
    import clay_engine_b200 as ce

    # a 128^3 world of four levels and a 32^3 body of two, as a scene unions them
    world = ce.SdfVolume(root, resolution=128, worldSize=8.0, origin=(-4.0, -4.0, -4.0))
    world.build(np.concatenate([brushes.make_brush("box", pos=(0, -2.5, 0), size=(3.5, 0.5, 3.5), material=0.3),
                                brushes.make_brush("sphere", pos=(1, -1, 0.5), size=1.2, material=0.6)]))
    body = ce.SdfVolume(root, resolution=32, worldSize=2.0, origin=(-1.0, -1.0, -1.0))
    body.build(brushes.make_brush("sphere", size=0.8, material=0.9))
    assert (world.mipLevels, body.mipLevels) == (4, 2)
    fw, fb = ce.volumeField(world), ce.offsetField(ce.volumeField(body), (-1.0, 0.2, 0.3))
    fu = ce.unionField(fw, fb)
    wd = oracle.VolumeData(128, 4, (-4.0, -4.0, -4.0), 8.0, world.band, dist=world.download()[0],
                           mat=world.download()[1])
    bd = oracle.VolumeData(32, 2, (-1.0, -1.0, -1.0), 2.0, body.band, dist=body.download()[0], mat=body.download()[1])
    of = oracle.make_field([wd, bd], offsets=[(0.0, 0.0, 0.0), (-1.0, 0.2, 0.3)])
    rng = np.random.default_rng(5)
    pts = rng.uniform(-4.5, 4.5, (3000, 3)).astype(np.float32)
    pts[:1000] = rng.uniform(-2.0, 1.0, (1000, 3))  # near the body and the sphere
    for mip in range(6):
        gs, gf = fu.query_mip(pts, mip)
        os_, of_ = oracle.field_query_mip_f32(of, pts, mip)
        assert np.array_equal(gs.view(np.uint32), os_.view(np.uint32)), mip
        assert np.array_equal(gf.view(np.uint32), of_.view(np.uint32)), mip
    # level 0 is the collider sampler
    s0, _ = fu.query_mip(pts, 0)
    c0, _ = fu.query(pts)
    assert np.array_equal(s0.view(np.uint32), c0.view(np.uint32))
    # past the top: the world's level 3 and the body's level 1
    s3, _ = fu.query_mip(pts, 3)
    s9, _ = fu.query_mip(pts, 9)
    assert np.array_equal(s3.view(np.uint32), s9.view(np.uint32))
    # bandWorld: min over the union at the capped levels; voxelWorld: max
    vw0, vb0 = 8.0 / 128, 2.0 / 32
    assert fu.bandWorld(0) == np.float32(np.float32(world.band) * np.float32(vw0))
    assert fu.voxelWorld(0) == np.float32(vb0)
    assert fu.voxelWorld(3) == np.float32(vw0 * 8)
    assert fu.bandWorld(3) == min(np.float32(np.float32(world.band) * np.float32(vw0)) * 8,
                                  np.float32(np.float32(body.band) * np.float32(vb0)) * 2)
    # a coarse level's zero set is within its voxel of the fine one (world sphere, inside the band)
    ws = ce.volumeField(world)
    probe = rng.normal(size=(400, 3))
    probe = (probe / np.linalg.norm(probe, axis=1, keepdims=True) * 1.2 + (1, -1, 0.5)).astype(np.float32)
    probe = probe[probe[:, 1] > -1.6]  # the floor box reaches y = -2 and swallows the sphere's bottom
    for mip in range(4):
        s, _ = ws.query_mip(probe, mip)
        assert np.abs(s[:, 0]).max() < 8.0 / 128 * 2 ** mip, mip
    for x in (ws, fu, world, body):
        x.destroy()


def test_device_points_match_the_host_hook(root, oracle):
    """clay_field_query_mip_device (device pointers, nothing allocated) gives what the host hook
    gives, at every level."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    v = ce.SdfVolume(root, resolution=64, worldSize=24.0, origin=scenes.WORLD_ORIGIN)
    v.build(scenes.random_brushes(8, seed=31, lo=(-10, -3.5, -10), hi=(10, 1.0, 10)))
    f = ce.volumeField(v)
    pts = np.random.default_rng(3).uniform(-11.0, 11.0, (5000, 3)).astype(np.float32)
    dp = torch.from_numpy(pts).cuda()
    s = torch.empty(len(pts), 2, device="cuda")
    g = torch.empty(len(pts), 2, device="cuda")
    for m in range(v.mipLevels + 1):
        hs, hf = f.query_mip(pts, m)
        f.query_mip_device(dp, s, g, m)
        torch.cuda.synchronize()
        assert np.array_equal(hs, s.cpu().numpy()) and np.array_equal(hf, g.cpu().numpy())
    with pytest.raises(ValueError):
        f.query_mip_device(dp.cpu(), s, g, 0)
    f.destroy()
    v.destroy()
