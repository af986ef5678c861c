"""clay_splat_bake_static: the SplatField bake for callers that may not allocate device memory
once running (a per-frame tick where cudaMalloc/cudaFree would stall the frame, a plugin host
that hands the library only pre-allocated buffers). Its scratch lives in a fixed device array
shared by all calls, so it is checked here on two calls in a row - the second must not see
the first's keys - against the allocating entry point's bake of the same cloud (bit for bit,
as every bake test here). It also refuses bakes beyond its fixed maximum.

Collected last (test_zz_*) so a failure here comes after every other test has run; it needs
nothing from them and also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cloud(n, seed, center):
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(n, 3)) * 0.6 + np.asarray(center)
    return p.astype(np.float32)


def _bake_both(root, host_pos, res, mips, band, radius, origin, cloud=None):
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import _native as N

    if cloud is None:
        dpos = torch.from_numpy(host_pos).cuda()
        cloud = ce.ParticleCloud(len(host_pos), dpos, stride=12)
    # the allocating entry point
    s = ce.SplatField(root, cloud, radius=radius, resolution=res, mipLevels=mips, band=band, worldSize=24.0,
                      origin=origin, material=2.0)
    s.bake()
    ref_d, ref_m = s.volume.download()
    total = s.volume.totalVoxels
    s.destroy()
    # the allocation-free entry point, through the C ABI
    opts = N.SplatOpts()
    opts.set = N.SPLAT["resolution"] | N.SPLAT["mipLevels"] | N.SPLAT["band"] | N.SPLAT["origin"] | \
        N.SPLAT["worldSize"] | N.SPLAT["material"]
    opts.radius, opts.resolution, opts.mip_levels, opts.band = radius, res, mips, band
    opts.origin[:] = origin
    opts.world_size, opts.material = 24.0, 2.0
    out_d = torch.zeros(total, dtype=torch.int16, device="cuda")
    out_m = torch.zeros(total, dtype=torch.int16, device="cuda")
    desc = cloud.desc()
    N.check(N.lib().clay_splat_bake_static(C.byref(desc), C.byref(opts), out_d.data_ptr(), out_m.data_ptr(), None))
    torch.cuda.synchronize()
    return ref_d, ref_m, out_d.cpu().numpy().view(np.uint16), out_m.cpu().numpy().view(np.uint16)


def test_static_bake_matches_the_allocating_bake_twice(root):
    origin = (-12.0, -4.0, -12.0)
    for call, (seed, center) in enumerate([(1, (0.0, 2.0, 0.0)), (2, (3.0, -1.0, 4.0))]):
        ref_d, ref_m, d, m = _bake_both(root, _cloud(20000, seed, center), 64, 3, 4.0, 0.11, origin)
        assert np.array_equal(d, ref_d), f"call {call}: {(d != ref_d).sum()} voxels differ"
        assert np.array_equal(m, ref_m), f"call {call}: material differs"
        assert (ref_d != 0x3C00).sum() > 1000, "vacuous: nothing was baked"


def test_static_bake_matches_for_discs_and_a_live_count(root):
    """The other branches of the splat: an oriented-disc cloud (normals rotated by a body
    quaternion, as bodyCloud bakes a clay body) and a cloud whose live count, read on the
    device, is below its capacity. Each twice in a row, bit for bit against clay_splat_bake."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    origin = (-12.0, -4.0, -12.0)
    pos, nrm = scenes.surface_net_sphere(0.95, 0.076, center=(1.0, 0.5, -0.5))
    rec = np.zeros((len(pos), 8), np.float32)  # 32-byte records: position, pad, normal, pad
    rec[:, 0:3], rec[:, 4:7] = pos, nrm
    drec = torch.from_numpy(rec).cuda()
    quat = torch.tensor([0.0, 0.3826834, 0.0, 0.9238795], dtype=torch.float32, device="cuda")
    discs = ce.ParticleCloud(len(pos), drec, stride=32, normals=drec[:, 4:], normal_stride=32, rotation=quat)
    dense = _cloud(30000, 5, (0.5, 1.0, 0.0))
    dpos = torch.from_numpy(dense).cuda()
    live = torch.tensor([21000], dtype=torch.int32, device="cuda")
    counted = ce.ParticleCloud(len(dense), dpos, stride=12, live=("count", live))
    for call in range(2):
        for name, cloud, radius in (("discs", discs, 0.083 * 1.15), ("live count", counted, 0.11)):
            ref_d, ref_m, d, m = _bake_both(root, None, 64, 3, 4.0, radius, origin, cloud=cloud)
            assert np.array_equal(d, ref_d), f"{name}, call {call}: {(d != ref_d).sum()} voxels differ"
            assert np.array_equal(m, ref_m), f"{name}, call {call}: material differs"
            assert (ref_d != 0x3C00).sum() > 1000, f"{name}: vacuous, nothing was baked"


def test_static_bake_refuses_beyond_its_maximum(root):
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import _native as N

    dpos = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    desc = ce.ParticleCloud(4, dpos, stride=12).desc()
    opts = N.SplatOpts()
    opts.set = N.SPLAT["resolution"]
    opts.radius, opts.resolution = 0.1, 128  # 128^3 x 4 levels = 2,396,160 voxels
    out = torch.zeros(16, dtype=torch.int16, device="cuda")
    rc = N.lib().clay_splat_bake_static(C.byref(desc), C.byref(opts), out.data_ptr(), None, None)
    assert rc == N.CLAY_EINVAL
    assert "static scratch holds at most 1048576" in N.lib().clay_last_error().decode()
