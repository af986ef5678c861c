"""Batched stepping: every scene of a batch gets exactly the result it gets alone.

Scenes of uneven size (and a clay-body shell baked in the same launch) are stepped as one
batch, with and without the CUDA graph, and compared bit for bit with the same scenes stepped
one per launch sequence.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORIGIN = (-12.0, -4.0, -12.0)


def scene(root, counts, seed, mode, collider):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    sims = []
    for i, n in enumerate(counts):
        s = ce.FluidSim(root, collider, dict(capacity=int(n) + 64, spacing=0.1, radius=0.05, substeps=2,
                                             gravity=(0, -9.8, 0), bakeResolution=64, bakeMipLevels=3, bakeBand=4.0,
                                             worldSize=24.0, origin=ORIGIN))
        s.set_mode(mode)
        p = scenes.lattice_block(int(n), 0.1, (0.3 * i - 1.0, 2.0 + 0.1 * i, 0.5), seed + i)
        p["vel"] = (0.2, -1.0, 0.1)
        s.upload(p)
        sims.append(s)
    return sims


@pytest.mark.parametrize("lanes", [1, 3])
@pytest.mark.parametrize("mode", ["reference", "fast"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_equals_alone(root, mode, use_graph, lanes):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    vol = ce.SdfVolume(root, resolution=64, worldSize=24.0, origin=ORIGIN)
    vol.build(scenes.config1_collider_brushes())
    field = ce.volumeField(vol)
    counts = [1500, 300, 4000, 2200, 64]
    alone = scene(root, counts, 10, mode, field)
    batch_sims = scene(root, counts, 10, mode, field)
    for s in batch_sims:
        s.spawn(50, (0.0, 5.0, 0.0), (0.0, -1.0, 0.0))
    for s in alone:
        s.spawn(50, (0.0, 5.0, 0.0), (0.0, -1.0, 0.0))
    b = ce.Batch(root, batch_sims, use_graph=use_graph)
    b.set_lanes(lanes)
    for frame in range(3):
        b.step()
        for s in alone:
            s.step()
        for s, t in zip(batch_sims, alone):
            g, a = s.download(), t.download()
            assert s.particleCount == t.particleCount
            for name in ("pos", "vel", "density", "pressure", "nvel"):
                assert np.array_equal(np.ascontiguousarray(g[name]).view(np.uint32),
                                      np.ascontiguousarray(a[name]).view(np.uint32)), (frame, name)
            gd, _ = s.surface.volume.download()
            ad, _ = t.surface.volume.download()
            assert np.array_equal(gd, ad), f"frame {frame}: bake differs"
    assert b.launches_per_step() > 0
    b.destroy()
    for s in alone + batch_sims:
        s.destroy()


def test_body_shell_baked_in_the_batch(root):
    """A clay-body shell (bodyCloud layout) baked in the batched launch equals its own bake."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    pos, nrm = scenes.surface_net_sphere(0.95, 0.076, center=(1.0, 0.0, 0.0))
    parts, body = scenes.body_records(pos, nrm, (1.0, 0.0, 0.0), capacity=4096,
                                      rot=(0.0, 0.3826834, 0.0, 0.9238795))
    dp = torch.from_numpy(parts.view(np.uint8)).cuda()
    db = torch.from_numpy(body.view(np.uint8)).cuda()
    cloud = ce.bodyCloud(dp, db, 0)
    box = 32 * 0.083
    s1 = ce.SplatField(root, cloud, radius=0.083 * 1.15, resolution=32, band=4.0, worldSize=box)
    s2 = ce.SplatField(root, cloud, radius=0.083 * 1.15, resolution=32, band=4.0, worldSize=box)
    for s in (s1, s2):
        s.setCenter((1.0, 0.0, 0.0))
    sim = ce.FluidSim(root, None, dict(capacity=256, spacing=0.1, substeps=1))
    b = ce.Batch(root, [sim], extra_splats=[s1])
    b.step()
    s2.bake()
    d1, _ = s1.volume.download()
    d2, _ = s2.volume.download()
    assert np.array_equal(d1, d2)
    assert (d1 != 0x3C00).sum() > 1000
    b.destroy()
    for x in (s1, s2, sim):
        x.destroy()


@pytest.mark.parametrize("use_graph", [True, False])
def test_upload_between_batched_frames(root, use_graph):
    """Particles uploaded into a batch's scenes between frames (as a server's re-admission or
    a restored state does), far from where the scenes were: the batch (its graph replayed as
    captured) and the same scenes stepped alone stay bit for bit the same."""
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    counts = [900, 2500, 300]
    alone = scene(root, counts, 30, "reference", None)
    batch_sims = scene(root, counts, 30, "reference", None)
    b = ce.Batch(root, batch_sims, use_graph=use_graph)
    for _ in range(2):
        b.step()
        for s in alone:
            s.step()
    for i, (s, t) in enumerate(zip(batch_sims, alone)):
        p = scenes.lattice_block(counts[i], 0.1, (5.0 - 4.0 * i, 9.0, -6.0 + 5.0 * i), 77 + i)
        p["vel"] = (-0.3, 0.5, 0.2)
        s.upload(p)
        t.upload(p)
    for frame in range(2):
        b.step()
        for s in alone:
            s.step()
        for s, t in zip(batch_sims, alone):
            g, a = s.download(), t.download()
            for name in ("pos", "vel", "density", "pressure", "nvel"):
                assert np.array_equal(np.ascontiguousarray(g[name]).view(np.uint32),
                                      np.ascontiguousarray(a[name]).view(np.uint32)), (frame, name)
    b.destroy()
    for s in alone + batch_sims:
        s.destroy()
