"""Continuous-batching server (clay_server_*): every request's result is the same alone and in
the mix (bit for bit: scenes in one batched launch never interact), admission respects the
device-byte budget, an evicted scene comes back with its state, a scene over the budget is
refused, and the byte estimate is what a FluidSim allocates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORIGIN = (-12.0, -4.0, -12.0)
COUNTS = [1500, 3000, 800, 2200, 1200]


def options(i):
    return dict(capacity=COUNTS[i], spacing=0.1, radius=0.05, substeps=2, bakeResolution=32, bakeBand=4.0,
                worldSize=24.0, origin=ORIGIN)


def particles(i):
    from clay_engine_b200 import scenes

    p = scenes.lattice_block(COUNTS[i], 0.1, (0.2 * i, 0.5, -0.3 * i), 7 + i)
    p["vel"] = (0.1 * i, -1.0, 0.0)
    return p


@pytest.fixture(scope="module")
def colliders(root):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    out = []
    for i in range(len(COUNTS)):
        vol = ce.SdfVolume(root, resolution=64, worldSize=24.0, origin=ORIGIN)
        vol.build(scenes.random_brushes(6, seed=100 + i))
        out.append((ce.volumeField(vol), vol))
    yield out
    for f, v in out:
        f.destroy()
        v.destroy()


def server(root, colliders, budget, stream):
    from clay_engine_b200.serve import Server

    srv = Server(root, stream, budget_bytes=budget)
    for i in range(len(COUNTS)):
        assert srv.add_scene(colliders[i][0], options(i), particles(i)) == i
    return srv


def plain(root, colliders, i, frames, stream):
    import torch

    import clay_engine_b200 as ce

    sim = ce.FluidSim(root, colliders[i][0], options(i))
    sim.upload(particles(i))
    for _ in range(frames):
        sim.step(stream)
    torch.cuda.synchronize()
    return sim


def same_particles(ga, gb):
    return all(np.array_equal(np.ascontiguousarray(ga[n]).view(np.uint32), np.ascontiguousarray(gb[n]).view(np.uint32))
               for n in ("pos", "vel", "density", "pressure", "nvel"))


def test_same_alone_and_in_the_mix(root, colliders):
    import torch

    stream = torch.cuda.Stream()
    alone = server(root, colliders, 0, stream)
    mix = server(root, colliders, 0, stream)
    alone.serve([(0.0, 0, 3)])
    # scene 0 gets the same request (k=3) while other scenes' requests overlap with it
    s = mix.serve([(0.0, 1, 2), (0.0, 0, 3), (0.001, 2, 5), (0.002, 1, 1), (0.003, 3, 4), (0.004, 4, 2)])
    torch.cuda.synchronize()
    a, m = alone.sim(0), mix.sim(0)
    assert same_particles(a.download(), m.download())
    assert np.array_equal(a.surface.volume.download()[0], m.surface.volume.download()[0])
    # and both equal the plain path: the scene stepped on its own three times
    ref = plain(root, colliders, 0, 3, stream)
    assert same_particles(ref.download(), m.download())
    assert np.array_equal(ref.surface.volume.download()[0], m.surface.volume.download()[0])
    assert s["completed"] == 6 and s["frames"] >= 5
    assert s["p99_ms"] >= s["p50_ms"] > 0
    assert mix.stats()["resident_scenes"] == 5
    ref.destroy()
    alone.close()
    mix.close()


def test_budget_admission_and_eviction_keep_state(root, colliders):
    import torch

    from clay_engine_b200 import serve

    stream = torch.cuda.Stream()
    est = [serve.scene_bytes_estimate(options(i)) for i in range(len(COUNTS))]
    budget = est[1] + est[3] + 1024  # two of the larger scenes at a time
    srv = server(root, colliders, budget, stream)
    # scene 0 steps twice and goes idle; scenes 1 and 3 then need more room than is left beside
    # it, so scene 0 (the least recently used idle scene) must be evicted to admit them
    srv.serve([(0.0, 0, 2)])
    srv.serve([(0.0, 1, 2), (0.0, 3, 2)])
    assert srv.sim(0) is None, "scene 0 should have been evicted"
    assert srv.stats()["evictions"] >= 1
    # scene 0 comes back with its state and steps twice more, in a mix with other scenes
    s = srv.serve([(0.0, 0, 2), (0.0, 2, 1), (0.001, 4, 1)])
    st = srv.stats()
    assert s["completed"] == 3 and st["completed"] == 6
    assert st["resident_bytes"] <= budget
    for i, frames in ((0, 4), (1, 2), (2, 1), (3, 2), (4, 1)):
        ref = plain(root, colliders, i, frames, stream)
        assert same_particles(srv.download(i), ref.download()), i
        ref.destroy()
    srv.close()


def test_scene_over_budget_is_refused(root, colliders):
    import torch

    srv = server(root, colliders, 1000, torch.cuda.Stream())
    with pytest.raises(MemoryError):
        srv.serve([(0.0, 1, 1)], timeout_s=30)
    srv.close()


def test_estimate_is_what_a_sim_allocates(root, colliders):
    import clay_engine_b200 as ce
    from clay_engine_b200 import serve

    for i in (0, 3):
        before = root.bytes_in_use()
        sim = ce.FluidSim(root, colliders[i][0], options(i))
        used = root.bytes_in_use() - before
        assert used == serve.scene_bytes_estimate(options(i))
        sim.destroy()
