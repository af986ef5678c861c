"""The autotuner picks a block size per scene-size bucket from real timed frames, leaves the
scenes' state as it found it, and the tuned batch computes exactly what the untuned one does."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORIGIN = (-12.0, -4.0, -12.0)


def make(root, counts, seed):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    sims = []
    for i, n in enumerate(counts):
        s = ce.FluidSim(root, None, dict(capacity=int(n), spacing=0.1, radius=0.05, substeps=2, bakeResolution=32,
                                         bakeBand=4.0, worldSize=24.0, origin=ORIGIN))
        p = scenes.lattice_block(int(n), 0.1, (0.0, 1.0, 0.0), seed + i)
        p["vel"] = (0.0, -1.0, 0.0)
        s.upload(p)
        sims.append(s)
    return sims


def test_tuning_restores_state_and_keeps_results(root):
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import autotune

    counts = [1000, 3000, 9000, 20000, 70000]
    a = make(root, counts, 5)
    b = make(root, counts, 5)
    before = [s.download() for s in a]
    stream = torch.cuda.Stream()
    result, report = autotune.tune(root, a, stream=stream, frames=1, use_cache=False)
    assert len(result["blocks"]) == len(autotune.BUCKETS)
    assert all(x in autotune.CANDIDATES for x in result["blocks"])
    assert len(report["trials"]) == len(autotune.CANDIDATES) * len({autotune.bucket_index(c) for c in counts})
    for s, snap in zip(a, before):
        now = s.download()
        assert np.array_equal(now["pos"].view(np.uint32), snap["pos"].view(np.uint32))
    tuned = ce.Batch(root, a, sph_block=result["default"])
    autotune.apply(tuned, result)
    plain = ce.Batch(root, b, sph_block=256)
    for _ in range(2):
        tuned.step(stream)
        plain.step(stream)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        gx, gy = x.download(), y.download()
        for name in ("pos", "vel", "density", "pressure", "nvel"):
            assert np.array_equal(np.ascontiguousarray(gx[name]).view(np.uint32),
                                  np.ascontiguousarray(gy[name]).view(np.uint32)), name
    for o in [tuned, plain] + a + b:
        o.destroy()
