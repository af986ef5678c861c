"""The autotuner picks its knobs per scene-size bucket from real timed frames, leaves the scenes'
state as it found it, and the tuned batch computes exactly what the untuned one does; and every
value of every knob gives the same frame as the defaults, in reference mode bit for bit."""
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
    assert len(result["tunings"]) == len(autotune.BUCKETS) + 1
    for t in result["tunings"]:
        assert all(t[k] in v for k, v in autotune.KNOBS.items())
    n_buckets = len({autotune.bucket_index(c) for c in counts})
    # each pass over the knobs times every value but the current one; a value adopted midway
    # makes the earlier current value a candidate again
    per_pass = sum(len(v) - 1 for v in autotune.KNOBS.values())
    per_pass_max = sum(len(v) for v in autotune.KNOBS.values())
    lanes = len(autotune.LANES) - 1
    assert per_pass + lanes <= len(report["trials"]) <= per_pass_max * (1 + n_buckets) + lanes + 1
    assert result["lanes"] in autotune.LANES
    assert all(t["ms"] > 0 and t["current_ms"] > 0 for t in report["trials"])
    assert result["default_ms"] > 0 and result["tuned_ms"] > 0
    for s, snap in zip(a, before):
        now = s.download()
        assert np.array_equal(now["pos"].view(np.uint32), snap["pos"].view(np.uint32))
    tuned = ce.Batch(root, a, sph_block=result["tunings"][-1]["sph_block"])
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


@pytest.mark.parametrize("knob", sorted(__import__("clay_engine_b200.autotune", fromlist=["KNOBS"]).KNOBS) + ["lanes"])
def test_every_setting_is_bit_exact_in_reference_mode(root, knob):
    """Each value of each knob, applied to every bucket, against the defaults: same particle
    state and bake after two frames (a batch with spheres and a clay-body shell of discs)."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import autotune, scenes

    counts = [1200, 5000, 20000, 70000]
    stream = torch.cuda.Stream()

    def run(setting):
        sims = make(root, counts, 9)
        for s in sims:
            s.set_mode("reference")
        pos, nrm = scenes.surface_net_sphere(0.95, 0.076, center=(1.0, 0.0, 0.0))
        parts, body = scenes.body_records(pos, nrm, (1.0, 0.0, 0.0), capacity=4096)
        dp = torch.from_numpy(parts.view(np.uint8)).cuda()
        db = torch.from_numpy(body.view(np.uint8)).cuda()
        shell = ce.SplatField(root, ce.bodyCloud(dp, db, 0), radius=0.095, resolution=32, band=4.0,
                              worldSize=32 * 0.083)
        shell.setCenter((1.0, 0.0, 0.0))
        b = ce.Batch(root, sims, extra_splats=[shell])
        setting = dict(setting)
        lanes = setting.pop("lanes", autotune.DEFAULT_LANES)
        tun = [dict(autotune.DEFAULT, **setting) for _ in range(len(autotune.BUCKETS) + 1)]
        autotune.apply(b, {"uppers": list(autotune.BUCKETS), "tunings": tun, "lanes": lanes})
        for _ in range(2):
            b.step(stream)
        torch.cuda.synchronize()
        out = [(s.download(), s.surface.volume.download()[0]) for s in sims] + [(None, shell.volume.download()[0])]
        b.destroy()
        for s in sims:
            s.destroy()
        shell.destroy()
        return out

    ref = run({})
    values = autotune.LANES if knob == "lanes" else autotune.KNOBS[knob]
    for v in values:
        if v == (autotune.DEFAULT_LANES if knob == "lanes" else autotune.DEFAULT[knob]):
            continue
        got = run({knob: v})
        for (ga, gd), (ra, rd) in zip(got, ref):
            assert np.array_equal(gd, rd), f"{knob}={v}: bake differs"
            if ga is None:
                continue
            for name in ("pos", "vel", "density", "pressure", "nvel"):
                assert np.array_equal(np.ascontiguousarray(ga[name]).view(np.uint32),
                                      np.ascontiguousarray(ra[name]).view(np.uint32)), f"{knob}={v}: {name}"
