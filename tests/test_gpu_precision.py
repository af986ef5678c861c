"""Precision study (1,048,576 particles, 288^3 collider of 64 seeded brushes, 128^3 x 4 bake,
band 4, spacing 0.1): error of the GPU's fast mode against the f64 twin of the oracle.

- density: one substep from the same state, relative error per particle (target <= 1e-4);
- bake: keys bit-exact against the f32 oracle; baked distance against the unquantised f64
  value (bounded by the key's quantisation step 1/32767.5 plus f16 storage rounding);
- drift: position difference to the f64 twin after 240 frames, on a 16k-particle blob (the
  f64 twin steps on the host cores; 1M particles for 240 frames would take hours there).

Set PRECISION_REPORT=<path> to write the figures as JSON.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORIGIN = (-12.0, -4.0, -12.0)
THREADS = os.cpu_count() or 8


def report(key, value):
    path = os.environ.get("PRECISION_REPORT")
    data = {}
    if path and os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[key] = value
    if path:
        with open(path, "w") as f:
            json.dump(data, f, indent=1)
    print(key, value)


def collider(root, oracle, res):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    v = ce.SdfVolume(root, resolution=res, worldSize=24.0, origin=ORIGIN)
    v.build(scenes.random_brushes(64, seed=2024))
    d, m = v.download()
    return v, ce.volumeField(v), oracle.VolumeData(res, v.mipLevels, ORIGIN, 24.0, 4.0, dist=d, mat=m)


def test_million_particle_density_and_bake(root, oracle):
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    n = 1 << 20
    vol, field, ov = collider(root, oracle, 288)
    opts = dict(capacity=n, spacing=0.1, radius=0.05, substeps=1, gravity=(0, -9.8, 0), bakeResolution=128,
                bakeMipLevels=4, bakeBand=4.0, worldSize=24.0, origin=ORIGIN)
    sim = ce.FluidSim(root, field, opts)
    p = scenes.lattice_block(n, 0.1, (0.0, 3.0, 0.0), 4)
    p["vel"] = (0.2, -1.0, 0.1)
    sim.upload(p)
    keys = torch.zeros(sim.surface.volume.totalVoxels, dtype=torch.int32, device="cuda")
    sim.surface.capture_keys(keys)
    sim.step()
    torch.cuda.synchronize()
    g = sim.download()
    # density vs f64 from the same input state
    from oracle.fluid_frame import OracleFluid

    ref = OracleFluid(oracle, [ov], threads=THREADS, **opts)
    prm = oracle.params_from(dict(ref.frozen, count=n, emit_base=0, emit_count=0))
    d64 = oracle.fluid_density_f64(ref.cfg, prm, p, threads=THREADS)[:, 0]
    rel = np.abs(g["density"].astype(np.float64) - d64) / np.abs(d64)
    report("density_rel_err_1m", {"max": float(rel.max()), "p99": float(np.percentile(rel, 99)),
                                  "mean": float(rel.mean()), "particles": n})
    assert rel.max() <= 1e-4
    # bake: keys bit-exact against the f32 oracle, distance against the f64 twin
    cfg = oracle.splat_cfg(128, 4, 4.0, 0.11, world_size=24.0, origin=ORIGIN)
    cloud = oracle.CloudData(np.ascontiguousarray(g["pos"]), live_mode=1, live_a=n)
    ok = oracle.splat_keys(cfg, cloud, threads=THREADS)
    gk = keys.cpu().numpy().view(np.uint32)
    assert np.array_equal(gk, ok), f"{(gk != ok).sum()} keys differ"
    v64 = oracle.splat_values_f64(cfg, cloud, threads=THREADS)
    gd, _ = sim.surface.volume.download()
    gv = gd.view(np.float16).astype(np.float64)
    err = np.abs(gv - v64)
    report("bake_1m", {"keys_bit_exact": True, "voxels": int(gk.size), "lowered": int((gk < 65535).sum()),
                       "max_abs_err_normalised": float(err.max()), "mean_abs_err_normalised": float(err.mean()),
                       "quantisation_step": 1 / 32767.5})
    assert err.max() <= 1 / 32767.5 + 2 ** -11  # key step + f16 rounding of values in [-1, 1]
    sim.destroy()
    field.destroy()
    vol.destroy()


def test_position_drift_over_240_frames(root, oracle):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    vol, field, ov = collider(root, oracle, 96)
    n = 16384
    opts = dict(capacity=n, spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0), bakeResolution=64,
                bakeMipLevels=3, bakeBand=4.0, worldSize=24.0, origin=ORIGIN)
    sim = ce.FluidSim(root, field, opts)
    p = scenes.lattice_block(n, 0.1, (0.5, 1.5, -0.5), 9)
    sim.upload(p)
    from oracle.fluid_frame import OracleFluid

    ref = OracleFluid(oracle, [ov], threads=THREADS, **opts)
    parts64 = oracle.to_f64(p)
    drift = []
    for frame in range(240):
        sim.step()
        prm = oracle.params_from(dict(ref.frozen, count=n, emit_base=0, emit_count=0))
        for _ in range(opts["substeps"]):
            oracle.fluid_substep_f64(ref.cfg, prm, ref.field, parts64, threads=THREADS)
        if frame in (0, 9, 59, 119, 239):
            g = sim.download()
            dp = np.linalg.norm(g["pos"].astype(np.float64) - parts64["pos"], axis=1)
            drift.append({"frame": frame + 1, "max": float(dp.max()), "mean": float(dp.mean())})
    report("position_drift_16k_vs_f64", drift)
    # chaotic dynamics: reported, not gated; a blown-up state would show as drift of metres
    assert drift[0]["max"] < 1e-4
    sim.destroy()
    field.destroy()
    vol.destroy()


def test_position_drift_million_particles(root, oracle):
    """Config 4's own size: 1,048,576 particles over the 288^3 collider, 2 substeps, against
    the f64 twin stepped on the host cores for 10 frames (about 2-4 s per frame on 16 cores;
    the 240 frames of the configuration would take over 10 minutes there, so the 240-frame
    drift is measured on 16k particles above). Reported, not gated beyond the first frame's
    99th percentile: the block starts partly inside the collider's solids, and deeper than
    the band the stored distance is clamped, so the field is flat there and the collision
    normal is the normalised central difference of rounding noise. The f32 and f64 runs push
    such a particle in unrelated directions: the f32 oracle on the host parts from the f64
    twin the same way (46 particles beyond 1 mm after one frame, the farthest by 0.49 m, all
    starting at the clamped distance), so the count is reported and bounded, not zero."""
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    n = 1 << 20
    vol, field, ov = collider(root, oracle, 288)
    opts = dict(capacity=n, spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0), bakeResolution=128,
                bakeMipLevels=4, bakeBand=4.0, worldSize=24.0, origin=ORIGIN)
    sim = ce.FluidSim(root, field, opts)
    p = scenes.lattice_block(n, 0.1, (0.0, 1.0, 0.0), 4)
    p["vel"] = (0.2, -1.0, 0.1)
    sim.upload(p)
    from oracle.fluid_frame import OracleFluid

    ref = OracleFluid(oracle, [ov], threads=THREADS, **opts)
    parts64 = oracle.to_f64(p)
    drift = []
    for frame in range(10):
        sim.step()
        prm = oracle.params_from(dict(ref.frozen, count=n, emit_base=0, emit_count=0))
        for _ in range(opts["substeps"]):
            oracle.fluid_substep_f64(ref.cfg, prm, ref.field, parts64, threads=THREADS)
        if frame in (0, 1, 4, 9):
            g = sim.download()
            dp = np.linalg.norm(g["pos"].astype(np.float64) - parts64["pos"], axis=1)
            drift.append({"frame": frame + 1, "max": float(dp.max()), "mean": float(dp.mean()),
                          "p99": float(np.percentile(dp, 99)), "over_1mm": int((dp > 1e-3).sum())})
    report("position_drift_1m_vs_f64", drift)
    assert drift[0]["p99"] < 1e-4
    assert drift[0]["over_1mm"] <= 100
    sim.destroy()
    field.destroy()
    vol.destroy()
