"""Fast-mode density over half-cells (density variant 3): the cells are ordered by half-cell and
each particle visits only the half-cells within reach. It must find exactly the neighbours the
reference's 27-cell scan accepts, so one frame from the same state stays within the fast-mode
tolerance of the f32 oracle, with particles outside the grid, and a scene whose cells overflow
(which reads whole cells, as the reference's bucket rule needs) in the same batch."""
import numpy as np
import pytest

from oracle.fluid_frame import OracleFluid

pytestmark = pytest.mark.gpu

ORIGIN = (-12.0, -4.0, -12.0)
FAST_REL_TOL = 2e-5
FAST_REL_TOL_PRESSURE = 2e-4
FAST_REL_TOL_VELOCITY = 1e-4


def test_half_cell_density_within_tolerance(root, oracle):
    import clay_engine_b200 as ce
    from clay_engine_b200 import autotune, scenes

    vol = ce.SdfVolume(root, resolution=64, worldSize=24.0, origin=ORIGIN)
    vol.build(scenes.config1_collider_brushes())
    d, m = vol.download()
    ov = oracle.VolumeData(64, vol.mipLevels, ORIGIN, 24.0, 4.0, dist=d, mat=m)
    field = ce.volumeField(vol)
    rng = np.random.default_rng(4)
    layouts = []
    a = scenes.lattice_block(9000, 0.1, (0.3, 1.2, -0.4), 8)
    a["pos"][:40] = rng.uniform(-20, 30, (40, 3)).astype(np.float32)  # some outside the grid
    a["vel"] = (0.4, -1.0, 0.2)
    layouts.append((a, dict(bucket=64)))
    b = scenes.jittered_lattice(14, 0.05, (0.0, 2.5, 0.0), 2)  # twice the rest density
    layouts.append((b, dict(bucket=16)))  # its cells overflow a bucket of 16
    c = scenes.lattice_block(2500, 0.1, (-2.0, 0.5, 2.0), 9)
    c["vel"] = (0.0, -2.0, 0.0)
    layouts.append((c, dict(bucket=64)))
    opts = dict(spacing=0.1, radius=0.05, substeps=2, gravity=(0, -9.8, 0), bakeResolution=64, bakeMipLevels=3,
                bakeBand=4.0, worldSize=24.0, origin=ORIGIN)
    sims, refs = [], []
    for p, extra in layouts:
        o = dict(opts, capacity=len(p), **extra)
        s = ce.FluidSim(root, field, o)
        s.set_mode("fast")
        s.upload(p)
        sims.append(s)
        refs.append(OracleFluid(oracle, [ov], **o))
    batch = ce.Batch(root, sims)
    tun = [dict(autotune.DEFAULT, density_variant=3) for _ in range(len(autotune.BUCKETS) + 1)]
    autotune.apply(batch, {"uppers": list(autotune.BUCKETS), "tunings": tun, "lanes": 1})
    for frame in range(3):
        for s, r in zip(sims, refs):
            r.upload(s.download())
        batch.step()
        for i, (s, r) in enumerate(zip(sims, refs)):
            r.step()
            n = s.particleCount
            g = s.download()
            for name in ("pos", "vel", "nvel", "density", "pressure"):
                x = g[name][:n].astype(np.float64)
                y = r.parts[name][:n].astype(np.float64)
                err = np.abs(x - y).max() / max(np.abs(y).max(), 1e-6)
                tol = {"pressure": FAST_REL_TOL_PRESSURE, "vel": FAST_REL_TOL_VELOCITY,
                       "nvel": FAST_REL_TOL_VELOCITY}.get(name, FAST_REL_TOL)
                assert err <= tol, f"scene {i} frame {frame} {name}: rel err {err:.3g}"
    batch.destroy()
    for s in sims:
        s.destroy()
    field.destroy()
    vol.destroy()
