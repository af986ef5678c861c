"""The oracle's f32 restatement of one FluidSim substep (fluid.ts:333-491) against its binary64
twin, on the CPU: from the same seeded lattice (spacing 0.1, 1,728 particles falling onto a
collider box), the densities agree to f32 precision and the moved positions and velocities to
a few f32 ulps of the step. The twin is the error reference of the GPU precision tests, so the
two restatements must not drift apart."""
import numpy as np

from clay_engine_b200 import brushes, scenes


def test_one_substep_f32_against_f64(oracle):
    from oracle.fluid_frame import OracleFluid

    vd = oracle.VolumeData(64, 1, scenes.WORLD_ORIGIN, 24.0, 4.0)
    d, m = oracle.build_brushes(vd, brushes.make_brush("box", pos=(0.0, -2.68, 0.0), size=(3.0, 0.5, 3.0)), threads=4)
    vd.dist[:], vd.mat[:] = d, m
    n = 1728
    opts = dict(capacity=n, spacing=0.1, radius=0.05, substeps=1, gravity=(0, -9.8, 0), bakeResolution=64,
                bakeMipLevels=1, bakeBand=4.0, worldSize=24.0, origin=scenes.WORLD_ORIGIN)
    ref = OracleFluid(oracle, [vd], threads=4, **opts)
    p = scenes.lattice_block(n, 0.1, (0.0, -1.6, 0.0), 11)
    p["vel"] = (0.3, -2.0, 0.1)
    prm = oracle.params_from(dict(ref.frozen, count=n, emit_base=0, emit_count=0))
    p32 = np.ascontiguousarray(p.astype(oracle.PARTICLE_DTYPE))
    p64 = oracle.to_f64(p32)
    contacts, _, _ = oracle.fluid_substep_f32(ref.cfg, prm, ref.field, p32, threads=4)
    oracle.fluid_substep_f64(ref.cfg, prm, ref.field, p64, threads=4)
    assert contacts > 0  # the lowest layer reached the collider box and was pushed out of it
    rel = np.abs(p32["density"].astype(np.float64) - p64["density"]) / np.abs(p64["density"])
    assert rel.max() < 5e-6, rel.max()
    assert np.abs(p32["pos"] - p64["pos"]).max() < 2e-6
    assert np.abs(p32["vel"] - p64["vel"]).max() < 1e-5 * max(1.0, np.abs(p64["vel"]).max())
