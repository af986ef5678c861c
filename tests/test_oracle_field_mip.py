"""Level sampling in the oracle (CPU): `sample(p, mip)` and `field(p, mip)` of
trace/field.ts:102-180 with the level capped at the volume's top level. The reference has no
test of it, so the restatement is held by properties: level 0 is the collider sampler the
fluid uses, levels past the top read the top, and the batched form the benchmark's CPU leg
times gives the per-point form's values exactly."""
import numpy as np

from clay_engine_b200 import scenes


def collider(oracle, res=64, mips=3, seed=5):
    vd = oracle.VolumeData(res, mips, scenes.WORLD_ORIGIN, 24.0, 4.0)
    d, m = oracle.build_brushes(vd, scenes.random_brushes(8, seed=seed, lo=(-10, -3.5, -10), hi=(10, 1.0, 10)),
                                threads=4)
    vd.dist[:], vd.mat[:] = d, m
    return oracle.make_field([vd]), vd


def points(n, seed=0):
    return np.random.default_rng(seed).uniform(-11.0, 11.0, (n, 3)).astype(np.float32)


def test_batched_query_equals_per_point(oracle):
    field, vd = collider(oracle)
    pts = points(400)
    for m in range(vd.mips + 1):
        s1, f1 = oracle.field_query_mip_f32(field, pts, m)
        s2, f2 = oracle.field_query_mip_batch(field, pts, m, threads=3)
        assert np.array_equal(s1, s2) and np.array_equal(f1, f2), m


def test_level_zero_is_the_collider_sampler(oracle):
    field, _ = collider(oracle)
    pts = points(400, seed=1)
    s0, _ = oracle.field_query_mip_batch(field, pts, 0, threads=2)
    sc, _ = oracle.field_query_f32(field, pts)
    assert np.array_equal(s0, sc)


def test_levels_past_the_top_read_the_top(oracle):
    field, vd = collider(oracle)
    pts = points(400, seed=2)
    top = oracle.field_query_mip_batch(field, pts, vd.mips - 1, threads=2)
    for m in (vd.mips, vd.mips + 3):
        past = oracle.field_query_mip_batch(field, pts, m, threads=2)
        assert np.array_equal(top[0], past[0]) and np.array_equal(top[1], past[1])
