"""Host-side logic that needs no GPU: the Poisson request stream the serving benchmark replays,
the autotuner's scene-size buckets, the per-scene device-memory estimate the server admits by,
and option checks that fail before any device work."""
import numpy as np
import pytest

from clay_engine_b200 import autotune, serve


def test_poisson_arrivals_shape_and_determinism():
    a = serve.poisson_arrivals(2000.0, 2.0, 1024, 1, 8, seed=7)
    t = np.array([x[0] for x in a])
    assert np.all(np.diff(t) >= 0) and t.min() >= 0.0 and t.max() < 2.0
    assert all(0 <= x[1] < 1024 and 1 <= x[2] <= 8 for x in a)
    assert abs(len(a) - 4000) < 5 * np.sqrt(4000)  # a Poisson count of mean 4000
    assert a == serve.poisson_arrivals(2000.0, 2.0, 1024, 1, 8, seed=7)
    assert a != serve.poisson_arrivals(2000.0, 2.0, 1024, 1, 8, seed=8)
    ks = np.array([x[2] for x in a])
    assert set(ks.tolist()) == set(range(1, 9))  # k uniform over 1..8


def test_autotune_buckets():
    assert [autotune.bucket_index(c) for c in (1, 4095, 4096, 16383, 16384, 65535, 65536, 10 ** 6)] == \
        [0, 0, 1, 1, 2, 2, 3, 3]

    class S:
        def __init__(self, c):
            self.capacity = c

    # scenes per bucket rounded up to a power of two
    assert autotune.signature([S(1000)] * 3 + [S(5000)] * 5 + [S(70000)]) == "t4-8-0-1"
    # every knob's default is one of its candidates
    assert all(autotune.DEFAULT[k] in v for k, v in autotune.KNOBS.items())


def test_estimate_counts_384_bytes_per_particle():
    """Per particle a scene holds its 48-byte record, key/rank/scratch/order words (16 B), four
    cell-ordered float4 copies (position, velocity, density record, neighbour view: 64 B) and the
    64-slot neighbour list (256 B)."""
    from clay_engine_b200 import core

    base = dict(spacing=0.1, radius=0.05, substeps=2, worldSize=24.0, origin=(-12.0, -4.0, -12.0),
                bakeResolution=64, bakeMipLevels=3, bakeBand=4.0)
    a = core.fluid_estimate_bytes(dict(base, capacity=1000))
    b = core.fluid_estimate_bytes(dict(base, capacity=3000))
    assert b - a == 2000 * 384
    c = core.fluid_estimate_bytes(dict(base, capacity=1000, bakeResolution=128, bakeMipLevels=4))
    voxels = lambda r, m: sum((r >> i) ** 3 for i in range(m))
    assert c - a == (voxels(128, 4) - voxels(64, 3)) * 8  # f16 distance + f16 material + u32 scratch


def test_solver_rejects_unknown_options_before_device_work():
    import clay_engine_b200 as ce

    with pytest.raises(ce.ClayError) as e:
        ce.ClaySolver(None, None, 1, None, 1, None, {"bogus": 1})
    assert "unknown option" in str(e.value)


def test_capacity_limit_keeps_list_offsets_in_32_bits():
    """A scene's neighbour list is addressed in 32-bit words (slot-major, slot j of particle k at
    (j / 4) * 4 * capacity + j % 4): capacities above 2^26 are refused before any allocation."""
    import pytest as _pytest

    from clay_engine_b200 import core

    base = dict(spacing=0.1, radius=0.05, substeps=2, worldSize=24.0, origin=(-12.0, -4.0, -12.0),
                bakeResolution=64, bakeMipLevels=3, bakeBand=4.0)
    assert core.fluid_estimate_bytes(dict(base, capacity=1 << 26)) > (1 << 26) * 384
    with _pytest.raises(Exception, match="capacity"):
        core.fluid_estimate_bytes(dict(base, capacity=(1 << 26) + 1))
