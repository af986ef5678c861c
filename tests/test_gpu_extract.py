"""SurfaceExtractor on the GPU against the CPU restatement, bit for bit: particle records,
body record, quad indices, draw arguments and counts (both sides give slots in lattice
order), for a plain volume field, a union of two volumes with materials and an offset, a
clamped capacity, two extractions in a row, and the motion-following re-extraction of
lib/test/gpu/extract.gpu.ts."""
import numpy as np
import pytest

from clay_engine_b200 import brushes, scenes

pytestmark = pytest.mark.gpu


def volume(root, oracle, brush_list, res, origin, world):
    import clay_engine_b200 as ce

    v = ce.SdfVolume(root, resolution=res, worldSize=world, origin=origin, mipLevels=1)
    v.build(np.concatenate(brush_list))
    d, m = v.download()
    return v, oracle.VolumeData(res, 1, origin, world, 4.0, dist=d, mat=m)


class ParticleSetDev:
    def __init__(self, capacity, max_bodies=1, parts=None, bodies=None):
        import torch

        p = parts if parts is not None else np.zeros(capacity, scenes.PARTICLE_RECORD)
        b = bodies if bodies is not None else np.zeros(max_bodies, scenes.BODY_RECORD)
        self.capacity, self.max_bodies = capacity, max_bodies
        self.parts = torch.from_numpy(p.view(np.uint8).copy()).cuda()
        self.bodies = torch.from_numpy(b.view(np.uint8).copy()).cuda()

    def host(self):
        import torch

        torch.cuda.synchronize()
        return (self.parts.cpu().numpy().view(scenes.PARTICLE_RECORD).copy(),
                self.bodies.cpu().numpy().view(scenes.BODY_RECORD).copy())


def same_records(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def run_both(root, oracle, field, ofield, res, origin, size, capacity, vel=(0.0, 0.0, 0.0), set_cap=None,
             base=0, parts=None, bodies=None, motion=None, preserve=False, follow=False, extractor=None, pset=None):
    """One extraction on the GPU and in the oracle from the same state; everything compared.
    `motion`: a CUDA ExtractMotion tensor (its value before the extraction feeds the oracle)."""
    import clay_engine_b200 as ce

    set_cap = set_cap or capacity + base
    if pset is None:
        pset = ParticleSetDev(set_cap, 1, parts, bodies)
    hm = None if motion is None else motion.cpu().numpy().copy()
    hp, hb = pset.host()
    x = extractor or ce.SurfaceExtractor(root, pset.parts, set_cap, pset.bodies, 1, field, 0, base, capacity,
                                         resolution=res, motion=motion)
    x.setRegion(origin, size, vel, preserve)
    x.extract()
    gp, gb = pset.host()
    gtri, gdraw = x.indices()
    gcnt = x.counts()
    idx, draw, cnt = oracle.extract(ofield, hp, hb, res, 0, base, capacity, origin, size, vel=vel, motion=hm,
                                    preserve=preserve, offset_by_motion=follow)
    assert tuple(int(c) for c in cnt) == gcnt
    assert np.array_equal(draw, gdraw)
    assert np.array_equal(idx[: int(draw[0])].reshape(-1, 3), gtri)
    diff = (hp.view(np.uint8).reshape(len(hp), -1) != gp.view(np.uint8).reshape(len(gp), -1)).any(1).sum()
    assert diff == 0, f"{diff} particle records differ"
    assert same_records(hb, gb)
    if hm is not None:
        assert np.array_equal(hm, motion.cpu().numpy())
    return x, pset, gp, gb, gtri


def test_sphere_bit_exact(root, oracle):
    import clay_engine_b200 as ce

    v, vd = volume(root, oracle, [brushes.make_brush("sphere", pos=(0.1, -0.2, 0.05), size=3.1, material=0.4)], 128,
                   (-4.0, -4.0, -4.0), 8.0)
    f = ce.volumeField(v)
    x, pset, gp, gb, tri = run_both(root, oracle, f, oracle.make_field([vd]), 20, (-4.0, -4.0, -4.0), 8.0, 20000,
                                    vel=(0.5, -1.0, 0.25))
    n = int(gb["count"][0])
    assert n > 500 and len(tri) > 900
    x.destroy()
    f.destroy()
    v.destroy()


def test_union_offset_material_capacity_and_repeat(root, oracle):
    import clay_engine_b200 as ce

    a, ad = volume(root, oracle, [brushes.make_brush("box", pos=(0.0, 0.0, 0.0), size=(1.2, 0.8, 1.0), material=0.2)],
                   64, (-2.0, -2.0, -2.0), 4.0)
    b, bd = volume(root, oracle, [brushes.make_brush("sphere", pos=(0.0, 0.0, 0.0), size=0.9, material=0.7),
                                  brushes.make_brush("box", "cut", pos=(0.5, 0.5, 0.0), size=0.5)],
                   64, (-2.0, -2.0, -2.0), 4.0)
    fb = ce.offsetField(ce.volumeField(b), (0.9, 0.3, -0.2))
    fu = ce.unionField(ce.volumeField(a), fb)
    of = oracle.make_field([ad, bd], offsets=[(0.0, 0.0, 0.0), (0.9, 0.3, -0.2)])
    # a clamped slice at base 100 of a larger set
    x, pset, gp, gb, tri = run_both(root, oracle, fu, of, 40, (-2.5, -2.5, -2.5), 5.0, 700, set_cap=2000, base=100)
    assert int(gb["count"][0]) == 700 and gb["first"][0] == 100
    mats = gp["material"][100:800]
    assert (np.abs(mats - 0.2) < 0.01).any() and (np.abs(mats - 0.7) < 0.01).any()
    # the same extractor again, over a moved region, from the state the first one left
    parts, bodies = pset.host()
    run_both(root, oracle, fu, of, 40, (-2.3, -2.6, -2.4), 4.9, 700, set_cap=2000, base=100, parts=parts,
             bodies=bodies, extractor=x, pset=pset)
    x.destroy()
    fu.destroy()
    a.destroy()
    b.destroy()


def test_motion_continuity(root, oracle):
    """extract.gpu.ts: re-extraction keeps the live GPU centre and mean velocity. Two particles
    at (3,5,6) and (5,5,6) with velocities (1,2,3) and (3,4,5); the motion starts at (99,99,99);
    a body-local sphere of radius 0.75 follows the motion's centre; region [-1.5, 1.5]^3 at
    resolution 16 with preserveMotion."""
    import clay_engine_b200 as ce

    v, vd = volume(root, oracle, [brushes.make_brush("sphere", size=0.75)], 64, (-2.0, -2.0, -2.0), 4.0)
    parts = np.zeros(1024, scenes.PARTICLE_RECORD)
    parts["pos"][0], parts["prev"][0], parts["vel"][0], parts["velPrev"][0] = (3, 5, 6), (3, 5, 6), (1, 2, 3), (1, 2, 3)
    parts["pos"][1], parts["prev"][1], parts["vel"][1], parts["velPrev"][1] = (5, 5, 6), (5, 5, 6), (3, 4, 5), (3, 4, 5)
    bodies = np.zeros(1, scenes.BODY_RECORD)
    bodies["first"], bodies["count"], bodies["com"], bodies["restCom"] = 0, 2, (4, 5, 6), (4, 5, 6)
    motion = ce.motion_buffer((99.0, 99.0, 99.0))
    local = ce.volumeField(v)
    field = ce.offsetFieldDevice(local, motion)
    x, pset, gp, gb, tri = run_both(root, oracle, field, oracle.make_field([vd]), 16, (-1.5, -1.5, -1.5), 3.0, 1000,
                                    set_cap=1024, parts=parts, bodies=bodies, motion=motion, preserve=True, follow=True)
    m = motion.cpu().numpy()
    assert tuple(m[:3]) == (4.0, 5.0, 6.0), "the new field must be centred on the live cloud"
    assert tuple(m[4:7]) == (2.0, 3.0, 4.0), "new particles must inherit the cloud mean velocity"
    n = int(gb["count"][0])
    assert n > 100
    assert np.all(gp["vel"][:n] == np.array([2, 3, 4], np.float32))
    assert np.abs(gp["pos"][:n].astype(np.float64).mean(0) - (4, 5, 6)).max() < 0.03
    x.destroy()
    field.destroy()
    v.destroy()
