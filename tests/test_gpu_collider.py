"""The collider side on the GPU: SdfVolume's mip rule and refusals (volume.gpu.ts:28-66), the
brush fold that builds collider volumes (builder.ts:87-142) and the collider queries the
fluid makes, sample(p,0) and normal(p) (trace/field.ts:102-180,246-315), against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_any_multiple_of_the_tile_is_a_legal_resolution(root):
    import clay_engine_b200 as ce

    odd = ce.SdfVolume(root, resolution=160, worldSize=12)
    assert odd.mipLevels == 3
    assert odd.tileResPerMip == [20, 10, 5]
    assert odd.totalCells == 20 ** 3 + 10 ** 3 + 5 ** 3
    flat = ce.SdfVolume(root, resolution=40, worldSize=4)
    assert flat.mipLevels == 1 and flat.tileResPerMip == [5]
    for res, levels in ((64, 3), (128, 4), (256, 5)):
        v = ce.SdfVolume(root, resolution=res)
        assert v.mipLevels == levels
        v.destroy()
    odd.destroy()
    flat.destroy()


def test_a_resolution_that_cannot_carry_the_chain_is_refused(root):
    import clay_engine_b200 as ce

    with pytest.raises(ce.ClayError, match="must be a multiple of 64"):
        ce.SdfVolume(root, resolution=160, mipLevels=4)
    with pytest.raises(ce.ClayError, match="multiple of 8"):
        ce.SdfVolume(root, resolution=100)


def build_both(root, oracle, brushes, res, world=24.0, origin=(-12.0, -4.0, -12.0), band=4.0):
    import clay_engine_b200 as ce

    v = ce.SdfVolume(root, resolution=res, worldSize=world, origin=origin, band=band)
    v.build(brushes)
    gd, gm = v.download()
    ov = oracle.VolumeData(res, v.mipLevels, origin, world, band)
    od, om = oracle.build_brushes(ov, brushes, threads=8)
    return v, gd, gm, od, om


def test_config1_collider_build_is_bit_exact(root, oracle):
    from clay_engine_b200 import scenes

    v, gd, gm, od, om = build_both(root, oracle, scenes.config1_collider_brushes(), 96)
    assert (gd == od).all(), f"{(gd != od).sum()} distance texels differ"
    assert (gm == om).all()
    assert (od != 0x3C00).any() and (od != 0xBC00).any()
    v.destroy()


def test_random_brush_build_is_bit_exact(root, oracle):
    from clay_engine_b200 import scenes

    b = scenes.random_brushes(24, seed=4)
    v, gd, gm, od, om = build_both(root, oracle, b, 64)
    assert (gd == od).all(), f"{(gd != od).sum()} distance texels differ"
    assert (gm == om).all()
    v.destroy()


def test_every_builtin_kind_builds_bit_exact(root, oracle):
    from clay_engine_b200.brushes import make_brush

    recs = [make_brush("sphere", pos=(-6, 0, -6), size=1.2), make_brush("box", pos=(-3, 0, -6), size=(1, 0.6, 0.8)),
            make_brush("roundBox", pos=(0, 0, -6), size=(1, 0.7, 0.9), radius=0.2),
            make_brush("capsule", pos=(3, 0, -6), size=(0, 1, 0), radius=0.4, euler=(0.3, 0.2, 0.1)),
            make_brush("torus", pos=(6, 0, -6), size=1.0, radius=0.3),
            make_brush("cylinder", pos=(-6, 0, 0), size=(0.8, 1.0, 0.8)),
            make_brush("boxFrame", pos=(-3, 0, 0), size=(1, 1, 1), radius=0.1),
            make_brush("cone", pos=(0, 0, 0), size=(1, 1, 0.3)), make_brush("octahedron", pos=(3, 0, 0), size=1.0),
            make_brush("tetrahedron", pos=(6, 0, 0), size=1.0), make_brush("dodecahedron", pos=(-6, 0, 6), size=1.0),
            make_brush("icosahedron", pos=(-3, 0, 6), size=1.0),
            make_brush("sphere", "cut", pos=(0, 0, 0), size=0.5, smooth=0.1),
            make_brush("plane", "paint", radius=-2.0, material=5.0),
            make_brush("box", pos=(0, 1, 0), size=(9, 0.2, 9), onlyMaterial=5.0)]
    b = np.concatenate(recs)
    v, gd, gm, od, om = build_both(root, oracle, b, 64)
    assert (gd == od).all(), f"{(gd != od).sum()} distance texels differ"
    assert (gm == om).all()
    v.destroy()


def test_collider_queries_are_bit_exact(root, oracle):
    """sample(p,0) and normal(p) at points inside, outside and around the box of two unioned
    volumes, one of them offset."""
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    a, gda, gma, oda, oma = build_both(root, oracle, scenes.config1_collider_brushes(), 64)
    b, gdb, gmb, odb, omb = build_both(root, oracle, scenes.random_brushes(8, seed=2, lo=(-2, -2, -2), hi=(2, 2, 2)),
                                       32, world=6.0, origin=(-3.0, -3.0, -3.0))
    fa, fb = ce.volumeField(a), ce.volumeField(b)
    fbo = ce.offsetField(fb, (1.0, 0.5, 0.0))
    f = ce.unionField(fa, fbo)
    rng = np.random.default_rng(1)
    pts = np.concatenate([rng.uniform(-13, 13, (2000, 3)), rng.uniform(-2, 4, (2000, 3)),
                          rng.uniform(-12, 12, (1000, 3)) * np.array([1, 0.02, 1]) + np.array([0, -0.4, 0])]).astype(np.float32)
    gs, gn = f.query(pts)
    va = oracle.VolumeData(64, a.mipLevels, (-12.0, -4.0, -12.0), 24.0, 4.0, dist=oda, mat=oma)
    vb = oracle.VolumeData(32, b.mipLevels, (-3.0, -3.0, -3.0), 6.0, 4.0, dist=odb, mat=omb)
    of = oracle.make_field([va, vb], [(0.0, 0.0, 0.0), (1.0, 0.5, 0.0)])
    os_, on = oracle.field_query_f32(of, pts)
    assert (gs.view(np.uint32) == os_.view(np.uint32)).all()
    assert (gn.view(np.uint32) == on.view(np.uint32)).all()
    for x in (f, fbo, fa, fb, a, b):
        x.destroy()


def test_rgba16f_export_has_the_reference_texel_layout(root, oracle):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    v, gd, gm, od, om = build_both(root, oracle, scenes.config1_collider_brushes(), 32)
    t = v.download_rgba16f(1)
    r = 16
    lvl = gd[v.levelOffsets[1]:v.levelOffsets[1] + r ** 3].reshape(r, r, r)
    assert (t[..., 0] == lvl).all()
    assert (t[..., 2] == 0).all() and (t[..., 3] == 0x3C00).all()
    v.destroy()
