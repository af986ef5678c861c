"""SurfaceExtractor restatement (oracle, CPU), pinned by the reference's own extractor tests:
lib/test/extract.test.mjs (a sphere of radius 3.1 on a 20^3 lattice over [-4, 4]^3: dual
vertices on the surface within a cell, a closed and consistently oriented mesh, outward
winding, an inverted field flipping every triangle) and lib/test/gpu/extract.gpu.ts
(re-extraction keeps the live centre and mean velocity through the GPU-side motion). The
reference's field there is analytic; here it is the same sphere baked into an SdfVolume."""
import numpy as np

from clay_engine_b200 import brushes, scenes

R_SPHERE = 3.1


def sphere_volume(oracle, radius, res, origin, world, material=0.25):
    vd = oracle.VolumeData(res, 1, origin, world, 4.0)
    d, m = oracle.build_brushes(vd, brushes.make_brush("sphere", "add", pos=(0.0, 0.0, 0.0), size=radius,
                                                       material=material))
    vd.dist[:], vd.mat[:] = d, m
    return vd


def extract(oracle, vd, res, origin, size, capacity=20000, invert=False, **kw):
    if invert:
        vd = oracle.VolumeData(vd.res, vd.mips, vd.origin, vd.world_size, vd.band, dist=vd.dist ^ 0x8000, mat=vd.mat)
    field = oracle.make_field([vd])
    parts = np.zeros(capacity, scenes.PARTICLE_RECORD)
    bodies = np.zeros(1, scenes.BODY_RECORD)
    idx, draw, cnt = oracle.extract(field, parts, bodies, res, 0, 0, capacity, origin, size, **kw)
    n = int(bodies["count"][0])
    q = int(draw[0]) // 6
    return parts[:n], bodies[0], idx[: q * 6].reshape(-1, 3), cnt


def test_vertices_on_the_surface(oracle):
    vd = sphere_volume(oracle, R_SPHERE, 128, (-4.0, -4.0, -4.0), 8.0)
    p, body, tris, cnt = extract(oracle, vd, 20, (-4.0, -4.0, -4.0), 8.0)
    cell = 8.0 / 20
    assert len(p) > 500 and cnt[0] == len(p)
    r = np.linalg.norm(p["pos"].astype(np.float64), axis=1)
    assert np.abs(r - R_SPHERE).max() < cell
    # the snap lands on the baked surface: well inside a voxel of the 128^3 bake
    assert np.abs(r - R_SPHERE).max() < 8.0 / 128
    # normals are the field gradient: radial on a sphere
    cosang = (p["restNormal"] * p["pos"]).sum(1) / r
    assert cosang.min() > 0.99
    assert np.all(p["body"] == 0) and np.array_equal(p["rest"], p["pos"]) and np.array_equal(p["prev"], p["pos"])
    assert np.allclose(p["material"], 0.25, atol=1e-3)
    assert body["first"] == 0 and body["count"] == len(p)
    assert np.allclose(body["com"], 0.0, atol=1e-3) and np.array_equal(body["com"], body["restCom"])
    assert tuple(body["rot"]) == (0.0, 0.0, 0.0, 1.0)


def test_mesh_closed_consistent_and_outward(oracle):
    vd = sphere_volume(oracle, R_SPHERE, 128, (-4.0, -4.0, -4.0), 8.0)
    p, _, tris, cnt = extract(oracle, vd, 20, (-4.0, -4.0, -4.0), 8.0)
    assert len(tris) == 2 * cnt[1]
    edges = {}
    for a, b, c in tris:
        for e in ((a, b), (b, c), (c, a)):
            edges[e] = edges.get(e, 0) + 1
    assert all(v == 1 for v in edges.values()), "a directed edge was used twice"
    assert all((b, a) in edges for (a, b) in edges), "boundary edges on a closed sphere"
    v = p["pos"].astype(np.float64)
    n = np.cross(v[tris[:, 1]] - v[tris[:, 0]], v[tris[:, 2]] - v[tris[:, 0]])
    mid = (v[tris[:, 0]] + v[tris[:, 1]] + v[tris[:, 2]]) / 3
    assert ((n * mid).sum(1) > 0).all(), "inward-facing triangles"


def test_inverted_field_flips_every_triangle(oracle):
    vd = sphere_volume(oracle, R_SPHERE, 128, (-4.0, -4.0, -4.0), 8.0)
    _, _, tris, _ = extract(oracle, vd, 20, (-4.0, -4.0, -4.0), 8.0)
    p, _, inv, _ = extract(oracle, vd, 20, (-4.0, -4.0, -4.0), 8.0, invert=True)
    assert len(inv) == len(tris)
    v = p["pos"].astype(np.float64)
    n = np.cross(v[inv[:, 1]] - v[inv[:, 0]], v[inv[:, 2]] - v[inv[:, 0]])
    mid = (v[inv[:, 0]] + v[inv[:, 1]] + v[inv[:, 2]]) / 3
    assert ((n * mid).sum(1) < 0).all()


def test_reextraction_keeps_live_centre_and_velocity(oracle):
    """extract.gpu.ts: a body of two particles at (3,5,6), (5,5,6) with velocities (1,2,3),
    (3,4,5); a body-local sphere of radius 0.75 offset by the motion centre; the region
    [-1.5, 1.5]^3 at resolution 16 with preserveMotion."""
    vd = sphere_volume(oracle, 0.75, 64, (-2.0, -2.0, -2.0), 4.0)
    field = oracle.make_field([vd])
    parts = np.zeros(1024, scenes.PARTICLE_RECORD)
    parts["pos"][0], parts["vel"][0] = (3, 5, 6), (1, 2, 3)
    parts["pos"][1], parts["vel"][1] = (5, 5, 6), (3, 4, 5)
    bodies = np.zeros(1, scenes.BODY_RECORD)
    bodies["first"], bodies["count"], bodies["com"], bodies["restCom"] = 0, 2, (4, 5, 6), (4, 5, 6)
    motion = np.array([99, 99, 99, 0, 0, 0, 0, 0], np.float32)
    oracle.extract(field, parts, bodies, 16, 0, 0, 1000, (-1.5, -1.5, -1.5), 3.0, motion=motion, preserve=True,
                   offset_by_motion=True)
    assert tuple(motion[:3]) == (4.0, 5.0, 6.0)
    assert tuple(motion[4:7]) == (2.0, 3.0, 4.0)
    n = int(bodies["count"][0])
    assert n > 100
    p = parts[:n]
    assert np.all(p["vel"] == np.array([2, 3, 4], np.float32))
    assert np.abs(p["pos"].astype(np.float64).mean(0) - (4, 5, 6)).max() < 0.03


def test_capacity_clamps_particles_and_quads(oracle):
    vd = sphere_volume(oracle, R_SPHERE, 128, (-4.0, -4.0, -4.0), 8.0)
    _, _, _, full = extract(oracle, vd, 20, (-4.0, -4.0, -4.0), 8.0)
    p, body, tris, cnt = extract(oracle, vd, 20, (-4.0, -4.0, -4.0), 8.0, capacity=300)
    assert cnt[0] == full[0] and len(p) == 300 and body["count"] == 300
    assert len(tris) <= 2 * int(np.ceil(300 * 1.5)) and (tris < 300).all()
