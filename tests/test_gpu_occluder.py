"""The oriented-disc bake puts a clay body's shell on its particles, the plain sphere bake a
radius outside them (lib/test/gpu/occluder.gpu.ts:214-248, same fixture :34-45,70-125).

The reference measures the shell with its sphere tracer, which is outside this path; here the
shell radius along each probe direction is found on the baked volume itself, as the first
sign change of the trilinear distance walking inward from 1.5 units out (the tracer's start)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLOOR = -1.0
BALL_R = 0.95
BALL = (0.0, FLOOR + BALL_R, 0.0)
BOX = 1.5 * 2 + (BALL_R / 8.5) * 2
SPLAT_R = (BOX / math.ceil(BOX / (BALL_R / 8.5))) * 1.15


def fibonacci_shell():
    spacing = BALL_R / 8.5
    n = math.ceil((4 * math.pi * BALL_R * BALL_R) / (spacing * spacing * 0.87))
    golden = math.pi * (3 - math.sqrt(5))
    i = np.arange(n)
    y = 1 - (2 * i) / (n - 1)
    rad = np.sqrt(np.maximum(0, 1 - y * y))
    a = golden * i
    pts = np.stack([BALL[0] + np.cos(a) * rad * BALL_R, BALL[1] + y * BALL_R, BALL[2] + np.sin(a) * rad * BALL_R], 1)
    nrm = (pts - np.array(BALL)) / BALL_R
    return pts.astype(np.float32), nrm.astype(np.float32)


def shell_radii(root, oracle, oriented, dirs):
    import torch

    import clay_engine_b200 as ce

    pts, nrm = fibonacci_shell()
    dp = torch.from_numpy(pts).cuda()
    dn = torch.from_numpy(nrm).cuda()
    cloud = ce.ParticleCloud(len(pts), dp, stride=12, normals=dn if oriented else None,
                             normal_stride=12 if oriented else None)
    s = ce.SplatField(root, cloud, radius=SPLAT_R, resolution=32, band=4, worldSize=BOX)
    s.setCenter(BALL)
    s.bake()
    d, m = s.volume.download()
    vol = oracle.VolumeData(32, s.volume.mipLevels, s.volume.origin, BOX, 4.0, dist=d, mat=m)
    field = oracle.make_field([vol])
    out = []
    for v in dirs:
        u = np.asarray(v, np.float64) / np.linalg.norm(v)
        ts = np.linspace(1.5, 0.0, 3001)
        probe = (np.array(BALL) + u[None, :] * ts[:, None]).astype(np.float32)
        sd, _ = oracle.field_query_f32(field, probe)
        k = np.nonzero(sd[:, 0] <= 0)[0]
        out.append(float(ts[k[0]]) if k.size else float("nan"))
    s.destroy()
    return out


def test_normals_put_the_shell_on_the_particles(root, oracle):
    dirs = [(1, 0, 0), (0, 1, 0), (0, -1, 0), (0.6, 0.5, -0.62)]
    plain = shell_radii(root, oracle, False, dirs)
    facets = shell_radii(root, oracle, True, dirs)
    slack = SPLAT_R / 2
    for i, d in enumerate(dirs):
        assert plain[i] > BALL_R + slack, f"spheres bulge past the particles along {d}: r={plain[i]}"
        assert abs(facets[i] - BALL_R) < slack, f"discs land on them along {d}: r={facets[i]}"
