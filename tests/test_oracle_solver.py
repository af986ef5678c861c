"""ClaySolver restatement (oracle, CPU). The reference has no test of its solver, so it is
pinned by properties of sim/pbd.ts's algorithm: the BDF2 predictor carries uniform motion
exactly, shape matching keeps a rigid body's shape and recovers a known rotation, world
contact leaves resting particles one radius out of the floor, kinematic bodies do not move,
an impulse is applied once. The sin/cos it shares with the CUDA path is held to its error
bound against binary64."""
import math

import numpy as np

from clay_engine_b200 import brushes, scenes


def floor(oracle, top=-1.0):
    vd = oracle.VolumeData(64, 1, (-4.0, -4.0, -4.0), 8.0, 4.0)
    d, m = oracle.build_brushes(vd, brushes.make_brush("box", pos=(0.0, top - 1.0, 0.0), size=(3.5, 1.0, 3.5)))
    vd.dist[:], vd.mat[:] = d, m
    return oracle.make_field([vd]), vd


def lattice_body(center, n=5, spacing=0.1, rot=None, vel=(0.0, 0.0, 0.0), flags=0, stiffness=1.0, plasticity=0.0,
                 capacity=256, h=1 / 120):
    g = (np.arange(n) - (n - 1) / 2) * spacing
    rest = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + np.asarray(center)
    pos = rest.copy()
    if rot is not None:  # rotate about the centre
        x, y, z, w = rot
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        pos = (rest - center) @ R.T + center
    parts = np.zeros(capacity, scenes.PARTICLE_RECORD)
    k = len(rest)
    parts["pos"][:k] = pos
    parts["prev"][:k] = pos - np.asarray(vel) * h
    parts["vel"][:k] = vel
    parts["velPrev"][:k] = vel
    parts["rest"][:k] = rest
    parts["body"][:k] = 0
    bodies = np.zeros(1, scenes.BODY_RECORD)
    bodies["first"], bodies["count"] = 0, k
    bodies["com"], bodies["restCom"] = pos.mean(0), rest.mean(0)
    bodies["rot"] = (0.0, 0.0, 0.0, 1.0)
    bodies["stiffness"], bodies["plasticity"], bodies["flags"] = stiffness, plasticity, flags
    return parts, bodies, k


def test_sincos_error_bound(oracle):
    xs = np.concatenate([np.linspace(-20, 20, 4001), np.geomspace(1e-8, 1.0, 200), -np.geomspace(1e-8, 1.0, 200)])
    worst = 0.0
    for x in xs.astype(np.float32):
        s, c = oracle.sincos(float(x))
        ts, tc = math.sin(float(x)), math.cos(float(x))
        worst = max(worst, abs(s - ts), abs(c - tc))
    assert worst < 4e-7  # a few ulp of 1: reduction by a two-part pi/2, Taylor to x^9 / x^10


def test_uniform_motion_and_rigid_shape(oracle):
    field, _ = floor(oracle, top=-3.5)
    cfg = oracle.solver_cfg(256, 1)
    h = cfg.h
    parts, bodies, k = lattice_body((0.0, 1.0, 0.0), vel=(1.0, 0.5, -0.25), flags=2, h=h)  # weightless
    x0 = parts["pos"][:k].astype(np.float64).copy()
    oracle.solver_step(cfg, field, parts, bodies, 1)
    x1 = parts["pos"][:k].astype(np.float64)
    d = 0.995
    disp = np.array([1.0, 0.5, -0.25]) * h * (1 + d * 4 / 3 - 1 / 3)  # second substep: (4 v d - v) / 3 * 2h/3 + v h/3 ...
    step = x1 - x0
    assert np.abs(step - step.mean(0)).max() < 1e-5  # rigid: every particle moved alike
    assert np.abs(step[0] - np.array([1.0, 0.5, -0.25]) * h * 2).max() < 0.02 * h
    # pairwise distances kept (shape matching at stiffness 1)
    def dists(p):
        return np.linalg.norm(p[:, None] - p[None], axis=-1)
    assert np.abs(dists(x1) - dists(x0)).max() < 1e-5
    assert abs(np.linalg.norm(bodies["rot"][0]) - 1) < 1e-6
    assert np.isfinite(disp).all()


def test_rotation_recovered(oracle):
    field, _ = floor(oracle, top=-3.5)
    ang = math.radians(30)
    axis = np.array([1.0, 2.0, 0.5]) / np.linalg.norm([1.0, 2.0, 0.5])
    q = (*(axis * math.sin(ang / 2)), math.cos(ang / 2))
    cfg = oracle.solver_cfg(256, 1, rotation_iterations=12)
    parts, bodies, k = lattice_body((0.5, 0.5, -0.5), rot=q, flags=2, h=cfg.h)
    oracle.solver_step(cfg, field, parts, bodies, 1)
    r = bodies["rot"][0].astype(np.float64)
    r = r if r[3] >= 0 else -r
    assert np.abs(r - np.array(q)).max() < 1e-4


def test_resting_on_the_floor(oracle):
    field, _ = floor(oracle, top=-1.0)
    cfg = oracle.solver_cfg(256, 1)
    parts, bodies, k = lattice_body((0.2, 0.0, 0.1), stiffness=0.8, h=cfg.h)
    for _ in range(150):
        oracle.solver_step(cfg, field, parts, bodies, 1)
    y = parts["pos"][:k, 1]
    assert y.min() > -1.0 + 0.1 - 0.02  # one radius (0.1) out of the floor top, a little sink allowed
    assert y.max() < -1.0 + 0.1 + 0.45 + 0.05  # lying on it, not bouncing
    # The contact moves `prev` with `pos` (pbd.ts:203-213), so the velocity read back as
    # (pos - prev) / h keeps the unobstructed motion: on a resting contact it grows substep
    # by substep up to the speed cap while the positions stay put. Only the cap holds.
    speed = np.linalg.norm(parts["vel"][:k].astype(np.float64), axis=1)
    assert speed.max() <= 40.0 * (1 + 1e-6)
    assert np.abs(parts["vel"][:k, [0, 2]]).max() < 0.05  # friction keeps it from sliding


def test_kinematic_still_and_impulse_once(oracle):
    field, _ = floor(oracle, top=-3.5)
    cfg = oracle.solver_cfg(256, 1)
    parts, bodies, k = lattice_body((0.0, 1.0, 0.0), flags=1, h=cfg.h)
    before = parts.copy()
    for _ in range(5):
        oracle.solver_step(cfg, field, parts, bodies, 1)
    assert np.array_equal(before.view(np.uint8), parts.view(np.uint8))
    parts, bodies, k = lattice_body((0.0, 1.0, 0.0), flags=2, h=cfg.h)
    oracle.solver_set_force(cfg, 0, (0.0, 0.0, 0.0), (0.0, 3.0, 0.0))
    oracle.solver_step(cfg, field, parts, bodies, 1)
    v1 = parts["vel"][:k, 1].mean()
    assert abs(v1 - 3.0 * 0.995 ** 2) < 0.05 and cfg.kicking == 0
    oracle.solver_step(cfg, field, parts, bodies, 1)
    assert parts["vel"][:k, 1].mean() < v1  # no second kick: only damping


def test_body_count_limits_the_match_only(oracle):
    """step(bodyCount) dispatches the match pass over the first bodyCount bodies (pbd.ts:400-416):
    a body past the count keeps its record, while its particles still go through the other
    passes (they only ask whether a particle's body index is below maxBodies). At stiffness 1 the
    pull lands them exactly on the pose of the record they still carry."""
    field, _ = floor(oracle, top=-3.5)
    cfg = oracle.solver_cfg(512, 2)
    a, ba, ka = lattice_body((0.0, 1.0, 0.0), vel=(0.5, 0.0, 0.0), h=cfg.h, capacity=512)
    b, bb, kb = lattice_body((1.0, 1.0, 0.0), vel=(0.0, 0.0, 1.0), h=cfg.h, capacity=512)
    parts = a.copy()
    parts[ka:ka + kb] = b[:kb]
    parts["body"][ka:ka + kb] = 1
    bodies = np.zeros(2, scenes.BODY_RECORD)
    bodies[0] = ba[0]
    bodies[1] = bb[0]
    bodies["first"][1] = ka
    before = bodies.copy()
    rec0 = parts[ka:ka + kb].copy()
    oracle.solver_step(cfg, field, parts, bodies, 1)
    assert np.array_equal(bodies[1:].view(np.uint8), before[1:].view(np.uint8))
    assert not np.array_equal(bodies[:1].view(np.uint8), before[:1].view(np.uint8))
    assert not np.array_equal(parts[ka:ka + kb]["vel"], rec0["vel"])  # predicted and finalized
    # the unmatched record has rotation 1, so its pose is com + (rest - restCom)
    target = bodies["com"][1] + (parts["rest"][ka:ka + kb] - bodies["restCom"][1])
    assert np.abs(parts["pos"][ka:ka + kb] - target).max() < 1e-6
