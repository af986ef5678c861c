"""ClaySolver on the GPU against the CPU restatement, bit for bit after every frame: particle
and body records of several bodies in one ParticleSet (free, kinematic, weightless, soft
with plasticity, one larger than the 256-thread match reduction), slots owned by no body,
a pushed body with a one-shot impulse, default and non-default SolveParams, world fields
that are one volume and a union with an offset, and the argument checks of step."""
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


def quat(axis, deg):
    a = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    s, c = np.sin(np.radians(deg) / 2), np.cos(np.radians(deg) / 2)
    return (*(a * s), c)


def rot_matrix(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def particle_set(specs, capacity, max_bodies, h, seed=0):
    """Bodies laid out one after another with one unowned slot before each; every body a
    jittered lattice, optionally turned and moving. The unowned slots name body 0 (outside
    its slice) or a body id past max_bodies, as a stale record would."""
    rng = np.random.default_rng(seed)
    parts = np.zeros(capacity, scenes.PARTICLE_RECORD)
    bodies = np.zeros(max_bodies, scenes.BODY_RECORD)
    parts["body"][:] = max_bodies + 3
    at = 0
    for b, sp in enumerate(specs):
        parts["body"][at] = 0 if b % 2 else max_bodies + 1
        parts["pos"][at] = (9.0, 9.0, 9.0)
        at += 1
        n, spacing = sp.get("n", 5), sp.get("spacing", 0.1)
        g = (np.arange(n) - (n - 1) / 2) * spacing
        rest = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
        rest = rest + rng.uniform(-0.01, 0.01, rest.shape) + np.asarray(sp["center"])
        pos = rest
        if "rot" in sp:
            c = np.asarray(sp["center"])
            pos = (rest - c) @ rot_matrix(sp["rot"]).T + c
        vel = np.asarray(sp.get("vel", (0.0, 0.0, 0.0)))
        k = len(rest)
        sl = slice(at, at + k)
        parts["pos"][sl], parts["rest"][sl] = pos, rest
        parts["prev"][sl] = pos - vel * h
        parts["vel"][sl] = vel
        parts["velPrev"][sl] = vel * 0.9
        parts["body"][sl] = b
        parts["restNormal"][sl] = (0.0, 1.0, 0.0)
        parts["material"][sl] = 0.3 + 0.1 * b
        bodies["first"][b], bodies["count"][b] = at, k
        bodies["com"][b], bodies["restCom"][b] = pos.mean(0), rest.mean(0)
        bodies["rot"][b] = (0.0, 0.0, 0.0, 1.0)
        bodies["stiffness"][b] = sp.get("stiffness", 1.0)
        bodies["plasticity"][b] = sp.get("plasticity", 0.0)
        bodies["flags"][b] = sp.get("flags", 0)
        at += k
    assert at <= capacity
    return parts, bodies


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def run_solver(root, oracle, field, ofield, parts, bodies, body_count, frames, options=None, forces=()):
    """`forces`: {frame: (body, accel, impulse)} applied before that frame on both sides."""
    import torch

    import clay_engine_b200 as ce

    forces = dict(forces)
    opts = dict(options or {})
    cfg = oracle.solver_cfg(len(parts), len(bodies), **{
        {"maxSpeed": "max_speed", "rotationIterations": "rotation_iterations"}.get(k, k): v for k, v in opts.items()})
    dp = torch.from_numpy(parts.view(np.uint8).copy()).cuda()
    db = torch.from_numpy(bodies.view(np.uint8).copy()).cuda()
    sv = ce.ClaySolver(root, dp, len(parts), db, len(bodies), field, opts)
    hp, hb = parts.copy(), bodies.copy()
    for f in range(frames):
        if f in forces:
            body, accel, impulse = forces[f]
            sv.setForce(body, accel, impulse)
            oracle.solver_set_force(cfg, body, accel, impulse)
        sv.step(body_count)
        oracle.solver_step(cfg, ofield, hp, hb, body_count)
        torch.cuda.synchronize()
        gp = dp.cpu().numpy().view(scenes.PARTICLE_RECORD)
        gb = db.cpu().numpy().view(scenes.BODY_RECORD)
        bad = (gp.view(np.uint8).reshape(len(gp), -1) != hp.view(np.uint8).reshape(len(hp), -1)).any(1)
        assert not bad.any(), f"frame {f}: {int(bad.sum())} particle records differ, first slot {int(np.argmax(bad))}"
        assert same(gb, hb), f"frame {f}: body records differ"
    sv.destroy()
    return hp, hb


def test_bodies_on_a_floor_bit_exact(root, oracle):
    import clay_engine_b200 as ce

    v, vd = volume(root, oracle, [brushes.make_brush("box", pos=(0.0, -2.0, 0.0), size=(3.5, 1.0, 3.5)),
                                  brushes.make_brush("sphere", pos=(1.0, -1.0, 0.5), size=0.6)],
                   64, (-4.0, -4.0, -4.0), 8.0)
    field = ce.volumeField(v)
    specs = [
        {"center": (0.2, -0.4, 0.1), "vel": (0.5, -1.0, 0.0), "stiffness": 0.8},
        {"center": (1.0, 0.2, 0.5), "rot": quat((1, 2, 0.5), 35), "stiffness": 0.6, "plasticity": 0.05},
        {"center": (-1.2, 0.0, -0.8), "flags": 1},  # kinematic
        {"center": (-0.5, 0.5, 1.0), "flags": 2, "vel": (0.0, 0.0, -2.0)},  # weightless
        {"center": (0.0, 1.2, -1.0), "n": 12, "spacing": 0.06, "stiffness": 0.9},  # 1728 > 256 threads
    ]
    parts, bodies = particle_set(specs, 2304, 6, 1 / 120)
    kin = parts["body"] == 2
    hp, hb = run_solver(root, oracle, field, oracle.make_field([vd]), parts, bodies, 5, 40,
                        forces={3: (0, (2.0, 0.0, 0.0), (0.0, 3.0, 0.0)), 20: (4, (0.0, 5.0, 0.0), (0.0, 0.0, 0.0))})
    assert same(hp[kin], parts[kin])  # the kinematic body never moved
    assert np.isfinite(hp["pos"]).all()
    assert not np.array_equal(hp["pos"][parts["body"] == 4], parts["pos"][parts["body"] == 4])
    field.destroy()
    v.destroy()


def test_union_offset_options_bit_exact(root, oracle):
    import clay_engine_b200 as ce

    a, ad = volume(root, oracle, [brushes.make_brush("box", pos=(0.0, -1.2, 0.0), size=(1.8, 0.3, 1.8))],
                   64, (-2.0, -2.0, -2.0), 4.0)
    b, bd = volume(root, oracle, [brushes.make_brush("sphere", pos=(0.0, 0.0, 0.0), size=0.5),
                                  brushes.make_brush("box", "cut", pos=(0.3, 0.3, 0.0), size=0.3)],
                   64, (-2.0, -2.0, -2.0), 4.0)
    fu = ce.unionField(ce.volumeField(a), ce.offsetField(ce.volumeField(b), (0.4, -0.6, 0.1)))
    of = oracle.make_field([ad, bd], offsets=[(0.0, 0.0, 0.0), (0.4, -0.6, 0.1)])
    specs = [
        {"center": (0.3, 0.1, 0.1), "vel": (0.0, -3.0, 0.0), "stiffness": 0.5, "plasticity": 0.2},
        {"center": (-0.6, -0.3, -0.4), "rot": quat((0, 1, 0), 80), "stiffness": 1.0, "n": 4},
    ]
    parts, bodies = particle_set(specs, 400, 3, 1 / 270, seed=7)
    options = {"dt": 1 / 90, "substeps": 3, "rotationIterations": 4, "friction": 0.6, "damping": 0.98,
               "maxSpeed": 6.0, "gravity": (0.5, -12.0, 0.25), "radius": 0.07}
    hp, _ = run_solver(root, oracle, fu, of, parts, bodies, 2, 30, options,
                       forces={0: (1, (0.0, 0.0, 0.0), (1.0, 0.0, -0.5))})
    live = hp["body"] < 2
    assert np.linalg.norm(hp["vel"][live].astype(np.float64), axis=1).max() <= 6.0 * (1 + 1e-6)
    fu.destroy()
    a.destroy()
    b.destroy()


def test_body_count_rules(root, oracle):
    import torch

    import clay_engine_b200 as ce

    v, vd = volume(root, oracle, [brushes.make_brush("box", pos=(0.0, -2.0, 0.0), size=(3.5, 1.0, 3.5))],
                   32, (-4.0, -4.0, -4.0), 8.0)
    field = ce.volumeField(v)
    parts, bodies = particle_set([{"center": (0.0, 0.0, 0.0)}, {"center": (1.0, 0.0, 0.0)}], 300, 2, 1 / 120)
    dp = torch.from_numpy(parts.view(np.uint8).copy()).cuda()
    db = torch.from_numpy(bodies.view(np.uint8).copy()).cuda()
    sv = ce.ClaySolver(root, dp, 300, db, 2, field)
    sv.step(0)  # no bodies: nothing runs (pbd.ts:401-404)
    torch.cuda.synchronize()
    assert same(dp.cpu().numpy(), parts.view(np.uint8)) and same(db.cpu().numpy(), bodies.view(np.uint8))
    with pytest.raises(ce.ClayError):
        sv.step(3)
    with pytest.raises(ce.ClayError):
        ce.ClaySolver(root, dp, 300, db, 2, field, {"substeps": 0})
    with pytest.raises(ce.ClayError):
        ce.ClaySolver(root, dp, 300, db, 2, field, {"bogus": 1})
    # body_count 1: the second body's particles are still predicted and finalized (every
    # slot whose owner is below max_bodies is), only its match is skipped
    sv.step(1)
    hp, hb = parts.copy(), bodies.copy()
    cfg = oracle.solver_cfg(300, 2)
    oracle.solver_step(cfg, oracle.make_field([vd]), hp, hb, 1)
    torch.cuda.synchronize()
    assert same(dp.cpu().numpy(), hp.view(np.uint8)) and same(db.cpu().numpy(), hb.view(np.uint8))
    sv.destroy()
    field.destroy()
    v.destroy()


def test_body_count_changes_between_steps(root, oracle):
    """One solver stepped with a body count that changes from step to step (the substeps'
    graph is captured again for each new count) stays bit-exact to the oracle."""
    import torch

    import clay_engine_b200 as ce

    v, vd = volume(root, oracle, [brushes.make_brush("box", pos=(0.0, -2.0, 0.0), size=(3.5, 1.0, 3.5))],
                   32, (-4.0, -4.0, -4.0), 8.0)
    field = ce.volumeField(v)
    specs = [{"center": (-1.0, 0.0, 0.0), "vel": (0.5, 0.0, 0.0)}, {"center": (0.0, 0.5, 0.0), "stiffness": 0.7},
             {"center": (1.0, 1.0, 0.0), "rot": quat((0, 0, 1), 20)}]
    parts, bodies = particle_set(specs, 400, 3, 1 / 120, seed=3)
    dp = torch.from_numpy(parts.view(np.uint8).copy()).cuda()
    db = torch.from_numpy(bodies.view(np.uint8).copy()).cuda()
    sv = ce.ClaySolver(root, dp, len(parts), db, len(bodies), field)
    cfg = oracle.solver_cfg(len(parts), len(bodies))
    ofield = oracle.make_field([vd])
    hp, hb = parts.copy(), bodies.copy()
    for f, count in enumerate((3, 3, 1, 2, 2, 3, 1, 3)):
        sv.step(count)
        oracle.solver_step(cfg, ofield, hp, hb, count)
        torch.cuda.synchronize()
        assert same(dp.cpu().numpy(), hp.view(np.uint8)), f"step {f} (bodies {count}): particle records differ"
        assert same(db.cpu().numpy(), hb.view(np.uint8)), f"step {f} (bodies {count}): body records differ"
    sv.destroy()
    field.destroy()
    v.destroy()
