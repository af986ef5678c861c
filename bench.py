#!/usr/bin/env python
"""Benchmark of the fluid hot path: particle-steps/s of FluidSim.step + SplatField.bake.

One particle-step is one particle advanced one frame (all substeps) plus that frame's bake.
The default workload is the batched configuration: 256 independent scenes (particle counts
log-uniform over 1k-64k, a 64^3 collider from 8 seeded brushes each, a 64^3 x 3 bake each,
every third scene also carrying a clay-body shell of ~3k particles baked into a 32^3 volume
unioned into its collider), all advanced one frame per batched launch captured in one CUDA
graph. The same scenes stepped one scene per launch sequence give the plain rate reported
beside it. Inputs are seeded synthetic data (no dataset): jittered lattices of spacing 0.1.

Beside the headline the line carries: `e2e` (the same frames through the public API, inputs up
from and results down to pinned host memory every frame), `served` (a native continuous-batching
server under Poisson arrivals of step-and-bake requests, p50/p99 latency, and a second stream
below capacity when the first one outruns the GPU), `roofline` (the dominant kernel against the
measured HBM peak, with the neighbour passes), `cpu_baseline` (the f32 oracle on the host cores),
`next_rows` (collider build, level sampling, surface nets and the ClaySolver, each against the
oracle on the same inputs), `clocks` and `gpu_launches`.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU: one process per GPU under torchrun; each rank steps its own 256 scenes (weak
scaling, no collective on the data path); timings are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/sec (step+bake) batched/served vs plain, 1 B200; p99 request latency"
UNIT = "particle-steps/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--small", action="store_true", help="a small case for profiling (16 scenes)")
    ap.add_argument("--serve-window", type=float, default=2.0, help="seconds of Poisson arrivals served")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="requests per second")
    ap.add_argument("--serve-pool", type=int, default=1024, help="resident scenes of the serving pool")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-next", action="store_true", help="skip the measurements of the rows after the frame")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (every bucket at the defaults)")
    ap.add_argument("--set", action="append", default=[], metavar="KNOB=VALUE",
                    help="with --no-tune: run every bucket at this setting of an autotuner knob instead of its default")
    ap.add_argument("--workload", default="batched", choices=["batched", "tap"],
                    help="batched: the 256-scene batch (+plain, served); tap: one 262,144-particle scene fed by a tap")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
# Workload

def fluid_opts(n):
    from clay_engine_b200 import scenes

    o = dict(scenes.CONFIG3["fluid"])
    o["capacity"] = int(n)
    return o


def build_scenes(root, n_scenes, seed, with_bodies=True):
    """The batched configuration on this GPU. Returns (sims, bodies, keepalive)."""
    from clay_engine_b200 import scenes

    cfg = scenes.CONFIG3
    counts = scenes.log_uniform_counts(n_scenes, cfg["n_lo"], cfg["n_hi"], seed)
    sims, bodies, keep = [], [], []
    for i, n in enumerate(counts):
        sc = scenes.config3_scene(root, i, int(n), seed, with_body=with_bodies)
        sims.append(sc["sim"])
        if sc["body"] is not None:
            bodies.append(sc["body"])
        keep += sc["keep"]
    return sims, bodies, keep


def serve_pool(root, n_scenes, seed, stream, budget):
    """The serving configuration: a native server holding `n_scenes` registered scenes, particle
    counts log-uniform over 2k-256k, bake volumes 32^3 / 64^3 / 128^3 (seeded choice), a 64^3
    collider of 8 brushes each (built up front: colliders stay resident, the budget covers the
    scenes' FluidSims). Returns (server, particle counts)."""
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes, serve

    cfg = scenes.CONFIG5
    counts = scenes.log_uniform_counts(n_scenes, cfg["n_lo"], cfg["n_hi"], seed)
    rng = np.random.default_rng(seed + 1)
    bakes = [int(cfg["bakes"][int(b)]) for b in rng.integers(0, len(cfg["bakes"]), n_scenes)]
    # at most 160 scenes per frame: in a backlog, frames of all waiting scenes ran slower per
    # particle-step than capped ones (measured: 421 M/s uncapped, 450 M/s at 160, 2400 req/s)
    srv = serve.Server(root, stream, budget_bytes=budget, max_batch=160)
    for i in range(n_scenes):
        vol = ce.SdfVolume(root, resolution=64, worldSize=24.0, origin=scenes.WORLD_ORIGIN)
        vol.build(scenes.random_brushes(8, seed=seed * 100003 + i, lo=(-10, -3.5, -10), hi=(10, 1.0, 10)))
        field = ce.volumeField(vol)
        o = dict(scenes.CONFIG3["fluid"])
        o.update(capacity=int(counts[i]), bakeResolution=bakes[i], bakeMipLevels=max(1, int(math.log2(bakes[i] / 8))))
        n = int(counts[i])
        side = math.ceil(n ** (1 / 3)) * 0.1
        srv.add_scene(field, o, scenes.lattice_block(n, 0.1, (0.0, -2.3 + side / 2, 0.0), seed * 7919 + i), keep=[vol])
    return srv, counts


def run_serving(root, args, seed, stream):
    from clay_engine_b200 import scenes, serve

    cfg = scenes.CONFIG5
    t0 = time.perf_counter()
    srv, counts = serve_pool(root, args.serve_pool, seed, stream, cfg["budget_bytes"])
    # every scene once (admits them and warms the kernels), then the measured arrivals
    srv.serve([(0.0, i, 1) for i in range(args.serve_pool)], timeout_s=600)
    setup_s = time.perf_counter() - t0
    arrivals = serve.poisson_arrivals(args.serve_rate, args.serve_window, args.serve_pool, cfg["k_lo"], cfg["k_hi"],
                                      seed + 2)
    out = srv.serve(arrivals, timeout_s=600)
    st = srv.stats()
    per_request = (cfg["k_lo"] + cfg["k_hi"]) / 2 * float(np.mean(counts))  # particle-steps offered per request
    out.update(rate_req_s=args.serve_rate, window_s_arrivals=args.serve_window, requests=len(arrivals),
               resident_scenes=st["resident_scenes"], resident_gb=st["resident_bytes"] / 1e9, setup_s=setup_s,
               budget_gb=cfg["budget_bytes"] / 1e9, server="native (clay_server_*)",
               demand_particle_steps_s=float(args.serve_rate * per_request))
    # When the offered load exceeds what the GPU sustains on this workload, the queue grows for
    # the whole window and the latency measures the backlog. A second stream at 70 % of the
    # throughput just measured gives the latency of a server that keeps up.
    if out["demand_particle_steps_s"] > out["throughput"] and out["throughput"] > 0:
        rate = 0.7 * out["throughput"] / per_request
        light = srv.serve(serve.poisson_arrivals(rate, args.serve_window, args.serve_pool, cfg["k_lo"], cfg["k_hi"],
                                                 seed + 3), timeout_s=600)
        light.update(rate_req_s=rate, demand_particle_steps_s=float(rate * per_request))
        out["below_capacity"] = {k: light[k] for k in ("rate_req_s", "demand_particle_steps_s", "throughput", "p50_ms",
                                                       "p99_ms", "mean_ms", "mean_batch", "completed")}
    srv.close()
    for f in srv.keep:
        if hasattr(f, "destroy"):
            f.destroy()
    return out


# ---------------------------------------------------------------------------------------
# Clocks during the timed region

class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled every few milliseconds by a thread
    through NVML (read-only queries), each sample time-stamped so the summary covers exactly the
    window between mark() and stop(). Falls back to `nvidia-smi -lms` where NVML is missing."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device, period_s=0.005):
        self.device = device
        self.period = period_s
        self.samples = []  # (time, sm_mhz, reason bits)
        self.max_mhz = None
        self.stop_flag = threading.Event()
        self.t = None
        self.proc = None
        self.start = self.end = None

    def _handle(self, N):
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return N.nvmlDeviceGetHandleByIndex(self.device)

    def _nvml_loop(self, N, h):
        while not self.stop_flag.is_set():
            try:
                mhz = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                bits = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), float(mhz), int(bits)))
            except Exception:
                pass
            time.sleep(self.period)

    def _smi_loop(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz, self.max_mhz = float(f[1]), float(f[2])
            except ValueError:
                continue
            bits = 0
            for (nm, b), v in zip(self.REASONS, f[5:9]):
                if v.lower().startswith("active"):
                    bits |= b
            self.samples.append((time.perf_counter(), mhz, bits))

    def __enter__(self):
        try:
            import pynvml as N

            N.nvmlInit()
            h = self._handle(N)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._nvml_loop, args=(N, h), daemon=True)
        except Exception:
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.t = threading.Thread(target=self._smi_loop, daemon=True)
            except OSError:
                return self
        self.t.start()
        t0 = time.time()
        while not self.samples and time.time() - t0 < 15:  # the first sample is in
            time.sleep(0.01)
        return self

    def mark(self):
        """Starts the sample window of the timed region."""
        self.start = time.perf_counter()

    def stop(self):
        self.end = time.perf_counter()

    def __exit__(self, *a):
        self.stop_flag.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=5)

    def summary(self):
        t0 = self.start if self.start is not None else -float("inf")
        t1 = self.end if self.end is not None else float("inf")
        inside = [x for x in self.samples if t0 <= x[0] <= t1]
        if not inside and self.samples:  # a window shorter than the period: the nearest sample
            inside = [min(self.samples, key=lambda x: abs(x[0] - t0))]
        reasons = sorted({nm for _, _, bits in inside for nm, b in self.REASONS if bits & b})
        sm = [x[1] for x in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# CPU baseline: the oracle (the f32 restatement of the reference WGSL) on host cores.

class CpuSample:
    """The oracle (the f32 restatement of the reference WGSL) on a bounded sample of the
    batched scenes: the scenes nearest the median size, up to `max_particles` particles, each
    with its own collider, built once. One rep = every scene of the sample advanced one frame
    from its initial state (the states are put back before each rep, untimed), so every rep,
    in this arm and in the reference arm, times the same work."""

    def __init__(self, n_scenes, seed, max_particles, threads):
        from clay_engine_b200 import scenes
        from oracle import oracle
        from oracle.fluid_frame import OracleFluid

        oracle.build()
        cfg = scenes.CONFIG3
        counts = scenes.log_uniform_counts(n_scenes, cfg["n_lo"], cfg["n_hi"], seed)
        order = np.argsort(np.abs(np.log(counts) - np.median(np.log(counts))))
        chosen, total = [], 0
        for i in order:
            if total + counts[i] > max_particles and chosen:
                break
            chosen.append(int(i))
            total += int(counts[i])
        self.sims, self.starts = [], []
        for i in chosen:
            vd = oracle.VolumeData(64, 3, scenes.WORLD_ORIGIN, 24.0, 4.0)
            d, m = oracle.build_brushes(vd, scenes.random_brushes(8, seed=seed * 100003 + i, lo=(-10, -3.5, -10),
                                                                   hi=(10, 1.0, 10)), threads=threads)
            vd.dist[:], vd.mat[:] = d, m
            ref = OracleFluid(oracle, [vd], threads=threads, **fluid_opts(counts[i]))
            side = math.ceil(counts[i] ** (1 / 3)) * 0.1
            self.starts.append(scenes.lattice_block(int(counts[i]), 0.1, (0.0, -2.3 + side / 2, 0.0), seed * 7919 + i))
            self.sims.append(ref)
        self.particles = total
        self.threads = threads
        self.desc = (f"{len(chosen)} of the {n_scenes} batched scenes nearest the median size, {total} particles, "
                     f"one frame each from their initial state per rep, f32 oracle, {threads} thread(s)")

    def rep(self) -> float:
        """Seconds of one rep."""
        for ref, p in zip(self.sims, self.starts):
            ref.upload(p)
        t0 = time.perf_counter()
        for ref in self.sims:
            ref.step()
        return time.perf_counter() - t0


def _event_ms(stream, fn, reps):
    """Device time of `reps` calls of fn() on `stream` (CUDA events on that stream), in ms."""
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _cpu_s(fn):
    t = time.perf_counter()
    fn()
    return time.perf_counter() - t


def body_set(shell, normals, centers, capacity=None):
    """A ParticleSet holding one surface-net shell per centre: 96-byte Particle and 64-byte Body
    records (particles.ts:18-68), rest shape relative to the body centre."""
    from clay_engine_b200 import scenes

    n = len(shell)
    cap = capacity or n * len(centers)
    parts = np.zeros(cap, scenes.PARTICLE_RECORD)
    bodies = np.zeros(len(centers), scenes.BODY_RECORD)
    for b, c in enumerate(centers):
        sl = slice(b * n, (b + 1) * n)
        parts["pos"][sl] = shell + np.asarray(c, np.float32)
        parts["prev"][sl] = parts["pos"][sl]
        parts["rest"][sl] = shell
        parts["restNormal"][sl] = normals
        parts["body"][sl] = b
        parts["material"][sl] = 0.5
        bodies["com"][b], bodies["first"][b], bodies["count"][b] = c, b * n, n
        bodies["rot"][b] = (0.0, 0.0, 0.0, 1.0)
        bodies["stiffness"][b] = 0.8
    return parts, bodies


def measure_next_rows(root, stream, threads):
    """The rows after the frame, each measured as the frame is: device throughput with CUDA
    events on the launching stream, achieved GB/s from algorithmic bytes, and the oracle on the
    host cores on the same inputs (a bounded sample where the full case would take long)."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import brushes as B
    from clay_engine_b200 import scenes
    from oracle import oracle

    oracle.build()
    out = {}
    origin = (-12.0, -4.0, -12.0)

    # 1. collider build (SdfBuilder brush fold): config 2's 192^3 world volume from 64 brushes
    br = scenes.random_brushes(64, seed=2024)
    vol = ce.SdfVolume(root, resolution=192, worldSize=24.0, origin=origin)
    vol.build(br, stream)
    ms = _event_ms(stream, lambda: vol.build(br, stream), 5) / 5
    vox = vol.totalVoxels
    cpu_vd = oracle.VolumeData(96, 3, origin, 24.0, 4.0)
    cpu_vox = oracle.total_voxels(96, 3)
    cs = _cpu_s(lambda: oracle.build_brushes(cpu_vd, br, threads=threads))
    out["collider_build"] = {
        "workload": f"192^3 x {vol.mipLevels} levels from 64 brushes", "value": vox / (ms / 1e3), "unit": "voxels/s",
        "ms_per_build": ms, "achieved_gbs": vox * 4 / (ms / 1e3) / 1e9, "bytes_per_voxel": 4,
        "bound": "fp32 (the brush fold per voxel)",
        "cpu_baseline": {"value": cpu_vox / cs, "unit": "voxels/s", "cores": threads, "kind": "port",
                         "sample": "the same 64 brushes into a 96^3 x 3 volume"}}

    # 2. level sampling: sample(p, mip) and field(p, mip) of that volume at 4M device points
    field = ce.volumeField(vol)
    n = 1 << 22
    g = torch.Generator(device="cuda").manual_seed(7)
    lo = torch.tensor(origin, device="cuda")
    pts = (torch.rand(n, 3, device="cuda", generator=g) * 24.0 + lo).contiguous()
    sxy = torch.empty(n, 2, device="cuda")
    fxy = torch.empty(n, 2, device="cuda")
    dist, mat = vol.download()
    ovd = oracle.VolumeData(192, vol.mipLevels, origin, 24.0, 4.0, dist=dist, mat=mat)
    ofield = oracle.make_field([ovd])
    hp = pts[: 1 << 18].cpu().numpy()
    levels = {}
    for m in range(vol.mipLevels):
        field.query_mip_device(pts, sxy, fxy, m, stream)
        ms = _event_ms(stream, lambda: field.query_mip_device(pts, sxy, fxy, m, stream), 5) / 5
        cs = _cpu_s(lambda: oracle.field_query_mip_batch(ofield, hp, m, threads=threads))
        levels[str(m)] = {"value": n / (ms / 1e3), "ms": ms, "achieved_gbs": n * 28 / (ms / 1e3) / 1e9,
                          "cpu_value": len(hp) / cs}
    out["field_sample_mip"] = {
        "workload": f"4,194,304 uniform points over the 192^3 volume, levels 0..{vol.mipLevels - 1}",
        "unit": "samples/s", "bytes_per_sample": 28, "bound": "L2/L1 latency of the trilinear gathers",
        "levels": levels, "cpu_baseline": {"unit": "samples/s", "cores": threads, "kind": "port",
                                           "sample": "262,144 of the points per level"}}

    # 3. SurfaceExtractor: the config-3 clay body (sphere r = 0.95) from a 64^3 bake of it, at the
    # game's lattice (32^3) and at 128^3
    box = 32 * 0.083
    bo = (-box / 2,) * 3
    sv = ce.SdfVolume(root, resolution=64, worldSize=box, origin=bo, mipLevels=1)
    sv.build(B.make_brush("sphere", pos=(0.0, 0.0, 0.0), size=0.95))
    sfield = ce.volumeField(sv)
    sd, smat = sv.download()
    sofield = oracle.make_field([oracle.VolumeData(64, 1, bo, box, 4.0, dist=sd, mat=smat)])
    ext = {}
    for res in (32, 128):
        cap = 65536
        parts = torch.zeros(cap * 96, dtype=torch.uint8, device="cuda")
        bodies = torch.zeros(64, dtype=torch.uint8, device="cuda")
        x = ce.SurfaceExtractor(root, parts, cap, bodies, 1, sfield, 0, 0, cap, resolution=res)
        x.setRegion(bo, box)
        x.extract(stream)
        reps = 50 if res == 32 else 10
        ms = _event_ms(stream, lambda: x.extract(stream), reps) / reps
        nv = int(x.counts(stream)[0])
        hpart = np.zeros(cap, scenes.PARTICLE_RECORD)
        hbody = np.zeros(1, scenes.BODY_RECORD)
        cs = _cpu_s(lambda: oracle.extract(sofield, hpart, hbody, res, 0, 0, cap, bo, box))
        ext[str(res)] = {"cells": res ** 3, "particles": nv, "ms_per_extract": ms, "value": res ** 3 / (ms / 1e3),
                         "achieved_gbs": (nv * 96 + res ** 3 * 36) / (ms / 1e3) / 1e9, "cpu_value": res ** 3 / cs}
        x.destroy()
    out["extract"] = {"workload": "surface nets of the clay-body sphere (r 0.95) over its 2.656 m box",
                      "unit": "lattice cells/s", "bytes": "96 B per particle + 36 B scratch per cell",
                      "bound": "field samples (8 + 9 per vertex cell, 4 per lattice point)", "lattices": ext,
                      "cpu_baseline": {"unit": "lattice cells/s", "cores": 1, "kind": "port", "sample": "the same"}}

    # 4. ClaySolver: 86 clay bodies (config 3's shell, 3,800 particles each) over a config-3
    # collider, default options (2 substeps)
    shell, shell_n = scenes.surface_net_sphere(0.95, 0.067)
    wv = ce.SdfVolume(root, resolution=64, worldSize=24.0, origin=scenes.WORLD_ORIGIN)
    wbr = scenes.random_brushes(8, seed=99, lo=(-10, -3.5, -10), hi=(10, 1.0, 10))
    wv.build(wbr)
    world = ce.volumeField(wv)
    rng = np.random.default_rng(5)
    centers = [(float(a), 2.5, float(c)) for a, c in rng.uniform(-9, 9, (86, 2))]
    hparts, hbodies = body_set(shell, shell_n, centers)
    dparts = torch.from_numpy(hparts.view(np.uint8).copy()).cuda()
    dbodies = torch.from_numpy(hbodies.view(np.uint8).copy()).cuda()
    solver = ce.ClaySolver(root, dparts, len(hparts), dbodies, len(hbodies), world)
    for _ in range(3):
        solver.step(len(hbodies), stream)
    frames = 20
    ms = _event_ms(stream, lambda: solver.step(len(hbodies), stream), frames) / frames
    npart = len(hparts)
    wd, wm = wv.download()
    wfield = oracle.make_field([oracle.VolumeData(64, wv.mipLevels, scenes.WORLD_ORIGIN, 24.0, 4.0, dist=wd, mat=wm)])
    sp, sb = body_set(shell, shell_n, centers[:8])
    cfg = oracle.solver_cfg(len(sp), len(sb))
    cs = _cpu_s(lambda: oracle.solver_step(cfg, wfield, sp, sb, len(sb)))
    # per particle and substep: predict reads the record (96 B) and writes pos + prev (24 B),
    # match reads pos + rest twice (48 B), apply reads the record and writes pos (+ prev) (120 B),
    # finalize reads pos, prev, vel (36 B) and writes vel, velPrev (24 B)
    per = 96 + 24 + 48 + 96 + 24 + 36 + 24
    out["solver"] = {"workload": f"86 bodies x {len(shell)} particles, 2 substeps, 2 rotation iterations",
                     "value": npart / (ms / 1e3), "unit": "particle-steps/s", "ms_per_step": ms,
                     "achieved_gbs": npart * 2 * per / (ms / 1e3) / 1e9, "bytes_per_particle_substep": per,
                     "launches_per_step": 8,
                     "cpu_baseline": {"value": len(sp) / cs, "unit": "particle-steps/s", "cores": 1, "kind": "port",
                                      "sample": f"8 of the bodies ({len(sp)} particles), 1 step"}}
    solver.destroy()
    for f in (world, sfield, field):
        f.destroy()
    for v in (wv, sv, vol):
        v.destroy()
    return out


def _tap_world(root, seed):
    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    cfg = scenes.CONFIG2
    vol = ce.SdfVolume(root, resolution=cfg["collider"]["resolution"], worldSize=24.0, origin=scenes.WORLD_ORIGIN)
    vol.build(scenes.random_brushes(64, seed=seed))
    return vol, ce.volumeField(vol)


def run_tap(root, stream, seed, frames, warmup):
    """The plain method at scale (one scene of capacity 262,144 over a 192^3 collider of 64
    seeded brushes, baked into 128^3 x 4, band 4), fed each frame by spawn(4096) at a tap with
    a downward speed ~ N(2, 0.3) (one speed per spawn: the reference emits one velocity per
    spawn). `frames` timed frames from an empty ring (it fills at frame 64, then wraps), each one
    FluidSim.step on one stream (no graph), after `warmup` frames of a separate sim."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    cfg = scenes.CONFIG2
    tap = cfg["tap"]
    vol, world = _tap_world(root, seed)
    rng = np.random.default_rng(seed)

    def frame(sim):
        sim.spawn(tap["n"], tap["pos"], (0.0, -float(rng.normal(*tap["speed"])), 0.0))
        sim.step(stream)
        return sim.particleCount

    warm = ce.FluidSim(root, world, cfg["fluid"])
    for _ in range(warmup):
        frame(warm)
    stream.synchronize()
    warm.destroy()
    sim = ce.FluidSim(root, world, cfg["fluid"])
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ce.kernel_launch_count()
    live_sum = 0
    a.record(stream)
    for _ in range(frames):
        live_sum += frame(sim)
    z.record(stream)
    z.synchronize()
    ms = a.elapsed_time(z)
    out = {"value": live_sum / (ms / 1000), "ms_per_step": ms / frames, "frames": frames,
           "gpu_launches": ce.kernel_launch_count() - l0, "live_at_end": sim.particleCount,
           "particle_steps": live_sum}
    sim.destroy()
    world.destroy()
    vol.destroy()
    return out


def run_small(root, stream, frames, warmup):
    """The plain method, small: 4,096 particles (a 16^3 jittered lattice of spacing 0.1 at
    y = 3, seed 1) over the 96^3 rounded-box collider, 2 substeps, a 64^3 x 3 bake, one
    FluidSim.step per frame on one stream."""
    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    cfg = scenes.CONFIG1
    vol = ce.SdfVolume(root, resolution=cfg["collider"]["resolution"], worldSize=24.0, origin=scenes.WORLD_ORIGIN)
    vol.build(scenes.config1_collider_brushes())
    world = ce.volumeField(vol)
    sim = ce.FluidSim(root, world, cfg["fluid"])
    sim.upload(scenes.jittered_lattice(16, 0.1, (0.0, 3.0, 0.0), 1))
    for _ in range(warmup):
        sim.step(stream)
    stream.synchronize()
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(frames):
        sim.step(stream)
    z.record(stream)
    z.synchronize()
    ms = a.elapsed_time(z)
    out = {"value": 4096 * frames / (ms / 1000), "ms_per_step": ms / frames, "frames": frames}
    sim.destroy()
    world.destroy()
    vol.destroy()
    return out


def cpu_small(threads, frames=20):
    """The oracle on the small configuration: the same 4,096 particles, `frames` frames."""
    from clay_engine_b200 import scenes
    from oracle import oracle
    from oracle.fluid_frame import OracleFluid

    oracle.build()
    cfg = scenes.CONFIG1
    vd = oracle.VolumeData(96, 3, scenes.WORLD_ORIGIN, 24.0, 4.0)
    d, m = oracle.build_brushes(vd, scenes.config1_collider_brushes(), threads=threads)
    vd.dist[:], vd.mat[:] = d, m
    ref = OracleFluid(oracle, [vd], threads=threads, **cfg["fluid"])
    ref.upload(scenes.jittered_lattice(16, 0.1, (0.0, 3.0, 0.0), 1))
    t0 = time.perf_counter()
    for _ in range(frames):
        ref.step()
    sec = time.perf_counter() - t0
    return {"value": 4096 * frames / sec, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the same 4,096 particles, {frames} frames"}


def cpu_tap(threads, seed, frames=2):
    """The oracle on the tap at scale with its ring full: 262,144 - 2,048 particles piled on the
    same 64-brush collider, then `frames` frames of spawn(4096) + step (the first one wraps)."""
    from clay_engine_b200 import scenes
    from oracle import oracle
    from oracle.fluid_frame import OracleFluid

    oracle.build()
    cfg = scenes.CONFIG2
    tap = cfg["tap"]
    vd = oracle.VolumeData(192, 4, scenes.WORLD_ORIGIN, 24.0, 4.0)
    d, m = oracle.build_brushes(vd, scenes.random_brushes(64, seed=seed), threads=threads)
    vd.dist[:], vd.mat[:] = d, m
    ref = OracleFluid(oracle, [vd], threads=threads, **cfg["fluid"])
    p = scenes.lattice_block(262144 - 2048, 0.1, (0.0, -1.0, 0.0), 21)
    p["vel"] = (0.0, -tap["speed"][0], 0.0)
    ref.upload(p)
    rng = np.random.default_rng(seed)
    steps = 0
    t0 = time.perf_counter()
    for _ in range(frames):
        ref.spawn(tap["n"], tap["pos"], (0.0, -float(rng.normal(*tap["speed"])), 0.0))
        ref.step()
        steps += ref.live
    sec = time.perf_counter() - t0
    return {"value": steps / sec, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{frames} frames of the full ring (262,144 particles), spawn(4096) each"}


# The CPU sample both arms time: the 131 batched scenes nearest the median size (1.48 M
# particles at the benchmark's seed), ~1.8 s per rep on 16 host cores.
CPU_SAMPLE_PARTICLES = 1_500_000


def reference_arm(args, ws, rank):
    """--impl reference: the oracle (the reference's algorithm restated on the CPU; the reference
    itself is WebGPU/TypeScript and cannot run here) timed on all host cores, on the same sample
    the other arm's cpu_baseline times: W untimed reps, then K timed ones."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sample = CpuSample(args.scenes, 3, CPU_SAMPLE_PARTICLES, threads)
    for _ in range(args.warmup):
        sample.rep()
    sec = sum(sample.rep() for _ in range(args.steps))
    value = sample.particles * args.steps / sec
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sec / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched-256-scenes (bounded CPU sample)", "scenes": args.scenes,
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample.desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------

def load_peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# Algorithmic bytes per particle and substep of the neighbour passes (the compulsory DRAM
# traffic if every input were read once and every output written once; neighbour re-reads
# are cache reuse and the neighbour list is an intermediate, neither is counted).
BYTES_PER_PARTICLE = {
    "density": 16 + 16 + 16 + 4,  # pos in; density record, neighbour view (pos, 1/density), pressure out
    "forces_integrate": 16 + 16 + 16 + 4 + 48,  # pos, vel, density record, id in; particle record out
}
# DRAM bytes (read + written) per particle of one k_splat launch over the fluid surfaces (3
# levels), from one ncu capture of that launch in the 128-scene batch (dram__bytes_read.sum +
# dram__bytes_write.sum): 107,473,408 + 5,515,008 bytes for 1,940,550 particles.
SPLAT_TRAFFIC_PER_PARTICLE = (107473408 + 5515008) / 1940550


def main():
    args = parse()
    from clay_engine_b200 import dist as D

    ws, rank, local = D.init("nccl")
    if args.impl == "reference":
        reference_arm(args, ws, rank)
        D.finalize()
        return

    import torch

    import clay_engine_b200 as ce
    from clay_engine_b200 import scenes

    torch.cuda.set_device(local)
    root = ce.init(local)
    if args.workload == "tap":
        stream = torch.cuda.Stream()
        with ClockSampler(local) as clocks:
            clocks.mark()
            r = run_tap(root, stream, D.rank_seed(11, rank), args.steps, args.warmup)
            clocks.stop()
        value = D.reduce_sum(r["value"])
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                              "config": {"workload": "plain-scale-262144-tap", "collider": "192^3 from 64 brushes",
                                         "bake": "128^3 x 4 mips band 4", "tap": "spawn(4096)/frame, speed N(2,0.3)",
                                         "live_at_end": r["live_at_end"]},
                              "gpu_launches": r["gpu_launches"], "clocks": clocks.summary()}), flush=True)
        root.destroy()
        D.finalize()
        return
    n_scenes = 16 if args.small else args.scenes
    seed = D.rank_seed(3, rank)
    sims, bodies, keep = build_scenes(root, n_scenes, seed)
    particles = sum(s.particleCount for s in sims)
    stream = torch.cuda.Stream()
    # autotune (untimed): per scene-size bucket, the particle passes' block size, the density
    # variant and the splat's strategy thresholds
    from clay_engine_b200 import autotune

    t_tune = time.perf_counter()
    if args.no_tune:
        n_b = len(autotune.BUCKETS) + 1
        fixed = dict(autotune.DEFAULT)
        for kv in args.set:
            k, v = kv.split("=")
            if k not in autotune.KNOBS and k != "lanes":
                raise SystemExit(f"--set: unknown knob {k}")
            fixed[k] = int(v)
        lanes = int(fixed.pop("lanes", autotune.DEFAULT_LANES))
        tuned = {"uppers": list(autotune.BUCKETS), "tunings": [dict(fixed) for _ in range(n_b)], "lanes": lanes,
                 "changed": [{k: v for k, v in fixed.items() if v != autotune.DEFAULT[k]}] if fixed != autotune.DEFAULT
                 else [], "gain": 0.0}
        tune_report = {"trials": []}
    else:
        tuned, tune_report = autotune.tune(root, sims, bodies, stream, frames=10, use_cache=False)
    t_tune = time.perf_counter() - t_tune
    batch = ce.Batch(root, sims, extra_splats=bodies, use_graph=True, sph_block=tuned["tunings"][-1]["sph_block"])
    autotune.apply(batch, tuned)
    torch.cuda.synchronize()
    clocks = ClockSampler(local).__enter__()

    # warm-up (also captures the graph)
    for _ in range(max(args.warmup, 1)):
        batch.step(stream)
    stream.synchronize()
    # the state the timed frames start from: the end-to-end frames start from it too, so both
    # measure the same frames (a fluid's cost changes as it falls and spreads)
    start_state = [s.download() for s in sims]

    # ---- device-resident throughput: K batched frames, CUDA events on the launching stream
    l0 = ce.kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    D.barrier()
    torch.cuda.synchronize()
    clocks.mark()
    # the timed frames sit in an NVTX range "timed", so a profiler can capture exactly them
    torch.cuda.nvtx.range_push("timed")
    ev0.record(stream)
    for _ in range(args.steps):
        batch.step(stream)
    ev1.record(stream)
    torch.cuda.nvtx.range_pop()
    ev1.synchronize()
    clocks.stop()
    torch.cuda.synchronize()
    D.barrier()
    launches = ce.kernel_launch_count() - l0
    ms = D.reduce_max(ev0.elapsed_time(ev1))
    total_particles = D.reduce_sum(particles)
    value = total_particles * args.steps / (ms / 1000)

    # ---- end to end through the public API: per frame the inputs (every scene's FluidParams)
    # go up from pinned memory and every scene's ContactList comes back to pinned memory. The
    # host keeps one frame in flight ahead of the one it reads (two pinned contact buffers, the
    # batch's parameter staging is double-buffered too): it waits for frame i's contacts after
    # issuing frame i + 1, so its own work overlaps the device's.
    h_contacts = [torch.empty(len(sims) * 528, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    done = [torch.cuda.Event(), torch.cuda.Event()]
    for s, st in zip(sims, start_state):
        s.upload(st)
    D.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(2, args.steps)  # the same frames as the device-resident timing
    e0.record(stream)
    for i in range(e2e_steps):
        batch.step(stream)
        batch.read_contacts_async(h_contacts[i % 2].data_ptr(), stream)
        done[i % 2].record(stream)
        if i > 0:
            done[(i - 1) % 2].synchronize()  # frame i - 1's contacts are on the host
    done[(e2e_steps - 1) % 2].synchronize()
    e1.record(stream)
    e1.synchronize()
    D.barrier()
    e2e_ms = D.reduce_max(e0.elapsed_time(e1))
    e2e_value = total_particles * e2e_steps / (e2e_ms / 1000)

    # the clock sampler's window closed with the timed frames; stop its thread before the
    # per-launch profile, whose event pairs would otherwise also time its NVML queries' stalls
    clocks.__exit__(None, None, None)
    prof = batch.profile(stream)
    frame_ms = sum(v[0] for v in prof.values())

    # ---- plain path: the same scenes, one scene per launch sequence, no graph
    plain_value = None
    if args.plain_steps > 0:
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for s in sims[:4]:
            s.step(stream)
        p0.record(stream)
        for _ in range(args.plain_steps):
            for s in bodies:
                s.bake(stream)
            for s in sims:
                s.step(stream)
        p1.record(stream)
        p1.synchronize()
        plain_ms = D.reduce_max(p0.elapsed_time(p1))
        plain_value = total_particles * args.plain_steps / (plain_ms / 1000)

    clk = clocks.summary()
    # ---- census of the frame's algorithmic work (untimed): neighbour candidates and accepted
    # pairs of the last substep, the bake's in-band (particle, voxel) pairs, per scene
    cand = acc = pairs = 0
    for s in sims:
        c = s.census(stream)
        cand += c["candidates"]
        acc += c["accepted"]
        pairs += c["splat_pairs"]
    body_pairs = sum(b.census(stream) for b in bodies)
    # algorithmic bytes of the bake: each (particle, level) reads its 16-byte position once; each
    # voxel the bake lowers is read and written once in the key grid (8 B)
    touched = 0
    for s in sims:
        d, _ = s.surface.volume.download()
        touched += int((d != 0x3C00).sum())
    mips = sims[0].surface.volume.mipLevels if sims else 0
    n_sims = len(sims)
    splat_bytes = 16 * particles * mips + 8 * touched
    # ---- roofline of the dominant kernel, k_splat (its fluid-surface launch "splat": the
    # SplatField bake of every fluid), from the per-launch event times of one frame
    peak, peak_kind = load_peaks()
    # FP32 issue peak at the clock seen during the timed frames: 148 SMs x 128 FP32 lanes
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    lane_peak = sms * 128 * mhz * 1e6
    splat_ms, splat_launches = prof.get("splat", (None, 0))
    roof = {"bound": "hbm", "kernel": "k_splat (fluid surfaces)", "achieved": None, "peak": peak, "unit": "GB/s",
            "frac": None, "traffic": None, "peak_source": peak_kind}
    if splat_ms:
        avg_ms = splat_ms / splat_launches
        achieved = splat_bytes / (avg_ms / 1000) / 1e9
        roof.update({"achieved": round(achieved, 2), "frac": achieved / peak,
                     "traffic": SPLAT_TRAFFIC_PER_PARTICLE * particles,
                     "algorithmic_bytes_per_launch": splat_bytes, "avg_launch_ms": round(avg_ms, 4)})
    # compute roofline (the kernels are issue-bound): algorithmic FP32 operations of the
    # reference's work per second against the FP32 lane-issue peak. k_splat: 9 per in-band pair
    # (3 sub, 3 mul, 2 add, 1 compare); k_density: 9 per candidate + 13 per accepted pair (the
    # kernel term and the sum), over both substeps (the census counts the last one)
    comp = {"unit": "FP32 lane-ops/s", "peak": lane_peak, "peak_source": f"{sms} SMs x 128 lanes x {mhz:.0f} MHz"}
    if splat_ms:
        ops = 9 * pairs
        comp["k_splat"] = {"pairs": pairs, "pairs_per_s": pairs / (splat_ms / 1000), "ops_per_pair": 9,
                           "frac": ops / (splat_ms / 1000) / lane_peak}
    body_ms = prof.get("body_splat", (None, 0))[0]
    if body_ms and body_pairs:
        comp["k_splat_bodies"] = {"pairs": body_pairs, "pairs_per_s": body_pairs / (body_ms / 1000),
                                  "frac": 12 * body_pairs / (body_ms / 1000) / lane_peak, "ops_per_pair": 12}
    if "density" in prof:
        dms = prof["density"][0]
        ops = 2 * (9 * cand + 13 * acc)
        comp["k_density"] = {"candidates": 2 * cand, "accepted": 2 * acc, "candidates_per_s": 2 * cand / (dms / 1000),
                             "frac": ops / (dms / 1000) / lane_peak}
    roof["compute"] = comp
    # the neighbour passes against the HBM peak (one launch per block-size group and substep)
    others = {}
    for name, per in BYTES_PER_PARTICLE.items():
        if name in prof:
            ms_k, n_k = prof[name]
            byt = per * particles * 2 / max(n_k, 1)  # 2 substeps spread over the launches
            others[name] = {"achieved_gbs": round(byt / (ms_k / n_k / 1000) / 1e9, 2),
                            "avg_launch_ms": round(ms_k / n_k, 4)}
    roof["neighbour_passes"] = others

    # ---- serving: free the batched scenes first, then a resident pool under Poisson arrivals
    batch.destroy()
    for s in sims:
        s.destroy()
    for x in bodies:
        x.destroy()
    sims, bodies, keep = [], [], []
    served = None
    if not args.no_serve and not args.small:
        served = run_serving(root, args, seed + 50, stream)
    threads = os.cpu_count() or 1
    # ---- the plain configurations (small, and the tap at scale over its 120 frames)
    configs = None
    if rank == 0 and ws == 1 and not args.small:
        small = run_small(root, stream, 120, max(args.warmup, 3))
        tap = run_tap(root, stream, 11, scenes.CONFIG2["steps"], max(args.warmup, 3))
        configs = {"small_4096": small, "tap_262144": tap}
        if not args.no_cpu:
            small["cpu_baseline"] = cpu_small(threads)
            tap["cpu_baseline"] = cpu_tap(threads, 11)
    next_rows = None
    if rank == 0 and ws == 1 and not args.small and not args.no_next:
        next_rows = measure_next_rows(root, stream, threads)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        sample = CpuSample(n_scenes, seed, CPU_SAMPLE_PARTICLES, threads)
        sample.rep()  # warm
        reps = 2
        sec = sum(sample.rep() for _ in range(reps))
        cpu = {"value": sample.particles * reps / sec, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": sample.desc + f", {reps} reps"}
        # the same oracle on one core, on a smaller sample (~10 s)
        one = CpuSample(n_scenes, seed, 120_000, 1)
        cpu["one_core"] = {"value": one.particles / one.rep(), "cores": 1, "sample": f"{one.particles} particles"}

    if rank == 0:
        # The details first, on a line of their own that is not JSON (the rows after the frame,
        # the per-kernel times, the full serving and tuning records) ...
        detail = {"kernels_ms_per_frame": {k: round(v[0], 4) for k, v in prof.items()},
                  "frame_ms_unfused": frame_ms, "served": served, "next_rows": next_rows,
                  "autotune_trials": tune_report.get("trials", []), "census": {
                      "particles": particles, "candidates_last_substep": cand, "accepted_last_substep": acc,
                      "splat_pairs": pairs, "body_splat_pairs": body_pairs}}
        print("# detail " + json.dumps(detail), flush=True)
        # ... then the one JSON line, kept short enough to be read whole from the tail of the
        # output, with the metric's own terms (plain, served) at its end
        def r3(x):
            return None if x is None else float(f"{x:.4g}")

        srv = None
        if served:
            srv = {"throughput": r3(served["throughput"]), "p50_ms": r3(served["p50_ms"]),
                   "p99_ms": r3(served["p99_ms"]), "rate_req_s": served["rate_req_s"],
                   "demand": r3(served["demand_particle_steps_s"]), "completed": served["completed"]}
            if "below_capacity" in served:
                bc = served["below_capacity"]
                srv["below_capacity"] = {"rate_req_s": r3(bc["rate_req_s"]), "throughput": r3(bc["throughput"]),
                                         "p50_ms": r3(bc["p50_ms"]), "p99_ms": r3(bc["p99_ms"])}
        cfgs = None
        if configs:
            cfgs = {k: {"value": r3(v["value"]), "ms_per_step": r3(v["ms_per_step"]), "frames": v["frames"],
                        "cpu": r3(v.get("cpu_baseline", {}).get("value"))} for k, v in configs.items()}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched-256-scenes" if not args.small else "batched-16-scenes",
                       "scenes_per_gpu": n_scenes, "particles_per_gpu": particles, "substeps": 2,
                       "bake": "64^3x3 band 4 (+32^3x2 bodies)", "collider": "64^3, 8 brushes",
                       "parallelism": f"{ws} GPU(s), independent scenes", "cuda_graph": True,
                       "l2": "working set > L2, no flush"},
            "gpu_launches": int(launches),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 80 * n_sims * ws,
                    "d2h_bytes_per_step": 528 * n_sims * ws},
            "clocks": clk,
            "cpu_baseline": cpu,
            "roofline": roof,
            "autotune": {"changed": tuned["changed"], "lanes": tuned.get("lanes", 1), "gain": r3(tuned["gain"]),
                         "trials": len(tune_report.get("trials", []))},
            "configs": cfgs,
            "plain": {"value": plain_value, "ratio_batched_over_plain": (value / plain_value) if plain_value else None},
            "served": srv,
        }
        print(json.dumps(line), flush=True)

    root.destroy()
    D.finalize()


if __name__ == "__main__":
    main()
