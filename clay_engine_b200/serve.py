"""Continuous-batching server for step-and-bake requests over device-resident scenes.

A request asks one scene to advance `k` frames (each frame: FluidSim.step, i.e. the substeps
and the SplatField bake) and is done when its last frame has completed on the device. The
server keeps every admitted scene's particles, grids and volumes resident in HBM and, every
frame, launches one batched step (`Batch.step_subset`) over the scenes that have a request in
progress. Requests that arrive while frames are on the GPU join at the next frame boundary,
so their work overlaps with requests already in flight; frames are enqueued up to `depth`
ahead of the device.

Admission is by an HBM budget: a scene is made resident only when its estimated bytes fit
beside the scenes already resident; otherwise idle scenes are evicted least-recently-used
first (their particle state is kept on the host and restored when they return), and a
request whose scene cannot be admitted waits until memory frees up.

Latency of a request = device completion time of its last frame - its arrival time, both on
one clock: the host clock at the start is tied to a CUDA event recorded on the idle stream.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

from .core import Batch


@dataclass
class Request:
    rid: int
    scene: int
    k: int
    t_arrival: float
    remaining: int = 0
    t_done: float | None = None
    particles: int = 0


@dataclass
class ServeStats:
    completed: int = 0
    particle_steps: float = 0.0
    frames: int = 0
    scene_frames: int = 0
    latencies: list = field(default_factory=list)
    t_first: float = 0.0
    t_last: float = 0.0
    evictions: int = 0
    admissions: int = 0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies) if self.latencies else np.zeros(1)
        span = max(self.t_last - self.t_first, 1e-9)
        return {"completed": self.completed, "throughput": self.particle_steps / span,
                "p50_ms": float(np.percentile(lat, 50) * 1000), "p99_ms": float(np.percentile(lat, 99) * 1000),
                "mean_ms": float(lat.mean() * 1000), "frames": self.frames,
                "mean_batch": self.scene_frames / max(self.frames, 1), "window_s": span,
                "evictions": self.evictions, "admissions": self.admissions}


def poisson_arrivals(rate, duration, n_scenes, k_lo, k_hi, seed):
    """(t, scene, k) sorted by t: Poisson arrivals at `rate` per second over `duration` s."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        out.append((t, int(rng.integers(0, n_scenes)), int(rng.integers(k_lo, k_hi + 1))))
    return out


class Server:
    """`factory(i)` creates scene i on the device and returns (FluidSim, keepalive list);
    `estimate(i)` is its device bytes (used for admission before creating it)."""

    def __init__(self, root, factory, estimate, n_scenes, budget_bytes, depth=2, max_batch=1 << 30,
                 sph_block=256):
        self.root = root
        self.factory = factory
        self.estimate = estimate
        self.n_scenes = n_scenes
        self.budget = budget_bytes
        self.depth = depth
        self.max_batch = max_batch
        self.sph_block = sph_block
        self.resident = collections.OrderedDict()  # scene -> (sim, keep, bytes); LRU order
        self.snapshots = {}
        self.batch = None
        self.index = {}
        self.dirty = True
        self.stats = ServeStats()
        self.busy = set()

    # -- residency ---------------------------------------------------------------------------
    def used_bytes(self) -> int:
        return sum(v[2] for v in self.resident.values())

    def admit(self, scene) -> bool:
        if scene in self.resident:
            self.resident.move_to_end(scene)
            return True
        need = self.estimate(scene)
        if need > self.budget:
            raise MemoryError(f"scene {scene} needs {need} bytes, over the {self.budget}-byte budget")
        while self.used_bytes() + need > self.budget:
            victim = next((s for s in self.resident if s not in self.busy), None)
            if victim is None:
                return False
            self.evict(victim)
        before = self.root.bytes_in_use()
        sim, keep = self.factory(scene)
        if scene in self.snapshots:
            sim.upload(self.snapshots.pop(scene))
        self.resident[scene] = (sim, keep, self.root.bytes_in_use() - before)
        self.stats.admissions += 1
        self.dirty = True
        return True

    def evict(self, scene):
        import torch

        sim, keep, _ = self.resident.pop(scene)
        torch.cuda.synchronize()  # its last frame may still be running on the serving stream
        self.snapshots[scene] = sim.download()
        sim.destroy()
        for x in keep:
            if hasattr(x, "destroy"):
                x.destroy()
        self.stats.evictions += 1
        self.dirty = True

    def _rebuild(self):
        if self.batch is not None:
            self.batch.destroy()
        order = list(self.resident)
        self.index = {s: i for i, s in enumerate(order)}
        self.batch = Batch(self.root, [self.resident[s][0] for s in order], sph_block=self.sph_block, use_graph=False)
        self.dirty = False

    def sim(self, scene):
        return self.resident[scene][0]

    # -- the request loop --------------------------------------------------------------------
    def serve(self, arrivals, stream, timeout_s=600.0):
        """Runs until every arrival (t, scene, k) has completed. Returns the requests."""
        import torch

        reqs = [Request(i, s, k, t) for i, (t, s, k) in enumerate(arrivals)]
        for r in reqs:
            r.remaining = r.k
        waiting = collections.defaultdict(collections.deque)
        active = {}
        inflight = collections.deque()
        nxt = 0
        done = 0
        stream.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ev0.synchronize()
        t0 = time.perf_counter()
        self.stats.t_first = reqs[0].t_arrival if reqs else 0.0
        while done < len(reqs):
            now = time.perf_counter() - t0
            if now > timeout_s:
                raise TimeoutError(f"serving did not finish within {timeout_s} s ({done}/{len(reqs)} done)")
            while nxt < len(reqs) and reqs[nxt].t_arrival <= now:
                waiting[reqs[nxt].scene].append(reqs[nxt])
                nxt += 1
            # activate the head request of every waiting scene whose scene can be resident
            for scene in list(waiting):
                if scene in active or not waiting[scene]:
                    continue
                if self.admit(scene):
                    r = waiting[scene].popleft()
                    r.particles = self.sim(scene).particleCount
                    active[scene] = r
                    self.busy.add(scene)
                if not waiting[scene]:
                    del waiting[scene]
            launched = False
            if active and len(inflight) < self.depth:
                if self.dirty:
                    stream.synchronize()
                    self._rebuild()
                scenes = list(active)[: self.max_batch]
                self.batch.step_subset([self.index[s] for s in scenes], stream)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(stream)
                finished = []
                for s in scenes:
                    r = active[s]
                    r.remaining -= 1
                    self.stats.particle_steps += r.particles
                    if r.remaining == 0:
                        finished.append(r)
                        del active[s]
                        self.busy.discard(s)
                inflight.append((ev, finished))
                self.stats.frames += 1
                self.stats.scene_frames += len(scenes)
                launched = True
            # retire completed frames
            while inflight and inflight[0][0].query():
                ev, finished = inflight.popleft()
                t = ev0.elapsed_time(ev) / 1000.0
                for r in finished:
                    r.t_done = t
                    self.stats.latencies.append(t - r.t_arrival)
                    self.stats.completed += 1
                    self.stats.t_last = max(self.stats.t_last, t)
                    done += 1
            if not launched:
                if inflight and len(inflight) >= self.depth:
                    inflight[0][0].synchronize()
                elif not active and nxt < len(reqs):
                    wait = reqs[nxt].t_arrival - (time.perf_counter() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.002))
                elif inflight:
                    inflight[0][0].synchronize()
        return reqs

    def close(self):
        if self.batch is not None:
            self.batch.destroy()
            self.batch = None
        for s in list(self.resident):
            sim, keep, _ = self.resident.pop(s)
            sim.destroy()
            for x in keep:
                if hasattr(x, "destroy"):
                    x.destroy()


def scene_bytes_estimate(n_particles, bake_res, bake_mips, grid_res, collider_res=64, collider_mips=3):
    """Device bytes of one scene as the library allocates them (FluidSim + surface + collider)."""
    per_particle = 48 + 4 * 4 + 16 + 16 + 16 + 4 * 64  # records, key/rank/tmp/id, spos, svel, sdp, neighbour list
    cells = grid_res ** 3
    bake = sum((bake_res >> m) ** 3 for m in range(bake_mips)) * (4 + 2 + 2)
    coll = sum((collider_res >> m) ** 3 for m in range(collider_mips)) * 4
    return int(n_particles * per_particle + (2 * cells + 3) * 4 + bake + coll + 4096)


def grid_res_for(world_size, h):
    return int(math.ceil(world_size / h)) + 2
