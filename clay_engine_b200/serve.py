"""Continuous-batching server for step-and-bake requests over device-resident scenes.

The scheduling loop is native (`clay_server_*` in include/clay_fluid.h): a request asks one
scene to advance `k` frames (each frame: FluidSim.step, i.e. the substeps and the SplatField
bake) and is done when its last frame has completed on the device. Every frame the server
launches one batched step over the scenes that have a request in progress; requests arriving
while frames run join at the next frame boundary, and up to `depth` frames are in flight.
Scenes become resident when a request needs them, within a device-byte budget: idle scenes are
evicted least-recently-used first (their particle state is kept on the host and restored when
they return). Latency of a request = device completion of its last frame - its submission,
on one clock (a CUDA event tied to the host's steady clock).

This module is the Python face of that server: scene registration from FluidSim options,
the replay of an arrival schedule (`serve`), and the latency statistics.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _native as N
from ._native import ClayError, check, lib, stream_handle
from .core import PARTICLE_DTYPE, FluidSim, fluid_estimate_bytes, fluid_options


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


def _check(rc):
    if rc == N.CLAY_ENOMEM:
        raise MemoryError(lib().clay_last_error().decode(errors="replace"))
    check(rc)


class Server:
    """A `clay_server`: scenes registered with `add_scene`, requests with `submit`."""

    def __init__(self, root, stream=None, budget_bytes=0, depth=2, max_batch=0, mode="fast", sph_block=0):
        o = N.ServerOpts(budget_bytes=int(budget_bytes), depth=int(depth), max_batch=int(max_batch),
                         mode=N.MODE_REFERENCE if mode == "reference" else N.MODE_FAST, sph_block=int(sph_block))
        h = C.c_void_p()
        self.stream = stream
        _check(lib().clay_server_create(root.handle, C.byref(o), stream_handle(stream), C.byref(h)))
        self.handle = h.value
        self.root = root
        self.budget = int(budget_bytes)
        self.tickets = []
        self.keep = []  # colliders of the registered scenes: they must outlive the server

    # -- scenes and requests ----------------------------------------------------------------
    def add_scene(self, world, options: dict, particles: np.ndarray | None = None, keep=()) -> int:
        o = fluid_options(options)
        a = np.ascontiguousarray(particles if particles is not None else np.zeros(0, PARTICLE_DTYPE), PARTICLE_DTYPE)
        sid = C.c_int32()
        _check(lib().clay_server_add_scene(self.handle, None if world is None else world.handle, C.byref(o),
                                           a.ctypes.data if len(a) else None, len(a), C.byref(sid)))
        self.keep += [world, *keep]
        return int(sid.value)

    def submit(self, scene: int, frames: int) -> int:
        t = C.c_int64()
        _check(lib().clay_server_submit(self.handle, int(scene), int(frames), C.byref(t)))
        self.tickets.append(int(t.value))
        return int(t.value)

    def pump(self) -> bool:
        launched = C.c_int32()
        _check(lib().clay_server_pump(self.handle, C.byref(launched)))
        return bool(launched.value)

    def wait(self, timeout_ms: float = -1.0):
        _check(lib().clay_server_wait(self.handle, float(timeout_ms)))

    def drain(self):
        _check(lib().clay_server_drain(self.handle))

    def poll(self, ticket: int):
        done, lat = C.c_int32(), C.c_double()
        _check(lib().clay_server_poll(self.handle, int(ticket), C.byref(done), C.byref(lat)))
        return bool(done.value), float(lat.value)

    def stats(self) -> dict:
        s = N.ServerStats()
        _check(lib().clay_server_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.ServerStats._fields_}

    def sim(self, scene: int) -> FluidSim | None:
        """The scene's FluidSim while resident (a view: the server owns it), else None."""
        h = C.c_void_p()
        _check(lib().clay_server_scene_sim(self.handle, int(scene), C.byref(h)))
        return None if not h.value else FluidSim(self.root, None, _handle=h.value)

    def download(self, scene: int) -> np.ndarray:
        """The scene's particles after all its submitted frames (resident or evicted)."""
        n = C.c_int64()
        _check(lib().clay_server_download(self.handle, int(scene), None, 0, C.byref(n)))
        out = np.zeros(int(n.value), PARTICLE_DTYPE)
        _check(lib().clay_server_download(self.handle, int(scene), out.ctypes.data if len(out) else None, len(out),
                                          C.byref(n)))
        return out

    # -- an arrival schedule ------------------------------------------------------------------
    def serve(self, arrivals, timeout_s=600.0) -> dict:
        """Replays `arrivals` [(t, scene, k)] (t in seconds from now, sorted): each request is
        submitted once its time has come, the server is pumped in between. Returns the
        statistics of these requests."""
        first = len(self.tickets)
        s0 = self.stats()
        t0 = time.perf_counter()
        nxt = 0
        while True:
            now = time.perf_counter() - t0
            if now > timeout_s:
                raise TimeoutError(f"serving did not finish within {timeout_s} s")
            while nxt < len(arrivals) and arrivals[nxt][0] <= now:
                self.submit(arrivals[nxt][1], arrivals[nxt][2])
                nxt += 1
            launched = self.pump()
            st = self.stats()
            if nxt == len(arrivals) and st["completed"] == st["submitted"]:
                break
            if launched:
                continue
            gap = (arrivals[nxt][0] - (time.perf_counter() - t0)) if nxt < len(arrivals) else None
            if st["inflight"] > 0:
                # wait on the device, but not past the next arrival
                self.wait(-1.0 if gap is None else max(0.0, min(gap, 0.005)) * 1000.0)
            elif gap is not None:
                time.sleep(max(0.0, min(gap, 0.002)))
            else:
                self.drain()  # raises when waiting scenes can never be admitted
        span = time.perf_counter() - t0
        lat = np.array([self.poll(t)[1] for t in self.tickets[first:]]) if len(self.tickets) > first else np.zeros(1)
        st = self.stats()
        return {"completed": st["completed"] - s0["completed"],
                "throughput": (st["particle_steps"] - s0["particle_steps"]) / max(span, 1e-9),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "frames": st["frames"] - s0["frames"],
                "mean_batch": (st["scene_frames"] - s0["scene_frames"]) / max(st["frames"] - s0["frames"], 1),
                "window_s": span, "evictions": st["evictions"] - s0["evictions"],
                "admissions": st["admissions"] - s0["admissions"]}

    def close(self):
        if self.handle:
            lib().clay_server_destroy(self.handle)
        self.handle = None


def scene_bytes_estimate(options: dict) -> int:
    """Device bytes of one scene's FluidSim (particles, grids, neighbour list, surface)."""
    return fluid_estimate_bytes(options)


def grid_res_for(world_size, h):
    return int(math.ceil(world_size / h)) + 2


__all__ = ["Server", "ClayError", "poisson_arrivals", "scene_bytes_estimate", "grid_res_for"]
