"""Autotuner: picks the thread-block size of the particle passes per scene-size bucket.

Scenes are grouped by capacity into buckets. For each bucket in turn (coordinate descent,
the other buckets held at their current choice), every candidate block size is timed over a
few real batched frames (CUDA graph replays, CUDA events on the launching stream) and the
fastest kept. The scenes' particle state is saved before tuning, restored before every
candidate (so all are timed from the same state) and after tuning, so tuning does not advance
the simulation. Results are cached per bucket signature in a JSON
file next to the library.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .core import Batch

BUCKETS = (4096, 16384, 65536)       # capacity < 4k, < 16k, < 64k, and the rest
CANDIDATES = (64, 128, 192, 256)
CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "autotune.json")


def bucket_index(capacity: int) -> int:
    for i, u in enumerate(BUCKETS):
        if capacity < u:
            return i
    return len(BUCKETS)


def signature(sims) -> str:
    counts = np.bincount([bucket_index(s.capacity) for s in sims], minlength=len(BUCKETS) + 1)
    # scenes per bucket rounded to a power of two: similar batches share a tuning
    return "b" + "-".join(str(1 << int(np.ceil(np.log2(c)))) if c else "0" for c in counts)


def _time(batch, stream, frames):
    import torch

    batch.step(stream)  # capture + warm
    stream.synchronize()
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(frames):
        batch.step(stream)
    z.record(stream)
    z.synchronize()
    return a.elapsed_time(z) / frames


def tune(root, sims, extra=(), stream=None, frames=8, use_cache=True, default=256, min_gain=0.02):
    """Returns ({"uppers": [...], "blocks": [...]}, report) for this set of scenes."""
    import torch

    stream = stream or torch.cuda.current_stream()
    sig = signature(sims)
    cache = {}
    if use_cache and os.path.exists(CACHE):
        try:
            with open(CACHE) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
    if use_cache and sig in cache:
        return cache[sig], {"cached": True, "signature": sig}
    present = sorted({bucket_index(s.capacity) for s in sims})
    choice = {i: default for i in range(len(BUCKETS) + 1)}
    snaps = [s.download() for s in sims]
    report = {"signature": sig, "trials": []}
    try:
        for bi in present:
            times = {}
            for cand in CANDIDATES:
                choice[bi] = cand
                # every candidate is timed from the same state (stepping moves the fluid, and a
                # later, more spread-out state would cost more whatever the block size)
                for s, snap in zip(sims, snaps):
                    s.upload(snap)
                batch = Batch(root, sims, extra_splats=extra, sph_block=choice[len(BUCKETS)], use_graph=True)
                batch.set_bucket_blocks(list(BUCKETS), [choice[i] for i in range(len(BUCKETS))])
                ms = _time(batch, stream, frames)
                batch.destroy()
                times[cand] = ms
                report["trials"].append({"bucket": bi, "block": cand, "ms": ms})
            # keep the default unless a candidate beats it by more than the timing noise
            best_b = min(times, key=times.get)
            if times[best_b] > times[default] * (1.0 - min_gain):
                best_b = default
            choice[bi] = best_b
    finally:
        torch.cuda.synchronize()
        for s, snap in zip(sims, snaps):
            s.upload(snap)
    result = {"uppers": list(BUCKETS), "blocks": [choice[i] for i in range(len(BUCKETS))],
              "default": choice[len(BUCKETS)]}
    if use_cache:
        cache[sig] = result
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        with open(CACHE, "w") as f:
            json.dump(cache, f, indent=1)
    return result, report


def apply(batch, result):
    batch.set_bucket_blocks(result["uppers"], result["blocks"])
