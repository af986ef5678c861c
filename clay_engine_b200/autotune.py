"""Autotuner: picks, per scene-size bucket, the launch shapes and strategies of the frame.

Scenes are grouped by capacity into buckets. The knobs of a bucket are the thread-block size of
the particle passes, the density pass's variant (one loop; distance tests then the accepted
neighbours; one loop over neighbours staged in shared memory) and the splat's strategy thresholds (how much larger than the particles' own voxel
boxes a block's union box may be and still take the register-blocked tile walk, or the block
walk); the batch as a whole also picks how many lanes (groups of scenes whose chains of
launches run side by side) it steps. Every setting gives the same results (reference mode bit for bit); they only move time
between code paths, so the choice is a pure timing decision.

Search: coordinate descent, knob after knob, first for every bucket at once (a setting that
differs between buckets splits a pass into one launch per distinct setting, which costs a
little by itself, so a knob is first tried without that cost), then bucket after bucket. A
candidate is timed over real batched frames (CUDA graph replays, CUDA events on the launching
stream) from the same saved particle state, between two timings of the current choice, and
replaces it only when it is faster than their mean by more than `min_gain` of the frame, so a
slow drift of the GPU's speed over the search cannot pass for a gain. The scenes' state is
restored after tuning, so tuning does not advance the simulation. Results are cached per
bucket signature in a JSON file next to the library.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .core import Batch

BUCKETS = (4096, 16384, 65536)       # capacity < 4k, < 16k, < 64k, and the rest
KNOBS = {
    "sph_block": (64, 128, 192, 256),
    "density_variant": (0, 1, 2),
    "splat_tile_ratio": (3, 6, 12),
    "splat_walk_weight": (2, 3, 6),
    "forces_split": (0, 1),
}
DEFAULT = {"sph_block": 256, "density_variant": 0, "splat_tile_ratio": 6, "splat_walk_weight": 3, "forces_split": 0}
# knobs of the whole batch: the number of lanes the scenes are split into (clay_batch_set_lanes)
LANES = (1, 2, 3, 4)
DEFAULT_LANES = 1
CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "autotune.json")


def bucket_index(capacity: int) -> int:
    for i, u in enumerate(BUCKETS):
        if capacity < u:
            return i
    return len(BUCKETS)


def signature(sims) -> str:
    counts = np.bincount([bucket_index(s.capacity) for s in sims], minlength=len(BUCKETS) + 1)
    # scenes per bucket rounded to a power of two: similar batches share a tuning
    return "t" + "-".join(str(1 << int(np.ceil(np.log2(c)))) if c else "0" for c in counts)


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


def _trial(root, sims, extra, snaps, choice, lanes, stream, frames):
    # every trial from the same state: stepping moves the fluid, and a later, more spread-out
    # state would cost more whatever the setting
    for s, snap in zip(sims, snaps):
        s.upload(snap)
    batch = Batch(root, sims, extra_splats=extra, sph_block=choice[len(BUCKETS)]["sph_block"], use_graph=True)
    apply(batch, {"uppers": list(BUCKETS), "tunings": [choice[i] for i in range(len(BUCKETS) + 1)], "lanes": lanes})
    ms = _time(batch, stream, frames)
    batch.destroy()
    return ms


def tune(root, sims, extra=(), stream=None, frames=10, use_cache=True, min_gain=0.004):
    """Returns ({"uppers": [...], "tunings": [per bucket dict], "gain": ...}, report)."""
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
    choice = {i: dict(DEFAULT) for i in range(len(BUCKETS) + 1)}
    lanes = DEFAULT_LANES
    snaps = [s.download() for s in sims]
    report = {"signature": sig, "trials": []}

    def timed(ch, ln=None):
        return _trial(root, sims, extra, snaps, ch, lanes if ln is None else ln, stream, frames)

    def consider(buckets, knob, label):
        nonlocal choice
        for v in KNOBS[knob]:
            if all(choice[b][knob] == v for b in buckets):
                continue
            cand = {i: dict(c) for i, c in choice.items()}
            for b in buckets:
                cand[b][knob] = v
            before = timed(choice)
            ms = timed(cand)
            after = timed(choice)
            cur = 0.5 * (before + after)
            report["trials"].append({"bucket": label, knob: v, "ms": round(ms, 4), "current_ms": round(cur, 4)})
            if ms < cur * (1.0 - min_gain):
                choice = cand

    try:
        # the lanes first, for the whole batch
        for v in LANES:
            if v == lanes:
                continue
            before = timed(choice)
            ms = timed(choice, v)
            after = timed(choice)
            cur = 0.5 * (before + after)
            report["trials"].append({"bucket": "batch", "lanes": v, "ms": round(ms, 4), "current_ms": round(cur, 4)})
            if ms < cur * (1.0 - min_gain):
                lanes = v
        everyone = list(range(len(BUCKETS) + 1))
        for knob in KNOBS:
            consider(everyone, knob, "all")
        if len(present) > 1:
            for bi in present:
                for knob in KNOBS:
                    consider([bi], knob, bi)
        # the chosen settings against the defaults, timed again side by side
        default = {i: dict(DEFAULT) for i in range(len(BUCKETS) + 1)}
        t_default = timed(default, DEFAULT_LANES)
        t_tuned = timed(choice)
    finally:
        torch.cuda.synchronize()
        for s, snap in zip(sims, snaps):
            s.upload(snap)
    result = {"uppers": list(BUCKETS), "tunings": [choice[i] for i in range(len(BUCKETS) + 1)], "lanes": lanes,
              "default_ms": t_default, "tuned_ms": t_tuned, "gain": t_default / t_tuned - 1.0,
              "changed": [{"bucket": i, **{k: v for k, v in choice[i].items() if v != DEFAULT[k]}}
                          for i in present if choice[i] != DEFAULT],
              "buckets_present": present}
    if use_cache:
        cache[sig] = result
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        with open(CACHE, "w") as f:
            json.dump(cache, f, indent=1)
    return result, report


def apply(batch, result):
    batch.set_bucket_tuning(result["uppers"], result["tunings"])
    batch.set_lanes(result.get("lanes", DEFAULT_LANES))
