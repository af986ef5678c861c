"""Two ranks driving the library, as `bench.py --gpus N` does on N GPUs: each process joins the
process group, builds its own rank-seeded scenes (weak scaling), steps them as one batch and
meets the other only at the host reductions. Run here as two processes sharing cuda:0 with the
gloo backend (no kernel of one rank waits on the other's), and checked against the same scenes
stepped in this process alone: every rank's particle state is bit for bit the same."""
import hashlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_scenes(root, rank):
    """Four small batched-configuration scenes of this rank's seed; returns (sims, keep)."""
    from clay_engine_b200 import dist as D
    from clay_engine_b200 import scenes

    seed = D.rank_seed(5, rank)
    counts = scenes.log_uniform_counts(4, 1024, 8192, seed)
    sims, keep = [], []
    for i, n in enumerate(counts):
        sc = scenes.config3_scene(root, i, int(n), seed)
        sims.append(sc["sim"])
        keep += sc["keep"]
    return sims, keep


def _step_digest(root, rank, frames=2):
    import torch

    import clay_engine_b200 as ce

    sims, keep = _rank_scenes(root, rank)
    batch = ce.Batch(root, sims, extra_splats=[k for k in keep if isinstance(k, ce.SplatField)])
    for _ in range(frames):
        batch.step()
    torch.cuda.synchronize()
    h = hashlib.sha256()
    total = 0
    for s in sims:
        g = s.download()
        total += len(g)
        h.update(np.ascontiguousarray(g).tobytes())
        h.update(np.ascontiguousarray(s.surface.volume.download()[0]).tobytes())
    batch.destroy()
    for s in sims:
        s.destroy()
    return h.hexdigest(), total


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import clay_engine_b200 as ce
    from clay_engine_b200 import dist as D

    ws, r, _ = D.init("gloo", timeout_s=120)
    torch.cuda.set_device(0)
    root = ce.init(0)
    D.barrier()
    digest, n = _step_digest(root, r)
    total = D.reduce_sum(float(n))
    gathered = [None] * ws
    dist.all_gather_object(gathered, digest)
    D.barrier()
    out[r] = {"digest": digest, "particles": n, "total": total, "gathered": gathered}
    root.destroy()
    D.finalize()


def test_two_ranks_step_their_own_scenes(root):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0]["digest"] != res[1]["digest"], "weak scaling: each rank steps its own scenes"
    assert res[0]["gathered"] == res[1]["gathered"] == [res[0]["digest"], res[1]["digest"]]
    assert res[0]["total"] == res[1]["total"] == float(res[0]["particles"] + res[1]["particles"])
    for r in range(world):
        alone, n = _step_digest(root, r)
        assert n == res[r]["particles"]
        assert alone == res[r]["digest"], f"rank {r}: the batch stepped in a rank differs from the same scenes alone"
