"""The multi-GPU host logic on CPU: two gloo ranks shard scenes with no overlap, own distinct
seeded scenes under weak scaling, and agree on the max/sum reductions the benchmark times with."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from clay_engine_b200 import dist as D
    from clay_engine_b200 import scenes

    ws, r, _ = D.init("gloo", timeout_s=60)
    owned = list(D.shard(257, r, ws))
    counts = scenes.log_uniform_counts(8, 1024, 65536, D.rank_seed(3, r))
    gathered = [None] * ws
    dist.all_gather_object(gathered, {"owned": owned, "counts": counts.tolist()})
    mx = D.reduce_max(10.0 * (r + 1))
    sm = D.reduce_sum(float(len(owned)))
    D.barrier()
    out[r] = {"gathered": gathered, "max": mx, "sum": sm}
    D.finalize()


def test_two_rank_sharding_and_reductions():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    a, b = res[0], res[1]
    g = a["gathered"]
    owned0, owned1 = set(g[0]["owned"]), set(g[1]["owned"])
    assert not owned0 & owned1 and owned0 | owned1 == set(range(257))
    assert g[0]["counts"] != g[1]["counts"], "weak scaling: each rank steps its own scenes"
    assert a["max"] == b["max"] == 20.0
    assert a["sum"] == b["sum"] == 257.0
