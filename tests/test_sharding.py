"""Host-side sharding of independent systems across ranks (no data-path collective):
greedy LPT balance, and a world-size-2 gloo run that gathers per-rank results."""
import os

import numpy as np
import torch.multiprocessing as mp

from kcfd.batch import lpt_shards


def test_lpt_balances_and_covers():
    rng = np.random.default_rng(0)
    w = np.exp(rng.uniform(np.log(2e3), np.log(2e5), 1024))
    sh = lpt_shards(w, 8)
    allidx = sorted(i for s in sh for i in s)
    assert allidx == list(range(1024))
    loads = [w[s].sum() for s in sh]
    assert max(loads) / min(loads) < 1.02


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = np.arange(1, 33, dtype=float)
    mine = lpt_shards(w, world)[rank]
    # stand-in per-system result: the system's weight squared (the device solve runs
    # per rank in production; only the host bookkeeping is under test here)
    res = torch.zeros(len(w), dtype=torch.float64)
    for i in mine:
        res[i] = w[i] ** 2
    dist.all_reduce(res)   # host-side gather of per-system results
    if rank == 0:
        out.put(res.numpy().tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = q.get(timeout=120)
    for p in ps:
        p.join(timeout=120)
    assert res == [float(v) ** 2 for v in range(1, 33)]
