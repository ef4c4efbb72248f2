"""The N > 1 path of the ERI sweep on CPU: two gloo ranks draw disjoint
quartet shards and agree on the slowest rank's time."""
import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from librint_b200 import shard, synthetic


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", world_size=world, rank=rank)
    try:
        w, r, _ = shard.world_info()
        m, shls = synthetic.eri_sweep((1, 1, 0, 0), 16, seed=shard.shard_seed(2, r))
        first_centre = float(m.env[m.atm[1]])
        t = shard.max_over_ranks(1.0 + r)          # rank-dependent "device time"
        firsts = [None] * w
        dist.all_gather_object(firsts, first_centre)
        q.put((r, w, t, firsts))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, t, firsts in out:
        assert w == 2 and t == 2.0                 # max over ranks of 1 + rank
        assert firsts[0] != firsts[1]              # different shards


def test_single_process_is_identity():
    assert shard.max_over_ranks(3.5) == 3.5
    assert shard.shard_seed(2, 0) == 2 and shard.shard_seed(2, 3) == 3002
    assert np.isfinite(shard.max_over_ranks(np.float64(1.25)))
