"""The N>1 path on CPU: shot sharding plus one all-reduce of the FP64 stacks,
run as two gloo ranks (no GPU).  The per-rank compute is the FP64 oracle, the
stand-in for each rank's GPU engine; the sharding and the exchange are the
product code (rtm_b200.shard) that bench.py uses under torchrun."""
import os
import socket
import tempfile

import numpy as np
import pytest

from helpers import random_problem, rel_l2
from rtm_b200 import shard


def test_assign_shots_balances_uneven_windows():
    rng = np.random.default_rng(3)
    costs = rng.uniform(400, 1150, 256).tolist()
    for world in (1, 2, 4, 8):
        a = shard.assign_shots(costs, world)
        assert sorted(i for r in a for i in r) == list(range(256))          # each shot exactly once
        loads = [sum(costs[i] for i in r) for r in a]
        assert max(loads) - min(loads) <= max(costs)                          # greedy LPT bound
        assert a == shard.assign_shots(costs, world)                          # deterministic
    assert shard.assign_shots([1.0] * 6, 3) == [[0, 3], [1, 4], [2, 5]]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import oracle
    p, v, shots = random_problem(seed=21, order=8, nx=30, nz=24, nb=7, nt=80, si=2)
    shots = shots + random_problem(seed=22, order=8, nx=30, nz=24, nb=7, nt=80, si=2)[2]
    mine = shard.rank_shots(shots, rank, world, p.nx, p.nz, p.nb, p.nt)
    if mine:
        img, ill = oracle.migrate(p, v, mine, np.float64)
    else:
        img, ill = np.zeros(p.nx * p.nz), np.zeros(p.nx * p.nz)
    img, ill = shard.allreduce_stack(img, ill)
    np.save(os.path.join(outdir, f"img{rank}.npy"), img)
    np.save(os.path.join(outdir, f"ill{rank}.npy"), ill)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_stack_equals_single_process_stack(world):
    import torch.multiprocessing as mp
    import oracle
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_rank_main, args=(world, _free_port(), td), nprocs=world, start_method="spawn",
                           join=True)
        imgs = [np.load(os.path.join(td, f"img{r}.npy")) for r in range(world)]
        ills = [np.load(os.path.join(td, f"ill{r}.npy")) for r in range(world)]
    p, v, shots = random_problem(seed=21, order=8, nx=30, nz=24, nb=7, nt=80, si=2)
    shots = shots + random_problem(seed=22, order=8, nx=30, nz=24, nb=7, nt=80, si=2)[2]
    ref_img, ref_ill = oracle.migrate(p, v, shots, np.float64)
    for r in range(world):
        assert np.array_equal(imgs[r], imgs[0])          # every rank holds the same stack
        assert rel_l2(ref_img, imgs[r]) < 1e-12          # only the summation order differs
        assert rel_l2(ref_ill, ills[r]) < 1e-12
