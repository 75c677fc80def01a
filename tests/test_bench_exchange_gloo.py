"""bench.py's multi-GPU step on CPU: two gloo ranks run `survey_step`, the code
the benchmark runs under torchrun, with a stand-in engine.

The stand-in writes known FP64 image and illumination stacks for its shots into
the rank's stack tensor through the same raw-address interface the real engine
uses (migrate_f64_into); `survey_step` then sums the stacks over the ranks in
place.  Every rank must end with the sum over all shots, equal to one rank
migrating every shot, and the tensor it holds must be the one it passed in (the
reduction is in place).
"""
import ctypes as C
import os
import socket
import tempfile

import numpy as np
import torch

from rtm_b200 import shard

N_IMG = 37


class StubEngine:
    """Per-shot FP64 contributions: image = f(shot) * ramp, illumination = ramp^2."""

    def migrate_f64_into(self, shots, img_ptr, ill_ptr):
        ramp = np.arange(1, N_IMG + 1, dtype=np.float64)
        img = sum(float(s["k"]) * ramp for s in shots) if shots else np.zeros(N_IMG)
        ill = sum(ramp * ramp for _ in shots) if shots else np.zeros(N_IMG)
        C.memmove(img_ptr, np.ascontiguousarray(img).ctypes.data, N_IMG * 8)
        C.memmove(ill_ptr, np.ascontiguousarray(ill).ctypes.data, N_IMG * 8)


def _shots():
    return [{"k": k + 1, "window_nx": 400 + 37 * k} for k in range(7)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    costs = [s["window_nx"] for s in _shots()]
    mine = [_shots()[i] for i in shard.assign_shots(costs, world)[rank]]
    stacks = torch.zeros(2 * N_IMG, dtype=torch.float64)
    ptr = stacks.data_ptr()
    bench.survey_step(StubEngine(), mine, stacks, world)
    assert stacks.data_ptr() == ptr
    np.save(os.path.join(outdir, f"s{rank}.npy"), stacks.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_survey_step_sums_the_fp64_stacks_in_place():
    import torch.multiprocessing as mp
    world = 2
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_rank_main, args=(world, _free_port(), td), nprocs=world, start_method="spawn",
                           join=True)
        got = [np.load(os.path.join(td, f"s{r}.npy")) for r in range(world)]
    single = torch.zeros(2 * N_IMG, dtype=torch.float64)
    import bench
    bench.survey_step(StubEngine(), _shots(), single, 1)
    for g in got:
        assert np.array_equal(g, single.numpy())
