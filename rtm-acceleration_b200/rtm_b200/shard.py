"""Shot sharding across ranks (one process per GPU) and the cross-rank stack.

Shots are independent (the reference calls the shot loop "embarrassingly
parallel", src/rtm/rtm.cpp:80-81), so the multi-GPU path has exactly one
exchange: the sum of every rank's FP64 image and illumination stacks at the end.
Shots are assigned to ranks by cost, cost = nt * (window_nx + 2 nb) * (nz + 2 nb)
cell updates per pass, longest first onto the least-loaded rank (a deterministic
greedy schedule every rank computes identically, no communication).
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def shot_cost(shot, nx: int, nz: int, nb: int, nt: int) -> float:
    w = getattr(shot, "window_nx", 0) or nx
    return float(nt) * (w + 2 * nb) * (nz + 2 * nb)


def assign_shots(costs: Sequence[float], world: int) -> List[List[int]]:
    """Indices of the shots each rank migrates (sorted ascending per rank)."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def rank_shots(shots, rank: int, world: int, nx: int, nz: int, nb: int, nt: int):
    costs = [shot_cost(s, nx, nz, nb, nt) for s in shots]
    return [shots[i] for i in assign_shots(costs, world)[rank]]


def allreduce_stacks_(stacks, group=None):
    """Sum every rank's FP64 stacks in place: ``stacks`` is one contiguous
    float64 tensor holding the image stack followed by the illumination stack
    (2*nx*nz doubles, on the rank's GPU for NCCL or on the host for gloo).  One
    all-reduce, the only exchange of the multi-GPU path."""
    import torch
    import torch.distributed as dist
    if stacks.dtype != torch.float64 or not stacks.is_contiguous():
        raise ValueError("stacks must be one contiguous float64 tensor")
    dist.all_reduce(stacks, op=dist.ReduceOp.SUM, group=group)
    return stacks


def allreduce_stack(image, illum, group=None, device=None):
    """Sum the FP64 image and illumination stacks of every rank; numpy arrays
    in, numpy arrays out (host copies), or torch tensors in and out."""
    import torch
    as_numpy = isinstance(image, np.ndarray)
    a = torch.as_tensor(image, dtype=torch.float64).reshape(-1)
    b = torch.as_tensor(illum, dtype=torch.float64).reshape(-1)
    buf = torch.cat([a, b])
    if device is not None:
        buf = buf.to(device)
    allreduce_stacks_(buf, group)
    n = a.numel()
    ri, rs = buf[:n], buf[n:]
    if as_numpy:
        return ri.cpu().numpy(), rs.cpu().numpy()
    return ri, rs
