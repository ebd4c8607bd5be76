"""Packet parallelism across ranks (one process per GPU).

The reference splits packets over MPI ranks and averages the tallies with
one Allreduce per quantity (J_nu and e_abs: src/transport/transport_mpi.cpp:374-407;
spectrum flux and clicks: src/transport/spectrum_array.cpp:425-463).  Here
every rank propagates its own packets with Philox stream ids offset by
rank * packets_per_rank, so N ranks draw exactly the packets a single run of
N * packets_per_rank would; the tallies are then averaged over ranks with
torch.distributed (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import Dict

import numpy as np


def first_packet_id(rank: int, packets_per_rank: int) -> int:
    return int(rank) * int(packets_per_rank)


def average_over_ranks(arrays: Dict[str, np.ndarray], device: str = "cpu") -> Dict[str, np.ndarray]:
    """Sum-allreduce each array and divide by the number of ranks, as
    transport::reduce_radiation and spectrum_array::MPI_average do."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size() if dist.is_initialized() else 1
    out = {}
    for k in sorted(arrays):  # same order on every rank
        t = torch.as_tensor(np.ascontiguousarray(arrays[k]), dtype=torch.float64, device=device)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
        out[k] = (t / world).cpu().numpy()
    return out


def max_over_ranks(x: float, device: str = "cpu") -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
