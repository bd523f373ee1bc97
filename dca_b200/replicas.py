"""Multi-GPU use of the accumulators: independent replicas.

Measurements are independent, so N GPUs run N accumulators on disjoint measurement streams (one
process per GPU) and nothing crosses between them on the data path.  The only cross-rank steps are
the ones the DCA loop itself has: the solver's once-per-iteration reduction of G4 and of the sign
sum over all ranks (ctaux_cluster_solver.hpp:492-511, an MPI sum in the reference), and, for
benchmarking, the slowest rank's time.  These helpers do those steps over an initialised
torch.distributed process group (NCCL between GPUs, gloo on CPU) and are plain no-ops in a
single process.
"""

from __future__ import annotations

import os
from datetime import timedelta
from typing import List, Sequence

import numpy as np


def world() -> int:
    import torch.distributed as dist
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def init_from_env(backend: str, timeout_s: float = 300.0):
    """Joins the process group described by RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT (as
    torchrun sets them).  Returns (world_size, rank, local_rank); a single process needs no group."""
    n = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if n > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return n, rank, local


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier():
    if world() > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float) -> float:
    """The slowest rank's value (times are reported as max over ranks)."""
    if world() == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    if world() == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def sum_g4(g4: Sequence[np.ndarray]) -> List[np.ndarray]:
    """Sums each channel's G4 (complex128, host) over the ranks: the solver's per-iteration
    reduction of the replicas' accumulations.  Every rank receives the total."""
    out = [np.array(g, dtype=np.complex128, copy=True) for g in g4]
    if world() == 1:
        return out
    import torch
    import torch.distributed as dist
    dev = _device()
    for g in out:
        t = torch.from_numpy(g.view(np.float64)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        g.view(np.float64)[:] = t.cpu().numpy()
    return out
