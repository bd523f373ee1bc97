"""Multi-process (replica) path on CPU: two gloo ranks, each with its own accumulator and its own
measurements; the per-iteration G4 reduction over ranks equals one accumulator that saw every
measurement, and the cross-rank timing helpers return the slowest rank's value."""

import os
import socket

import numpy as np
import pytest

from helpers import case_from_workload, rel_err
from dca_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    from dca_b200 import replicas
    from oracle import pyoracle
    n, r, _ = replicas.init_from_env("gloo", timeout_s=60)
    assert (n, r) == (world, rank)
    try:
        case = case_from_workload(W.WORKLOADS["c1"], 6)
        acc = pyoracle.OracleTp(case.G0, case.tp_params())
        for m in case.measurements[rank::world]:  # disjoint measurement streams
            acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        total = replicas.sum_g4(acc.get_G4())
        slowest = replicas.max_over_ranks(10.0 + rank)
        count = replicas.sum_over_ranks(len(case.measurements[rank::world]))
        replicas.barrier()
        np.save(os.path.join(out_dir, f"g4_{rank}.npy"), np.stack(total))
        np.save(os.path.join(out_dir, f"scalars_{rank}.npy"), np.array([slowest, count]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_reduce_to_one_accumulator(tmp_path, oracle_lib):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    case = case_from_workload(W.WORKLOADS["c1"], 6)
    ref = oracle_lib.OracleTp(case.G0, case.tp_params())
    for m in case.measurements:
        ref.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    want = np.stack(ref.get_G4())
    for rank in range(world):
        got = np.load(tmp_path / f"g4_{rank}.npy")
        assert rel_err(got, want) <= 1e-14  # only the order of the FP64 sums differs
        slowest, count = np.load(tmp_path / f"scalars_{rank}.npy")
        assert slowest == 10.0 + world - 1
        assert count == len(case.measurements)


def test_single_process_helpers_are_no_ops():
    from dca_b200 import replicas
    assert replicas.world() == 1
    assert replicas.max_over_ranks(3.5) == 3.5
    g = [np.arange(4, dtype=np.complex128)]
    assert np.array_equal(replicas.sum_g4(g)[0], g[0])
