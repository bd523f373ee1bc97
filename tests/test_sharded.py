"""G4 distributed over ranks by momentum transfer (dca_b200/sharded.py; the reference's
DistType::LINEAR accumulator, tp_accumulator_gpu.hpp:350-352 and ringG :534-581).

CPU: the transfer split and the placement of a slice in the full G4 (host code of the C ABI), and
two and three gloo ranks whose per-rank accumulator is the oracle, exchanging their measurements
and assembling the full G4, against one oracle that saw every measurement.  GPU: slices computed by
handles with cut transfer lists on one B200 against the full handle, and the exchange over a
one-rank NCCL group with device-resident M."""

import os
import socket

import numpy as np
import pytest

from helpers import golden, rel_err


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_transfer_split_covers_every_transfer_once():
    from dca_b200.sharded import shard_of
    for n_q in (1, 4, 16, 36):
        for n_ranks in range(1, n_q + 1):
            runs = [shard_of(n_q, r, n_ranks) for r in range(n_ranks)]
            assert runs[0][0] == 0
            for (f0, c0), (f1, _) in zip(runs, runs[1:]):
                assert f1 == f0 + c0  # consecutive
            assert sum(c for _, c in runs) == n_q
            assert max(c for _, c in runs) - min(c for _, c in runs) <= 1


def test_transfer_split_rejects_bad_ranks():
    from dca_b200 import _native as N
    from dca_b200.accumulators import LogicError
    from dca_b200.sharded import shard_of
    for args in ((4, 0, 5), (4, 4, 4), (4, -1, 2), (4, 0, 0)):
        with pytest.raises(LogicError):
            shard_of(*args)
    assert b"n_ranks" in N.lib.dcaacc_last_error()


def test_placing_every_slice_rebuilds_the_full_g4():
    """The slice of rank r is the full G4's (q, wq) slabs of its transfers (q and wq are the two
    slowest indices); placing every rank's slice gives the full G4 back, for an uneven split and
    several frequency transfers."""
    from dca_b200.accumulators import LogicError
    from dca_b200.sharded import place_shard, shard_of, shard_parameters
    case, _ = golden("sq2_all")  # 2x2 cluster: 4 momentum transfers, 3 frequency transfers
    p = case.tp_params()
    shape = p.g4_shape()
    rng = np.random.default_rng(5)
    full = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    full = np.asfortranarray(full)
    for n_ranks in (1, 2, 3, 4):
        out = np.zeros(full.size, np.complex128)
        for r in range(n_ranks):
            first, count = shard_of(len(p.k_ex), r, n_ranks)
            assert shard_parameters(p, r, n_ranks).k_ex == list(p.k_ex)[first:first + count]
            sl = np.asfortranarray(full[..., first:first + count, :]).reshape(-1, order="F")
            place_shard(p, r, n_ranks, sl, out)
        assert np.array_equal(out, full.reshape(-1, order="F"))
    with pytest.raises(LogicError):
        place_shard(p, 0, 2, np.zeros(3, np.complex128), out)


class _OracleAdapter:
    """The CPU oracle with the accumulator's lifecycle method names (the per-rank accumulator of
    the CPU test; on a GPU it is TpAccumulator)."""

    def __init__(self, G0, p):
        from oracle import pyoracle
        self.acc = pyoracle.OracleTp(G0, p)

    def resetAccumulation(self, dca_loop=0):
        self.acc.resetAccumulation()

    def accumulate(self, M_pair, configs, sign):
        self.acc.accumulate(list(M_pair), list(configs), sign)
        return 0.0

    def finalize(self):
        pass

    def get_G4(self):
        return self.acc.get_G4()


def _calls(ms, rank, world):
    """Rank's measurements (disjoint streams), grouped into the calls every rank makes together:
    one accumulate_batch of two, then single accumulate calls."""
    mine = ms[rank::world]
    return [mine[:2]] + [[m] for m in mine[2:]]


def _gloo_rank(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    from dca_b200 import replicas
    from dca_b200.sharded import ShardedTpAccumulator
    replicas.init_from_env("gloo", timeout_s=60)
    try:
        case, _ = golden("sq2_all")
        ms = case.measurements * 2
        acc = ShardedTpAccumulator(case.G0, case.tp_params(), local_factory=_OracleAdapter)
        acc.resetAccumulation(0)
        for call in _calls(ms, rank, world):
            if len(call) > 1:
                acc.accumulate_batch([[s.M for s in m.sectors] for m in call], [list(m.sectors) for m in call],
                                     [m.sign for m in call])
            else:
                acc.accumulate([s.M for s in call[0].sectors], list(call[0].sectors), call[0].sign)
        acc.finalize()
        np.save(os.path.join(out_dir, f"g4_{rank}.npy"), np.stack(acc.get_G4()))
        np.save(os.path.join(out_dir, f"slice_{rank}.npy"), np.stack(acc.get_G4_slice()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_assemble_the_full_g4(tmp_path, oracle_lib, world):
    """Each rank accumulates its own measurements; after the exchange every rank's slice holds
    every measurement, and the assembled G4 equals one oracle that added the measurements in the
    same order (call by call, rank 0 first), bit for bit."""
    import torch.multiprocessing as mp
    mp.spawn(_gloo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    case, _ = golden("sq2_all")
    ms = case.measurements * 2
    ref = oracle_lib.OracleTp(case.G0, case.tp_params())
    per_rank = [_calls(ms, r, world) for r in range(world)]
    for i in range(len(per_rank[0])):
        for r in range(world):
            for m in per_rank[r][i]:
                ref.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    want = np.stack(ref.get_G4())
    from dca_b200.sharded import shard_of
    p = case.tp_params()
    for rank in range(world):
        got = np.load(tmp_path / f"g4_{rank}.npy")
        assert np.array_equal(got, want)
        first, count = shard_of(len(p.k_ex), rank, world)
        sl = np.load(tmp_path / f"slice_{rank}.npy")
        for c in range(len(want)):
            want_sl = want[c].reshape(p.g4_shape(), order="F")[..., first:first + count, :]
            assert np.array_equal(sl[c], want_sl.reshape(-1, order="F"))


def _uneven_rank(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    from dca_b200 import replicas
    from dca_b200.sharded import ShardedTpAccumulator
    replicas.init_from_env("gloo", timeout_s=60)
    try:
        case, _ = golden("sq2_all")
        ms = case.measurements
        acc = ShardedTpAccumulator(case.G0, case.tp_params(), local_factory=_OracleAdapter)
        acc.resetAccumulation(0)
        for call in _uneven_calls(ms, rank):
            acc.accumulate_batch([[s.M for s in m.sectors] for m in call], [list(m.sectors) for m in call],
                                 [m.sign for m in call])
        acc.finalize()
        np.save(os.path.join(out_dir, f"g4_{rank}.npy"), np.stack(acc.get_G4()))
    finally:
        dist.destroy_process_group()


def _uneven_calls(ms, rank):
    """Three collective calls in which the ranks bring different numbers of measurements, none
    included: rank 0 brings 2, 0, 1; rank 1 brings 0, 3, 1."""
    return [[ms[0], ms[1]], [], [ms[2]]] if rank == 0 else [[], [ms[2], ms[0], ms[1]], [ms[0]]]


def test_gloo_ranks_with_uneven_calls(tmp_path, oracle_lib):
    """The exchange gathers parts of different lengths (and empty ones) per call; every rank adds
    them in call order, rank 0's part first, and assembles the same G4 as one oracle fed that order."""
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_uneven_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    case, _ = golden("sq2_all")
    ms = case.measurements
    ref = oracle_lib.OracleTp(case.G0, case.tp_params())
    per_rank = [_uneven_calls(ms, r) for r in range(world)]
    for i in range(3):
        for r in range(world):
            for m in per_rank[r][i]:
                ref.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    want = np.stack(ref.get_G4())
    for rank in range(world):
        assert np.array_equal(np.load(tmp_path / f"g4_{rank}.npy"), want)


def _fill(acc, ms):
    acc.resetAccumulation(0)
    for m in ms:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    acc.finalize()
    return acc.get_G4()


@pytest.mark.gpu
@pytest.mark.parametrize("wname", ["sq2_all", "c3"])
def test_slices_on_one_gpu_assemble_the_full_g4(wname):
    """Handles with cut transfer lists (the slices of 2 and 3 ranks) on one GPU, each fed every
    measurement: FP64 slices placed side by side equal the full FP64 handle's G4 to 1e-13; mixed
    slices (which run without the mirror halving and the all-transfer tensor-core direct term)
    stay within 1e-6 of it."""
    from dca_b200 import workloads as W
    from dca_b200.accumulators import TpAccumulator
    from dca_b200.sharded import place_shard, shard_parameters
    from helpers import case_from_workload
    if wname == "c3":
        case = case_from_workload(W.WORKLOADS["c3"], 6)
    else:
        case, _ = golden(wname)
    ms = case.measurements
    p64 = case.tp_params()
    want = _fill(TpAccumulator(case.G0, p64), ms)
    for precision, tol in ((0, 1e-13), (1, 1e-6)):
        p = case.tp_params(precision=precision, max_batch=4)
        for n_ranks in (2, 3):
            full = [np.zeros(w.size, np.complex128) for w in want]
            for r in range(n_ranks):
                sl = _fill(TpAccumulator(case.G0, shard_parameters(p, r, n_ranks)), ms)
                for c in range(len(want)):
                    place_shard(p, r, n_ranks, sl[c], full[c])
            for c in range(len(want)):
                err = rel_err(full[c], want[c])
                assert err <= tol, (precision, n_ranks, c, err)


@pytest.mark.gpu
def test_exchange_over_a_one_rank_nccl_group():
    """The sharded accumulator over a real NCCL group (one rank on this GPU): device-resident M goes
    through the all_gather and reaches the handle as device M; the result is the plain handle's, in
    FP64 and in mixed precision with batches larger than a call (each call processes what it
    gathered before its buffers go; freshly allocated tensors in between would expose a late read)."""
    import torch
    import torch.distributed as dist
    from dca_b200.accumulators import TpAccumulator
    from dca_b200.sharded import ShardedTpAccumulator
    case, _ = golden("sq2_all")
    ms = case.measurements * 3
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(_free_port())})
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        for precision, tol in ((0, 1e-13), (1, 1e-6)):
            p = case.tp_params(precision=precision, max_batch=4)
            want = _fill(TpAccumulator(case.G0, case.tp_params()), ms)
            acc = ShardedTpAccumulator(case.G0, p)
            assert acc.n_ranks == 1 and acc.shard == (0, len(p.k_ex))
            acc.resetAccumulation(0)
            for m in ms:
                Md = [torch.from_numpy(np.asarray(s.M)).cuda() for s in m.sectors]
                acc.accumulate(Md, list(m.sectors), m.sign)
                del Md
                # Fresh allocations of the gathered buffers' sizes take their freed blocks back.
                junk = [torch.full((k,), float("nan"), dtype=torch.float64, device="cuda") for k in (1, 16, 256, 2048)]
                del junk
            acc.finalize()
            got = acc.get_G4()
            torch.cuda.synchronize()
            for g, w in zip(got, want):
                assert rel_err(g, w) <= tol, (precision, rel_err(g, w))
    finally:
        dist.destroy_process_group()
