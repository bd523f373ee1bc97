"""G4 distributed over ranks by momentum transfer: the reference's distributed two-particle
accumulator, TpAccumulator<Parameters, DistType::LINEAR, GPU> (tp_accumulator_gpu.hpp:350-352;
the ring of G, ringG, :534-581; each rank's slice bounds, G4_[0].get_start() / get_end(), :421-423).

The reference gives each MPI rank a contiguous range of G4's linear index and passes every
measurement's G from rank to rank around a ring, so that each rank adds every measurement into
its range.  Here a rank's range is a run of whole momentum transfers (dcaacc_tp_g4_shard): rank r
owns transfers [first, first + count) of the transfer list, which is the G4 of an ordinary handle
created with that sub-list, bit for bit the full G4's entries with those transfers, since no G4
entry mixes transfers.  What crosses between ranks is each measurement's walker output (M and the
vertex configuration, n x n real numbers per spin) rather than its G (D x D complex numbers per
spin): every rank recomputes the G of every measurement, which on a B200 takes less time than
moving G over NVLink would (c3: about 11 us of front-end kernels per measurement against 16.8 MB
of FP32 G; c5: 0.34 ms against 340 MB).  Sharding trades that replicated front-end work for G4
memory: each GPU holds 1/n_ranks of G4 and of its FP64 read-modify-write traffic.  For the
benchmark configurations, whose G4 fits on one GPU, independent replicas (replicas.py) are faster.

Exchange: one torch.distributed all_gather per accumulate call for the vertex data and signs (a
host array, staged through the device on NCCL) and one for the M matrices, which stay on the
device on NCCL and reach the accumulator as device M.  Every rank then feeds its handle the
measurements of rank 0, 1, ..., n_ranks - 1 in that order and processes them before the call
returns (the gathered M buffers belong to the call), so a call should carry about a batch's worth
of measurements across the ranks (max_batch / n_ranks per rank in mixed precision).  get_G4
all-gathers the slices and assembles the full G4 on every rank (dcaacc_tp_g4_place_shard).  In a single process without a
process group the shard is the whole transfer list and nothing is exchanged.
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from . import workloads as W
from .accumulators import LogicError, TpAccumulator, TpParameters, _check, _dptr, _iptr

_VERTEX_FIELDS = ("tau", "left_band", "right_band", "left_site", "right_site")


def shard_of(n_k_ex: int, rank: int, n_ranks: int) -> Tuple[int, int]:
    """(first, count): the momentum transfers [first, first + count) of the transfer list that
    rank owns among n_ranks (dcaacc_tp_g4_shard)."""
    first, count = ctypes.c_int32(), ctypes.c_int32()
    _check(N.lib.dcaacc_tp_g4_shard(int(n_k_ex), int(rank), int(n_ranks), ctypes.byref(first), ctypes.byref(count)))
    return first.value, count.value


def shard_parameters(parameters: TpParameters, rank: int, n_ranks: int) -> TpParameters:
    """The parameters of rank's G4 slice: the full ones with the transfer list cut to its run."""
    first, count = shard_of(len(parameters.k_ex), rank, n_ranks)
    return dataclasses.replace(parameters, k_ex=list(parameters.k_ex)[first:first + count])


def _config(p: TpParameters, keep: list) -> N.TpConfig:
    # Only the sizes and the transfer counts are read by dcaacc_tp_g4_place_shard.
    k_ex = np.ascontiguousarray(p.k_ex, np.int32)
    w_ex = np.ascontiguousarray(p.w_ex, np.int32)
    ch = np.ascontiguousarray(p.channels, np.int32)
    keep.extend((k_ex, w_ex, ch))
    null_d = ctypes.POINTER(ctypes.c_double)()
    null_i = ctypes.POINTER(ctypes.c_int32)()
    return N.TpConfig(p.n_bands, p.n_sites, p.n_w_half, p.n_sp_freq, len(k_ex), _iptr(k_ex), len(w_ex), _iptr(w_ex),
                      len(ch), _iptr(ch), p.beta, null_d, null_d, null_d, null_i, null_i, int(p.non_density),
                      p.precision, p.max_batch, p.max_order, p.accumulators)


def place_shard(parameters: TpParameters, rank: int, n_ranks: int, shard: np.ndarray, full: np.ndarray) -> None:
    """Copies one channel of rank's G4 slice (complex128) into its place in the full G4 (complex128,
    both in the layout (b1, b2, b3, b4, k1, w1, k2, w2, q, wq), first index fastest)."""
    if shard.dtype != np.complex128 or full.dtype != np.complex128 or not full.flags.c_contiguous:
        raise LogicError("place_shard takes contiguous complex128 arrays")
    shard = np.ascontiguousarray(shard)
    keep: list = []
    cfg = _config(parameters, keep)
    _check(N.lib.dcaacc_tp_g4_place_shard(ctypes.byref(cfg), int(rank), int(n_ranks), _dptr(shard.view(np.float64)),
                                          shard.size, _dptr(full.view(np.float64)), full.size))


class ShardedTpAccumulator:
    """The two-particle accumulator with G4 distributed over the ranks of a torch.distributed
    process group (see the module docstring).  Method set of TpAccumulator; accumulate and
    accumulate_batch are collective (every rank calls them the same number of times, in the same
    order), as are get_G4 and get_G4_normalized.  ``local_factory(G0, parameters)`` builds the
    per-rank accumulator (TpAccumulator by default)."""

    def __init__(self, G0: np.ndarray, parameters: TpParameters, thread_id: int = 0, group=None,
                 local_factory: Optional[Callable] = None):
        import torch.distributed as dist
        self._dist = dist if dist.is_available() and dist.is_initialized() else None
        self._group = group
        self.rank = self._dist.get_rank(group) if self._dist else 0
        self.n_ranks = self._dist.get_world_size(group) if self._dist else 1
        self.parameters = parameters
        self.shard = shard_of(len(parameters.k_ex), self.rank, self.n_ranks)
        self.shard_parameters = shard_parameters(parameters, self.rank, self.n_ranks)
        if local_factory is None:
            self.local = TpAccumulator(G0, self.shard_parameters, thread_id)
        else:
            self.local = local_factory(G0, self.shard_parameters)
        self._g4: Optional[List[np.ndarray]] = None

    # -- exchange ------------------------------------------------------------------------------
    def _device(self):
        import torch
        if self._dist.get_backend(self._group) == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def _all_gather(self, t):
        """all_gather of a 1-D float64 tensor whose length differs between ranks."""
        import torch
        n = torch.tensor([t.numel()], dtype=torch.int64, device=t.device)
        sizes = [torch.zeros_like(n) for _ in range(self.n_ranks)]
        self._dist.all_gather(sizes, n, group=self._group)
        sizes = [int(s.item()) for s in sizes]
        width = max(max(sizes), 1)
        buf = torch.zeros(width, dtype=t.dtype, device=t.device)
        buf[:t.numel()] = t
        parts = [torch.empty_like(buf) for _ in range(self.n_ranks)]
        self._dist.all_gather(parts, buf, group=self._group)
        return [p[:s] for p, s in zip(parts, sizes)]

    def _exchange(self, Ms, configs, signs):
        """Every rank's (Ms, configs, signs) of this call, in rank order."""
        import torch
        dev = self._device()
        count = len(signs)
        # Vertex data and signs: [count, then per measurement sign, n0, n1, then per sector the five
        # vertex arrays], in float64 (band and site indices are exact there).
        head = [float(count)]
        body = []
        for m in range(count):
            head.append(float(np.real(signs[m])))
            for c in configs[m]:
                head.append(float(len(c.tau)))
                body.extend(np.asarray(getattr(c, f), np.float64) for f in _VERTEX_FIELDS)
        meta = np.concatenate([np.asarray(head, np.float64)] + body) if body else np.asarray(head, np.float64)
        mats = []
        for pair in Ms:
            for M in pair:
                if isinstance(M, torch.Tensor):
                    mats.append(M.to(device=dev, dtype=torch.float64).t().reshape(-1))  # column major
                else:
                    a = np.asarray(M, np.float64)
                    mats.append(torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order="F"))).to(dev))
        mat = torch.cat(mats) if mats else torch.zeros(0, dtype=torch.float64, device=dev)
        metas = [p.cpu().numpy() for p in self._all_gather(torch.from_numpy(meta).to(dev))]
        matss = self._all_gather(mat)
        out = []
        for r in range(self.n_ranks):  # this rank's own inputs too, so that every rank adds the same bits
            meta_r, mat_r = metas[r], matss[r]
            cnt = int(meta_r[0])
            pos, vpos, mpos = 1, 1 + 3 * cnt, 0
            Ms_r, cf_r, sg_r = [], [], []
            for _ in range(cnt):
                sg_r.append(int(meta_r[pos]))
                ns = (int(meta_r[pos + 1]), int(meta_r[pos + 2]))
                pos += 3
                pair_m, pair_c = [], []
                for n in ns:
                    arrs = [meta_r[vpos + k * n: vpos + (k + 1) * n] for k in range(5)]
                    vpos += 5 * n
                    flat = mat_r[mpos: mpos + n * n]
                    mpos += n * n
                    if dev.type == "cuda":
                        M = flat.view(n, n).t()  # column major, on the device
                    else:
                        M = np.asfortranarray(flat.numpy().reshape((n, n), order="F"))
                    pair_m.append(M)
                    pair_c.append(W.Sector(arrs[0].copy(), *(a.astype(np.int32) for a in arrs[1:]),
                                           M if dev.type != "cuda" else np.zeros((0, 0))))
                Ms_r.append(pair_m)
                cf_r.append(pair_c)
            out.append((Ms_r, cf_r, sg_r))
        return out

    # -- reference method set ------------------------------------------------------------------
    def resetAccumulation(self, dca_loop: int = 0):
        self.local.resetAccumulation(dca_loop)
        self._g4 = None

    def accumulate(self, M_pair, configs, sign: int) -> float:
        """Collective: adds every rank's measurement of this call into this rank's G4 slice."""
        return self.accumulate_batch([M_pair], [configs], [sign])

    def accumulate_batch(self, Ms: Sequence, configs: Sequence, signs: Sequence) -> float:
        """Collective: every rank's measurements of this call, in rank order, into this rank's slice.
        Returns the flops of this rank's handle."""
        if self._dist is None:
            if hasattr(self.local, "accumulate_batch"):
                return self.local.accumulate_batch(Ms, configs, signs)
            return sum(self.local.accumulate(M_pair, cfg, s) or 0.0 for M_pair, cfg, s in zip(Ms, configs, signs))
        parts = self._exchange(Ms, configs, signs)
        flops = 0.0
        for Ms_r, cf_r, sg_r in parts:
            if not sg_r:
                continue
            if hasattr(self.local, "accumulate_batch"):
                flops += self.local.accumulate_batch(Ms_r, cf_r, sg_r) or 0.0
            else:
                for M_pair, cfg, s in zip(Ms_r, cf_r, sg_r):
                    flops += self.local.accumulate(M_pair, cfg, s) or 0.0
        # The gathered M buffers are this call's temporaries, while a mixed-precision handle reads a
        # measurement's M only when its batch runs: process what is queued and wait for it before
        # the buffers go (a rank's call returns with its handle idle).
        if hasattr(self.local, "flush"):
            self.local.flush()
        if hasattr(self.local, "synchronizeCopy"):
            self.local.synchronizeCopy()
        return flops

    def finalize(self):
        self.local.finalize()
        self._g4 = None

    def get_G4_slice(self) -> List[np.ndarray]:
        """This rank's slice of each channel's G4: the transfers [first, first + count) of shard."""
        return self.local.get_G4()

    def _assemble(self, slices: List[np.ndarray]) -> List[np.ndarray]:
        import torch
        p = self.parameters
        full_size = int(np.prod(p.g4_shape()))
        out = []
        for c, mine in enumerate(slices):
            full = np.zeros(full_size, np.complex128)
            if self._dist is None:
                place_shard(p, 0, 1, mine, full)
            else:
                dev = self._device()
                parts = self._all_gather(torch.from_numpy(np.ascontiguousarray(mine).view(np.float64)).to(dev))
                for r, part in enumerate(parts):
                    place_shard(p, r, self.n_ranks, part.cpu().numpy().view(np.complex128), full)
            out.append(full)
        return out

    def get_G4(self) -> List[np.ndarray]:
        """Collective: the full G4 of every channel, assembled from all ranks' slices (after finalize)."""
        if self._g4 is None:
            self._g4 = self._assemble(self.local.get_G4())
        return self._g4

    def get_G4_normalized(self) -> List[np.ndarray]:
        """Collective: the full G4 / (accumulated sign * beta^2).  Every rank has seen every
        measurement, so each slice carries the global sign sum."""
        return self._assemble(self.local.get_G4_normalized())

    def sign_sum(self):
        return self.local.sign_sum()

    def sumTo(self, other: "ShardedTpAccumulator"):
        """Adds this rank's slice into other's slice of the same transfers (tp_accumulator_cpu.hpp:896-904)."""
        if other.shard != self.shard:
            raise LogicError("sumTo between shards of different transfers")
        self.local.sumTo(other.local)
