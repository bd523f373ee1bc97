"""Shared test helpers: load golden cases, build accumulator inputs, compare results."""

from __future__ import annotations

import dataclasses
import os
import struct
from typing import List

import numpy as np

from dca_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@dataclasses.dataclass
class Case:
    nb: int
    nc: int
    nw_half: int
    n_sp: int
    all_transfers: bool
    freq_transfer: int
    k_transfer: int
    channels: List[int]
    flags: int
    beta: float
    r_vecs: np.ndarray
    k_vecs: np.ndarray
    k_add: np.ndarray  # [i, j]
    k_sub: np.ndarray
    r_add: np.ndarray
    r_sub: np.ndarray
    a_vecs: np.ndarray
    G0: np.ndarray
    measurements: list

    def k_ex(self):
        return list(range(self.nc)) if self.all_transfers else [self.k_transfer]

    def w_ex(self):
        return list(range(self.freq_transfer + 1)) if self.all_transfers else [self.freq_transfer]

    def tp_params(self, **kw):
        from dca_b200.accumulators import TpParameters
        max_n = max([max(s.n for s in m.sectors) for m in self.measurements] + [1])
        args = dict(n_bands=self.nb, n_sites=self.nc, n_w_half=self.nw_half, n_sp_freq=self.n_sp,
                    beta=self.beta, channels=self.channels, k_ex=self.k_ex(), w_ex=self.w_ex(),
                    r_vecs=self.r_vecs, k_vecs=self.k_vecs, a_vecs=self.a_vecs, k_add=self.k_add,
                    k_sub=self.k_sub, r_sub=self.r_sub, max_order=max_n)
        args.update(kw)
        return TpParameters(**args)

    def sp_params(self, **kw):
        from dca_b200.accumulators import SpParameters
        max_n = max([max(s.n for s in m.sectors) for m in self.measurements] + [1])
        args = dict(n_bands=self.nb, n_sites=self.nc, n_sp_freq=self.n_sp, beta=self.beta,
                    r_sub=self.r_sub, max_order=max_n)
        args.update(kw)
        return SpParameters(**args)


def read_case(path) -> Case:
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"DCACASE1"
    off = 8
    h = struct.unpack_from("<8i", data, off)
    off += 32
    ch = struct.unpack_from("<4i", data, off)
    off += 16
    n_meas, flags = struct.unpack_from("<2i", data, off)
    off += 8
    (beta,) = struct.unpack_from("<d", data, off)
    off += 8
    nb, nc, nw_half, n_sp = h[0], h[1], h[2], h[3]

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(data, dtype, count, off).copy()
        off += a.nbytes
        return a

    r_vecs = take(np.float64, 2 * nc).reshape(nc, 2)
    k_vecs = take(np.float64, 2 * nc).reshape(nc, 2)
    tables = [take(np.int32, nc * nc).reshape(nc, nc).T.copy() for _ in range(4)]
    a_vecs = take(np.float64, 2 * nb).reshape(nb, 2)
    G0 = take(np.complex128, (2 * nb) ** 2 * nc * 2 * n_sp)
    ms = []
    for _ in range(n_meas):
        (sign,) = struct.unpack_from("<i", data, off)
        off += 4
        secs = []
        for _s in range(2):
            (n,) = struct.unpack_from("<i", data, off)
            off += 4
            tau = take(np.float64, n)
            lb, rb, ls, rs = (take(np.int32, n) for _ in range(4))
            M = take(np.float64, n * n).reshape(n, n, order="F") if n else np.zeros((0, 0))
            secs.append(W.Sector(tau, lb, rb, ls, rs, np.asfortranarray(M)))
        ms.append(W.Measurement(sign, tuple(secs)))
    return Case(nb, nc, nw_half, n_sp, bool(h[4]), h[5], h[6], list(ch[: h[7]]), flags, beta,
                r_vecs, k_vecs, tables[0], tables[1], tables[2], tables[3], a_vecs, G0, ms)


def golden(name):
    from oracle import casefile as CF
    return read_case(os.path.join(GOLDEN, name + ".case")), CF.read_result(os.path.join(GOLDEN, name + ".ref"))


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def case_from_workload(w: W.Workload, n_meas: int, start: int = 0) -> Case:
    cl = w.cluster()
    mu = w.chemical_potential()
    g0 = W.make_g0(w.model, cl, w.beta, mu, w.n_sp).reshape(-1)
    ms = W.make_measurements(w, n_meas, start)
    return Case(w.nb, cl.nc, w.nw_half, w.n_sp, w.all_transfers, w.freq_transfer, w.k_transfer,
                list(w.channels), 0, w.beta, cl.r_vecs, cl.k_vecs, cl.k_add, cl.k_sub, cl.r_add,
                cl.r_sub, w.model.a_vecs(), g0, ms)
