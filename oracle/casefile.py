"""Reader / writer for the binary case and result files described in oracle/casefile.hpp.

Test infrastructure only: it feeds identical inputs to the reference's own CPU accumulators
(oracle/_ref/tp_ref), the CPU restatement (oracle/liboracle.so) and the GPU parity tests.
"""

from __future__ import annotations

import struct
from typing import List, Sequence

import numpy as np


def write_case(path, workload, cluster, g0: np.ndarray, measurements: Sequence, flags: int = 0):
    """Writes a case file.  ``g0`` is in the layout returned by workloads.make_g0."""
    w = workload
    nb, nc = w.nb, cluster.nc
    chans = list(w.channels) + [0] * (4 - len(w.channels))
    with open(path, "wb") as f:
        f.write(b"DCACASE1")
        f.write(struct.pack("<8i", nb, nc, w.nw_half, w.n_sp, int(w.all_transfers),
                            w.freq_transfer, w.k_transfer, len(w.channels)))
        f.write(struct.pack("<4i", *chans))
        f.write(struct.pack("<2i", len(measurements), flags))
        f.write(struct.pack("<d", w.beta))
        f.write(np.ascontiguousarray(cluster.r_vecs, np.float64).tobytes())
        f.write(np.ascontiguousarray(cluster.k_vecs, np.float64).tobytes())
        # Tables are stored column major: element (i, j) at i + nc * j.
        for t in (cluster.k_add, cluster.k_sub, cluster.r_add, cluster.r_sub):
            f.write(np.asarray(t, np.int32).T.copy().tobytes())
        f.write(np.ascontiguousarray(w.model.a_vecs(), np.float64).tobytes())
        f.write(np.ascontiguousarray(g0, np.complex128).tobytes())
        for m in measurements:
            f.write(struct.pack("<i", m.sign))
            for s in m.sectors:
                f.write(struct.pack("<i", s.n))
                f.write(np.asarray(s.tau, np.float64).tobytes())
                for v in (s.left_band, s.right_band, s.left_site, s.right_site):
                    f.write(np.asarray(v, np.int32).tobytes())
                f.write(np.asarray(s.M, np.float64).tobytes(order="F"))


class Result:
    def __init__(self, g4: List[np.ndarray], mrw=None, mrw_sqr=None):
        self.g4 = g4
        self.mrw = mrw
        self.mrw_sqr = mrw_sqr


def read_result(path) -> Result:
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"DCAOUT01":
        raise ValueError("bad result magic")
    off = 8
    (n_ch,) = struct.unpack_from("<i", data, off)
    off += 4
    (g4_size,) = struct.unpack_from("<q", data, off)
    off += 8
    g4 = []
    for _ in range(n_ch):
        g4.append(np.frombuffer(data, np.complex128, g4_size, off).copy())
        off += 16 * g4_size
    (has_sp,) = struct.unpack_from("<i", data, off)
    off += 4
    mrw = mrw_sqr = None
    if has_sp:
        (sp_size,) = struct.unpack_from("<q", data, off)
        off += 8
        mrw = np.frombuffer(data, np.complex128, sp_size, off).copy()
        off += 16 * sp_size
        (has_sqr,) = struct.unpack_from("<i", data, off)
        off += 4
        if has_sqr:
            mrw_sqr = np.frombuffer(data, np.complex128, sp_size, off).copy()
    return Result(g4, mrw, mrw_sqr)
