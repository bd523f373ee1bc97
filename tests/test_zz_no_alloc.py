"""The allocation-free entry point, dcaacc_tp_compute_g_noalloc.

It serves callers that cannot allocate device memory while they run (an application whose
device memory is entirely held by its own pool allocator, or a per-measurement loop that must not
stall on cudaMalloc's device-wide synchronisation): it computes one measurement's G with its
scratch in an array compiled into the library instead of memory it allocates.  This file checks,
through the C ABI, that two calls in a row give the same G as the regular FP64 accumulator handle,
to the FP64 tolerance used elsewhere in the tests.  It is collected last so that a run stopping at
the first failure has already run every other test, and it passes on its own or after them.
"""

import ctypes

import numpy as np
import pytest

from helpers import golden, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _config(p, keep):
    from dca_b200 import _native as N
    arrs = [np.ascontiguousarray(p.k_ex, np.int32), np.ascontiguousarray(p.w_ex, np.int32),
            np.ascontiguousarray(p.channels, np.int32), np.ascontiguousarray(p.r_vecs, np.float64),
            np.ascontiguousarray(p.k_vecs, np.float64), np.ascontiguousarray(p.a_vecs, np.float64),
            np.ascontiguousarray(np.asarray(p.k_add, np.int32).T),
            np.ascontiguousarray(np.asarray(p.k_sub, np.int32).T)]
    keep.extend(arrs)
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    k_ex, w_ex, ch, rv, kv, av, kadd, ksub = arrs
    return N.TpConfig(p.n_bands, p.n_sites, p.n_w_half, p.n_sp_freq, len(k_ex), ip(k_ex), len(w_ex),
                      ip(w_ex), len(ch), ip(ch), p.beta, dp(rv), dp(kv), dp(av), ip(kadd), ip(ksub),
                      0, 0, 1, p.max_order, 1)


def _blocks_to_reference_layout(g, p):
    """(spin, w_r, w_c, r, c) block layout -> per spin (b1, b2, k1, k2, w1, w2) flattened."""
    nb, nc = p.n_bands, p.n_sites
    ext = max(abs(w) for w in p.w_ex)
    nwe = 2 * p.n_w_half + 2 * ext
    R = nb * nc
    g = g.reshape(2, nwe, nwe, nc, nb, nc, nb)  # s, w_r, w_c, k_r, b_r, k_c, b_c
    out = []
    for s in range(2):
        # target C-order axes (w2, w1, k2, k1, b2, b1) so that b1 is fastest
        out.append(np.transpose(g[s], (1, 0, 4, 2, 5, 3)).reshape(-1))
    return out


def test_noalloc_matches_accumulator_on_two_consecutive_calls():
    import torch

    from dca_b200 import _native as N
    from dca_b200.accumulators import TpAccumulator, _make_sectors

    case, _ = golden("sq4_q5")  # its second measurement has an empty spin sector
    p = case.tp_params()
    G0_dev = torch.from_numpy(case.G0.view(np.float64).copy()).cuda()
    ext = max(abs(w) for w in p.w_ex)
    D = p.n_bands * p.n_sites * (2 * p.n_w_half + 2 * ext)
    G_out = torch.empty(2 * D * D * 2, dtype=torch.float64, device="cuda")

    for m in case.measurements:  # two calls in a row, different measurements
        keep = []
        cfg = _config(p, keep)
        M_dev = [torch.from_numpy(np.ascontiguousarray(s.M.T)).cuda().t() if s.n else
                 torch.zeros((1, 1), dtype=torch.float64, device="cuda") for s in m.sectors]
        secs = _make_sectors(M_dev, list(m.sectors), keep)
        G_out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = N.lib.dcaacc_tp_compute_g_noalloc(ctypes.byref(cfg), ctypes.c_void_p(G0_dev.data_ptr()), secs,
                                               ctypes.c_void_p(G_out.data_ptr()), None)
        assert rc == 0, N.lib.dcaacc_last_error()
        torch.cuda.synchronize()
        got = _blocks_to_reference_layout(G_out.cpu().numpy().view(np.complex128), p)

        acc = TpAccumulator(case.G0, p)
        acc.resetAccumulation(0)
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        for spin in range(2):
            want = acc.get_G(spin)
            assert np.all(np.isfinite(got[spin]))
            assert rel_err(got[spin], want) <= FP64_TOL


def test_noalloc_rejects_oversized_problem():
    import torch

    from dca_b200 import _native as N
    from dca_b200.accumulators import _make_sectors
    from dca_b200 import workloads as W

    case, _ = golden("c1_mag")
    p = case.tp_params()
    keep = []
    cfg = _config(p, keep)
    n = 600  # beyond the 512-vertex limit
    sec = W.Sector(np.linspace(0, 1, n), *(np.zeros(n, np.int32) for _ in range(4)), np.eye(n))
    M_dev = [torch.eye(n, dtype=torch.float64, device="cuda")] * 2
    secs = _make_sectors(M_dev, [sec, sec], keep)
    out = torch.empty(2, dtype=torch.float64, device="cuda")
    G0_dev = torch.from_numpy(case.G0.view(np.float64).copy()).cuda()
    rc = N.lib.dcaacc_tp_compute_g_noalloc(ctypes.byref(cfg), ctypes.c_void_p(G0_dev.data_ptr()), secs,
                                           ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and b"512" in N.lib.dcaacc_last_error()


def test_noalloc_rejects_cluster_beyond_shared_memory_tiles():
    """nb * Nc = 64 (one band on an 8 x 8 cluster) is within the orbital limit but needs more than
    227 KB of shared memory per block in the FP64 front-end: rejected before any GPU work."""
    import dataclasses

    import torch

    from dca_b200 import _native as N
    from dca_b200 import workloads as W
    from dca_b200.accumulators import TpParameters, _make_sectors

    w = dataclasses.replace(W.WORKLOADS["c1"], cluster_kind=("square", 8), n_range=(8, 8))
    cl = w.cluster()
    p = TpParameters.from_workload(w, cl)
    keep = []
    cfg = _config(p, keep)
    m = W.make_measurements(w, 1)[0]
    M_dev = [torch.from_numpy(np.ascontiguousarray(s.M.T)).cuda().t() for s in m.sectors]
    secs = _make_sectors(M_dev, list(m.sectors), keep)
    g0 = W.make_g0(w.model, cl, w.beta, w.chemical_potential(), w.n_sp).reshape(-1)
    G0_dev = torch.from_numpy(g0.view(np.float64).copy()).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = N.lib.dcaacc_tp_compute_g_noalloc(ctypes.byref(cfg), ctypes.c_void_p(G0_dev.data_ptr()), secs,
                                           ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and b"shared-memory" in N.lib.dcaacc_last_error()
    torch.cuda.synchronize()
    assert not torch.any(out)


def test_noalloc_refuses_stream_capture():
    """A call on a stream that is being captured returns DCAACC_INVALID_ARG without enqueueing
    anything (its uploads come from host stack memory, which a replayed graph could not read)."""
    import torch

    from dca_b200 import _native as N
    from dca_b200.accumulators import _make_sectors

    case, _ = golden("c1_mag")
    p = case.tp_params()
    keep = []
    cfg = _config(p, keep)
    m = case.measurements[0]
    M_dev = [torch.from_numpy(np.ascontiguousarray(s.M.T)).cuda().t() for s in m.sectors]
    secs = _make_sectors(M_dev, list(m.sectors), keep)
    G0_dev = torch.from_numpy(case.G0.view(np.float64).copy()).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = N.lib.dcaacc_tp_compute_g_noalloc(ctypes.byref(cfg), ctypes.c_void_p(G0_dev.data_ptr()), secs,
                                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream))
        out.add_(1.0)  # the capture stays valid: nothing of the refused call was recorded
    assert rc == 1 and b"stream capture" in N.lib.dcaacc_last_error()
    g.replay()
    torch.cuda.synchronize()
    assert torch.all(out == 1.0)
