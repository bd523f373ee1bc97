"""Python handle on the CPU restatement oracle (oracle/_build/liboracle.so).

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm use it as the checker or the timed CPU baseline; the product never imports it.
The C structs mirror include/dcaacc.h (declared here again so the oracle does not depend on the
product library being built).
"""

from __future__ import annotations

import ctypes
import os
import sys
import time
import subprocess
from ctypes import POINTER, c_double, c_int32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "tp_ref")


class _TpConfig(ctypes.Structure):
    _fields_ = [
        ("n_bands", c_int32), ("n_sites", c_int32), ("n_w_half", c_int32), ("n_sp_freq", c_int32),
        ("n_k_ex", c_int32), ("k_ex", POINTER(c_int32)), ("n_w_ex", c_int32), ("w_ex", POINTER(c_int32)),
        ("n_channels", c_int32), ("channels", POINTER(c_int32)), ("beta", c_double),
        ("r_vecs", POINTER(c_double)), ("k_vecs", POINTER(c_double)), ("a_vecs", POINTER(c_double)),
        ("k_add", POINTER(c_int32)), ("k_sub", POINTER(c_int32)), ("non_density", c_int32),
        ("precision", c_int32), ("max_batch", c_int32), ("max_order", c_int32),
        ("accumulators", c_int32),
    ]


class _SpConfig(ctypes.Structure):
    _fields_ = [
        ("n_bands", c_int32), ("n_sites", c_int32), ("n_sp_freq", c_int32), ("beta", c_double),
        ("r_sub", POINTER(c_int32)), ("accumulate_m_sqr", c_int32), ("max_order", c_int32),
    ]


class _Sector(ctypes.Structure):
    _fields_ = [
        ("n", c_int32), ("tau", POINTER(c_double)), ("left_band", POINTER(c_int32)),
        ("right_band", POINTER(c_int32)), ("left_site", POINTER(c_int32)),
        ("right_site", POINTER(c_int32)), ("M", c_void_p), ("ldm", c_int32), ("m_on_device", c_int32),
    ]


def build():
    """Compiles liboracle.so (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_tp_g4_size.restype = ctypes.c_size_t
        L.oracle_tp_g4_size.argtypes = [c_void_p]
        L.oracle_tp_g_size.restype = ctypes.c_size_t
        L.oracle_tp_g_size.argtypes = [c_void_p]
        L.oracle_sp_out_size.restype = ctypes.c_size_t
        L.oracle_sp_out_size.argtypes = [c_void_p]
        L.oracle_sp_ftau_size.restype = ctypes.c_size_t
        L.oracle_sp_ftau_size.argtypes = [c_void_p]
        for n in ("oracle_tp_destroy", "oracle_sp_destroy"):
            getattr(L, n).argtypes = [c_void_p]
            getattr(L, n).restype = None
        L.oracle_tp_accumulate.argtypes = [c_void_p, POINTER(_Sector), c_int32]
        L.oracle_sp_accumulate.argtypes = [c_void_p, POINTER(_Sector), c_double]
        L.oracle_tp_get_g4.argtypes = [c_void_p, c_int32, POINTER(c_double), ctypes.c_size_t]
        L.oracle_tp_get_g.argtypes = [c_void_p, c_int32, POINTER(c_double), ctypes.c_size_t]
        L.oracle_sp_get.argtypes = [c_void_p, c_int32, POINTER(c_double), ctypes.c_size_t]
        L.oracle_sp_get_ftau.argtypes = [c_void_p, c_int32, POINTER(c_double), ctypes.c_size_t]
        L.oracle_tp_reset.argtypes = [c_void_p]
        L.oracle_sp_reset.argtypes = [c_void_p]
        L.oracle_sp_finalize.argtypes = [c_void_p]
        L.oracle_run_case.argtypes = [ctypes.c_char_p, ctypes.c_char_p, c_int32, c_int32]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {lib().oracle_last_error().decode()}")


def _ip(a):
    return a.ctypes.data_as(POINTER(c_int32))


def _dp(a):
    return a.ctypes.data_as(POINTER(c_double))


def _sectors(M_pair, configs, keep):
    secs = (_Sector * 2)()
    for s in range(2):
        c = configs[s]
        arrs = [np.ascontiguousarray(c.tau, np.float64)] + [
            np.ascontiguousarray(getattr(c, k), np.int32)
            for k in ("left_band", "right_band", "left_site", "right_site")]
        n = arrs[0].shape[0]
        M = np.asfortranarray(np.asarray(M_pair[s], np.float64)) if n else np.zeros((1, 1), order="F")
        keep.extend(arrs + [M])
        secs[s] = _Sector(n, _dp(arrs[0]), _ip(arrs[1]), _ip(arrs[2]), _ip(arrs[3]), _ip(arrs[4]),
                          c_void_p(M.ctypes.data), max(n, 1), 0)
    return secs


class OracleTp:
    """FP64 CPU two-particle accumulator (restatement of TpAccumulator<CPU>)."""

    def __init__(self, G0, p):
        self.p = p
        self._keep = [np.ascontiguousarray(p.k_ex, np.int32), np.ascontiguousarray(p.w_ex, np.int32),
                      np.ascontiguousarray(p.channels, np.int32),
                      np.ascontiguousarray(p.r_vecs, np.float64), np.ascontiguousarray(p.k_vecs, np.float64),
                      np.ascontiguousarray(p.a_vecs, np.float64),
                      np.ascontiguousarray(np.asarray(p.k_add, np.int32).T),
                      np.ascontiguousarray(np.asarray(p.k_sub, np.int32).T)]
        k_ex, w_ex, ch, rv, kv, av, kadd, ksub = self._keep
        cfg = _TpConfig(p.n_bands, p.n_sites, p.n_w_half, p.n_sp_freq, len(k_ex), _ip(k_ex), len(w_ex),
                        _ip(w_ex), len(ch), _ip(ch), p.beta, _dp(rv), _dp(kv), _dp(av), _ip(kadd),
                        _ip(ksub), int(p.non_density), 0, 1, p.max_order, 1)
        g0 = np.ascontiguousarray(G0, np.complex128).reshape(-1)
        self._h = c_void_p()
        _check(lib().oracle_tp_create(ctypes.byref(cfg), _dp(g0.view(np.float64)), ctypes.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_tp_destroy(self._h)
            self._h = None

    def resetAccumulation(self):
        _check(lib().oracle_tp_reset(self._h))

    def accumulate(self, M_pair, configs, sign):
        keep = []
        _check(lib().oracle_tp_accumulate(self._h, _sectors(M_pair, configs, keep), int(sign)))

    def get_G4(self):
        size = lib().oracle_tp_g4_size(self._h)
        out = []
        for c in range(len(self.p.channels)):
            g = np.empty(size, np.complex128)
            _check(lib().oracle_tp_get_g4(self._h, c, _dp(g.view(np.float64)), size))
            out.append(g)
        return out

    def get_G(self, spin):
        size = lib().oracle_tp_g_size(self._h)
        g = np.empty(size, np.complex128)
        _check(lib().oracle_tp_get_g(self._h, spin, _dp(g.view(np.float64)), size))
        return g


class OracleSp:
    """FP64 CPU single-particle accumulator (restatement of SpAccumulator<CPU> + Dnfft1D)."""

    def __init__(self, p, accumulate_m_squared=False):
        self.p = p
        self._rsub = np.ascontiguousarray(np.asarray(p.r_sub, np.int32).T)
        cfg = _SpConfig(p.n_bands, p.n_sites, p.n_sp_freq, p.beta, _ip(self._rsub),
                        int(accumulate_m_squared), p.max_order)
        self._h = c_void_p()
        _check(lib().oracle_sp_create(ctypes.byref(cfg), ctypes.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_sp_destroy(self._h)
            self._h = None

    def resetAccumulation(self):
        _check(lib().oracle_sp_reset(self._h))

    def accumulate(self, M_pair, configs, factor):
        keep = []
        _check(lib().oracle_sp_accumulate(self._h, _sectors(M_pair, configs, keep), float(factor)))

    def finalize(self):
        _check(lib().oracle_sp_finalize(self._h))

    def get(self, sqr=False):
        size = lib().oracle_sp_out_size(self._h)
        out = np.empty(size, np.complex128)
        _check(lib().oracle_sp_get(self._h, int(sqr), _dp(out.view(np.float64)), size))
        return out

    def get_ftau(self, spin):
        size = lib().oracle_sp_ftau_size(self._h)
        out = np.empty(size, np.float64)
        _check(lib().oracle_sp_get_ftau(self._h, spin, _dp(out), size))
        return out


def run_case(case_path, out_path, tp=True, sp=True, warmup=0, report=False):
    """Runs the restatement on a case file.  report: prints the wall-clock window of the whole run
    on stderr in tp_ref's --time format (warm-up measurements are inside it: the restatement has
    no per-measurement timer)."""
    t0 = time.time()
    _check(lib().oracle_run_case(str(case_path).encode(), str(out_path).encode(), int(tp), int(sp)))
    if report:
        print(f"tp_epoch_start={t0!r} tp_epoch_end={time.time()!r} blas=none", file=sys.stderr)


def run_reference(case_path, out_path, tp=True, sp=True, timeout=3600):
    """Runs the reference's own CPU accumulators (oracle/_ref/tp_ref) on a case file."""
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    args = [REF_BIN, str(case_path), str(out_path), "--time"]
    if not tp:
        args.append("--no-tp")
    if not sp:
        args.append("--no-sp")
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"tp_ref failed: {r.stderr}")
    return r.stderr
