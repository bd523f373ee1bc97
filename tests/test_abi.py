"""The C ABI library loads and exports what include/dcaacc.h declares; host-side validation."""

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dcaacc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dcaacc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from dca_b200 import _native
    syms = declared_symbols()
    assert len(syms) >= 29
    for s in syms:
        assert hasattr(_native.lib, s), s


def test_static_device_fingerprint_is_the_static_scratch():
    """staticDeviceFingerprint: the process-wide device state is the allocation-free entry point's
    48 MiB static scratch array (no device call is needed to report it)."""
    from dca_b200.accumulators import TpAccumulator
    assert TpAccumulator.staticDeviceFingerprint() == 48 << 20


def test_invalid_configuration_rejected_before_any_device_work():
    from dca_b200 import _native as N
    from dca_b200 import workloads as W
    w = W.WORKLOADS["c1"]
    cl = w.cluster()
    k_ex = np.array([0], np.int32)
    w_ex = np.array([0], np.int32)
    ch = np.array([9], np.int32)  # not a FourPointType
    rv = np.ascontiguousarray(cl.r_vecs)
    kv = np.ascontiguousarray(cl.k_vecs)
    av = np.zeros((1, 2))
    kadd = np.ascontiguousarray(cl.k_add.T.astype(np.int32))
    ksub = np.ascontiguousarray(cl.k_sub.T.astype(np.int32))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cfg = N.TpConfig(1, cl.nc, 8, 64, 1, ip(k_ex), 1, ip(w_ex), 1, ip(ch), 10.0, dp(rv), dp(kv),
                     dp(av), ip(kadd), ip(ksub), 0, 0, 1, 64, 1)
    g0 = np.zeros(4 * cl.nc * 128 * 2)
    h = ctypes.c_void_p()
    assert N.lib.dcaacc_tp_create(ctypes.byref(cfg), dp(g0), ctypes.byref(h)) == 6  # UNSUPPORTED
    ch[0] = N.PRECISION_FP64 + 2
    kadd[0, 0] = 99  # corrupt table
    assert N.lib.dcaacc_tp_create(ctypes.byref(cfg), dp(g0), ctypes.byref(h)) == 1  # INVALID_ARG
    assert b"out of range" in N.lib.dcaacc_last_error()
    kadd[0, 0] = 0
    cfg.n_sp_freq = 2  # too few single-particle frequencies for the extended mesh
    assert N.lib.dcaacc_tp_create(ctypes.byref(cfg), dp(g0), ctypes.byref(h)) == 1
    assert b"too small" in N.lib.dcaacc_last_error()
    assert N.lib.dcaacc_tp_reset(None) == 1


def test_bench_reference_arm_prints_one_contract_line():
    """bench.py --impl reference (the reference's own CPU accumulator on the host cores, or the
    restatement where it was not built) prints one JSON line with the contract's keys."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "meas/s"
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "meas/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_integration_notes_cover_every_entry_point():
    """Every entry point the header declares has its row (reference counterpart or none) in the
    integration notes."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    doc = open(os.path.join(root, "INTEGRATION.md")).read()
    missing = [s for s in declared_symbols() if s not in doc]
    assert not missing, missing
