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


# The C ABI's entry points.  A change to the header must be made here too (and in the Python
# binding), so that an entry point cannot appear or disappear unnoticed.
ENTRY_POINTS = """
dcaacc_last_error dcaacc_set_allocation_failure
dcaacc_tp_create dcaacc_tp_destroy dcaacc_tp_reset dcaacc_tp_reset_loop dcaacc_tp_share_g4
dcaacc_tp_accumulate dcaacc_tp_accumulate_typed dcaacc_tp_accumulate_batch dcaacc_tp_flush dcaacc_tp_finalize
dcaacc_tp_get_g4 dcaacc_tp_g4_size dcaacc_tp_sum_to dcaacc_tp_get_g dcaacc_tp_set_stream
dcaacc_tp_get_stream dcaacc_tp_synchronize dcaacc_tp_device_fingerprint dcaacc_tp_kernel_launches
dcaacc_tp_sign_sum dcaacc_tp_get_g4_normalized dcaacc_tp_static_device_fingerprint
dcaacc_tp_mirror_mode dcaacc_tp_enable_timing dcaacc_tp_stage_times dcaacc_tp_set_graphs
dcaacc_tp_graph_stats dcaacc_tp_tuning_settled dcaacc_tp_tuning_report dcaacc_tp_peek_g4
dcaacc_tp_peek_g4_async dcaacc_tp_compute_g_noalloc dcaacc_tp_set_fault_injection
dcaacc_tp_g4_shard dcaacc_tp_g4_place_shard
dcaacc_sp_create dcaacc_sp_destroy dcaacc_sp_reset dcaacc_sp_accumulate dcaacc_sp_finalize
dcaacc_sp_get_m_r_w dcaacc_sp_get_m_r_w_sqr dcaacc_sp_sum_to dcaacc_sp_get_single_measurement_m_r_w
dcaacc_sp_get_single_measurement_f_tau dcaacc_sp_clear_single_measurement dcaacc_sp_f_tau_size
dcaacc_sp_set_stream dcaacc_sp_synchronize dcaacc_sp_device_fingerprint dcaacc_sp_kernel_launches
""".split()


def test_header_declares_exactly_the_known_entry_points():
    """The header's declarations are the list above, and the Python binding types each of them."""
    from dca_b200 import _native
    assert sorted(ENTRY_POINTS) == declared_symbols()
    for s in ENTRY_POINTS:
        assert getattr(_native.lib, s).argtypes is not None, s
