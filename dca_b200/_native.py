"""ctypes binding of libdcaacc.so (the C ABI declared in include/dcaacc.h).

The library is built in-tree (dca_b200/_lib/libdcaacc.so, by ``python -m dca_b200.build`` or
``__graft_entry__.build()``).  There is no fallback: if the library is missing or does not load,
importing this module raises, and every accumulator call fails loudly.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int32, c_size_t, c_uint64, c_void_p

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libdcaacc.so")

OK = 0
STATUS_NAMES = {
    0: "DCAACC_OK",
    1: "DCAACC_INVALID_ARG",
    2: "DCAACC_NOT_READY",
    3: "DCAACC_OOM",
    4: "DCAACC_CUDA_ERR",
    5: "DCAACC_DEVICE_INDEX_ERR",
    6: "DCAACC_UNSUPPORTED",
}

PRECISION_FP64 = 0
PRECISION_MIXED = 1


class TpConfig(ctypes.Structure):
    _fields_ = [
        ("n_bands", c_int32),
        ("n_sites", c_int32),
        ("n_w_half", c_int32),
        ("n_sp_freq", c_int32),
        ("n_k_ex", c_int32),
        ("k_ex", POINTER(c_int32)),
        ("n_w_ex", c_int32),
        ("w_ex", POINTER(c_int32)),
        ("n_channels", c_int32),
        ("channels", POINTER(c_int32)),
        ("beta", c_double),
        ("r_vecs", POINTER(c_double)),
        ("k_vecs", POINTER(c_double)),
        ("a_vecs", POINTER(c_double)),
        ("k_add", POINTER(c_int32)),
        ("k_sub", POINTER(c_int32)),
        ("non_density", c_int32),
        ("precision", c_int32),
        ("max_batch", c_int32),
        ("max_order", c_int32),
        ("accumulators", c_int32),
    ]


class SpConfig(ctypes.Structure):
    _fields_ = [
        ("n_bands", c_int32),
        ("n_sites", c_int32),
        ("n_sp_freq", c_int32),
        ("beta", c_double),
        ("r_sub", POINTER(c_int32)),
        ("accumulate_m_sqr", c_int32),
        ("max_order", c_int32),
        ("stamping", c_int32),
    ]


class Sector(ctypes.Structure):
    """dcaacc_sector; the pointer fields are declared void* (same ABI) so that addresses can be
    assigned as integers without building ctypes pointer objects per call."""
    _fields_ = [
        ("n", c_int32),
        ("tau", c_void_p),          # const double*
        ("left_band", c_void_p),    # const int32_t*
        ("right_band", c_void_p),
        ("left_site", c_void_p),
        ("right_site", c_void_p),
        ("M", c_void_p),
        ("ldm", c_int32),
        ("m_on_device", c_int32),
    ]


class DcaAccError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m dca_b200.build` "
            "(the accumulators have no non-CUDA implementation)")
    lib = ctypes.CDLL(LIB_PATH)
    i, p, sz = c_int32, c_void_p, c_size_t
    sigs = {
        "dcaacc_last_error": (ctypes.c_char_p, []),
        "dcaacc_tp_create": (i, [POINTER(TpConfig), POINTER(c_double), POINTER(p)]),
        "dcaacc_tp_destroy": (None, [p]),
        "dcaacc_tp_reset": (i, [p]),
        "dcaacc_tp_accumulate": (i, [p, POINTER(Sector), i, POINTER(c_double)]),
        "dcaacc_tp_accumulate_typed": (i, [p, i, POINTER(Sector), i, POINTER(c_double), POINTER(c_double),
                                           POINTER(c_double)]),
        "dcaacc_tp_accumulate_batch": (i, [p, i, POINTER(Sector), POINTER(c_int32), POINTER(c_double)]),
        "dcaacc_tp_flush": (i, [p]),
        "dcaacc_tp_finalize": (i, [p]),
        "dcaacc_tp_get_g4": (i, [p, i, POINTER(c_double), sz]),
        "dcaacc_tp_g4_size": (sz, [p]),
        "dcaacc_tp_sum_to": (i, [p, p]),
        "dcaacc_tp_get_g": (i, [p, i, POINTER(c_double), sz]),
        "dcaacc_tp_set_stream": (i, [p, p]),
        "dcaacc_tp_get_stream": (p, [p]),
        "dcaacc_tp_synchronize": (i, [p]),
        "dcaacc_tp_device_fingerprint": (sz, [p]),
        "dcaacc_tp_kernel_launches": (c_uint64, [p]),
        "dcaacc_tp_mirror_mode": (i, [p]),
        "dcaacc_tp_enable_timing": (i, [p, i]),
        "dcaacc_tp_stage_times": (i, [p, POINTER(c_double), POINTER(c_uint64), i]),
        "dcaacc_tp_set_graphs": (i, [p, i]),
        "dcaacc_tp_graph_stats": (i, [p, POINTER(c_uint64), POINTER(c_uint64)]),
        "dcaacc_tp_tuning_settled": (i, [p]),
        "dcaacc_tp_tuning_report": (i, [p, ctypes.c_char_p, sz, POINTER(sz)]),
        "dcaacc_tp_peek_g4": (i, [p, i, sz, sz, POINTER(c_double)]),
        "dcaacc_tp_peek_g4_async": (i, [p, i, sz, sz, POINTER(c_double)]),
        "dcaacc_tp_compute_g_noalloc": (i, [POINTER(TpConfig), p, POINTER(Sector), p, p]),
        "dcaacc_sp_create": (i, [POINTER(SpConfig), POINTER(p)]),
        "dcaacc_sp_destroy": (None, [p]),
        "dcaacc_sp_reset": (i, [p]),
        "dcaacc_sp_accumulate": (i, [p, POINTER(Sector), c_double]),
        "dcaacc_sp_finalize": (i, [p]),
        "dcaacc_sp_get_m_r_w": (i, [p, POINTER(c_double), sz]),
        "dcaacc_sp_get_m_r_w_sqr": (i, [p, POINTER(c_double), sz]),
        "dcaacc_sp_sum_to": (i, [p, p]),
        "dcaacc_sp_set_stream": (i, [p, p]),
        "dcaacc_sp_synchronize": (i, [p]),
        "dcaacc_sp_device_fingerprint": (sz, [p]),
        "dcaacc_sp_kernel_launches": (c_uint64, [p]),
        "dcaacc_sp_get_single_measurement_m_r_w": (i, [p, POINTER(c_double), sz]),
        "dcaacc_sp_get_single_measurement_f_tau": (i, [p, POINTER(c_double), sz]),
        "dcaacc_sp_clear_single_measurement": (i, [p]),
        "dcaacc_sp_f_tau_size": (sz, [p]),
        "dcaacc_tp_static_device_fingerprint": (sz, []),
        "dcaacc_tp_sign_sum": (i, [p, POINTER(c_double), POINTER(c_uint64)]),
        "dcaacc_tp_share_g4": (i, [p, p]),
        "dcaacc_tp_reset_loop": (i, [p, i]),
        "dcaacc_tp_get_g4_normalized": (i, [p, i, POINTER(c_double), sz]),
        "dcaacc_tp_set_fault_injection": (i, [p, i, ctypes.c_uint32]),
        "dcaacc_set_allocation_failure": (i, [ctypes.c_int64]),
        "dcaacc_tp_g4_shard": (i, [i, i, i, POINTER(c_int32), POINTER(c_int32)]),
        "dcaacc_tp_g4_place_shard": (i, [POINTER(TpConfig), i, i, POINTER(c_double), sz, POINTER(c_double), sz]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int):
    if status != OK:
        raise DcaAccError(status, lib.dcaacc_last_error().decode(errors="replace"))
