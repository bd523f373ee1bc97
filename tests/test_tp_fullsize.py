"""Parity at the full sizes of the multiband and large-cluster configurations, through the C ABI.

* c5 (6x6 single band, Nw = 128, all 36 momentum transfers, PH-magnetic; G4 is 764M complex
  entries, 12.2 GB FP64): one full measurement of the plain FP64 GPU path against the oracle
  (FP64, <= 1e-12), and the seeded 256-measurement accuracy subset -- two full batches of 128
  through the mixed path against the FP64 GPU path, <= 1e-6 per channel.
* c4 (three-band Emery model on the Betts 8 cluster, Nw = 32, 8 momentum x 4 frequency transfers,
  PP up-down): two full batches of 32 through the mixed path against the FP64 GPU path (whose
  full-size c4 measurement is pinned to the oracle in test_tp_gpu.py).

Run as a script (python tests/test_tp_fullsize.py) it prints the c5 subset's errors as JSON.
"""

import json
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from helpers import case_from_workload  # noqa: E402
from dca_b200 import workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-6
C5_SUBSET = 256  # seeded measurements 0..255 of the c5 workload


def rel_err_chunked(a, b, chunk=1 << 24):
    """||a - b|| / ||b|| without a full-size temporary (G4 here is up to 12 GB)."""
    num = den = 0.0
    for i in range(0, b.size, chunk):
        x, y = a[i:i + chunk], b[i:i + chunk]
        num += float(np.vdot(x - y, x - y).real)
        den += float(np.vdot(y, y).real)
    return (num / den) ** 0.5 if den > 0 else num ** 0.5


def max_abs_rel(a, b, chunk=1 << 24):
    """max |a - b| / max |b|."""
    md = mb = 0.0
    for i in range(0, b.size, chunk):
        md = max(md, float(np.max(np.abs(a[i:i + chunk] - b[i:i + chunk]))))
        mb = max(mb, float(np.max(np.abs(b[i:i + chunk]))))
    return md / mb if mb > 0 else md


def _gpu(case, measurements, **kw):
    from dca_b200.accumulators import TpAccumulator
    acc = TpAccumulator(case.G0, case.tp_params(**kw))
    acc.resetAccumulation(0)
    for m in measurements:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    acc.finalize()
    return acc


def _oracle(oracle_lib, case, measurements):
    acc = oracle_lib.OracleTp(case.G0, case.tp_params())
    for m in measurements:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    return acc


@pytest.mark.parametrize("wname", ["c5"])  # c2 and c4: test_tp_gpu.py
def test_fp64_full_measurement_matches_oracle(oracle_lib, wname):
    case = case_from_workload(W.WORKLOADS[wname], 1)
    m = case.measurements
    gpu = _gpu(case, m, precision=0, max_batch=1)
    got = gpu.get_G4()
    del gpu
    want = _oracle(oracle_lib, case, m).get_G4()
    for a, b in zip(got, want):
        err = rel_err_chunked(a, b)
        print(wname, "FP64 GPU vs oracle, one full measurement:", err)
        assert err <= FP64_TOL


def c5_subset_errors(n_meas=C5_SUBSET):
    """Mixed vs FP64 GPU on the seeded c5 subset: per channel the relative Frobenius error and
    max |difference| / max |G4|."""
    w = W.WORKLOADS["c5"]
    case = case_from_workload(w, n_meas)
    ms = case.measurements
    fp64 = _gpu(case, ms, precision=0, max_batch=1)
    want = fp64.get_G4()
    del fp64
    mixed = _gpu(case, ms, precision=1, max_batch=w.batch)
    got = mixed.get_G4()
    mode = mixed.mirror_mode()
    del mixed
    orders = [s.n for m in ms for s in m.sectors]
    return {"workload": w.describe(), "measurements": n_meas, "mixed_batches": -(-n_meas // w.batch),
            "orders": [min(orders), max(orders)], "mirror_mode": mode,
            "rel_frobenius": [rel_err_chunked(a, b) for a, b in zip(got, want)],
            "max_abs_over_max": [max_abs_rel(a, b) for a, b in zip(got, want)]}


def test_c5_seeded_subset_mixed_vs_fp64():
    r = c5_subset_errors()
    print("c5 seeded subset:", json.dumps(r))
    assert max(r["rel_frobenius"]) <= MIXED_TOL


def test_c4_full_batches_mixed_vs_fp64():
    w = W.WORKLOADS["c4"]
    case = case_from_workload(w, 2 * w.batch)
    fp64 = _gpu(case, case.measurements, precision=0, max_batch=1)
    mixed = _gpu(case, case.measurements, precision=1, max_batch=w.batch)
    for a, b in zip(mixed.get_G4(), fp64.get_G4()):
        err = rel_err_chunked(a, b)
        print("c4 mixed vs FP64 GPU, two full batches of 32:", err, max_abs_rel(a, b))
        assert err <= MIXED_TOL


if __name__ == "__main__":
    print(json.dumps(c5_subset_errors()))
