"""Single-particle accumulator on the GPU against the reference outputs and the oracle."""

import numpy as np
import pytest

from conftest import GOLDEN_CASES
from helpers import case_from_workload, golden, rel_err
from dca_b200 import workloads as W

pytestmark = pytest.mark.gpu

SP_TOL = 1e-9  # the reference's own Dnfft1DGpu vs Dnfft1D tolerance (dnfft_1d_gpu_test.cpp:48-92)


def run_sp(case, measurements=None, sqr=True):
    from dca_b200.accumulators import SpAccumulator
    acc = SpAccumulator(case.sp_params(), accumulate_m_squared=sqr)
    acc.resetAccumulation()
    for m in (measurements if measurements is not None else case.measurements):
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    acc.finalize()
    return acc


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_sp_matches_reference_golden(name):
    case, ref = golden(name)
    acc = run_sp(case, sqr=ref.mrw_sqr is not None)
    assert rel_err(acc.get_sign_times_M_r_w(), ref.mrw) <= SP_TOL
    if ref.mrw_sqr is not None:
        assert rel_err(acc.get_sign_times_M_r_w_sqr(), ref.mrw_sqr) <= SP_TOL


@pytest.mark.parametrize("wname", ["c2", "c4"])
def test_sp_full_size_matches_oracle(oracle_lib, wname):
    case = case_from_workload(W.WORKLOADS[wname], 2)
    acc = run_sp(case, sqr=False)
    ora = oracle_lib.OracleSp(case.sp_params())
    for m in case.measurements:
        ora.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    ora.finalize()
    assert rel_err(acc.get_sign_times_M_r_w(), ora.get()) <= SP_TOL


def test_sp_sum_to_linearity():
    from dca_b200.accumulators import SpAccumulator
    case, _ = golden("c1_mag")
    a = SpAccumulator(case.sp_params())
    b = SpAccumulator(case.sp_params())
    a.resetAccumulation()
    b.resetAccumulation()
    m0, m1 = case.measurements[:2]
    a.accumulate([s.M for s in m0.sectors], list(m0.sectors), m0.sign)
    b.accumulate([s.M for s in m1.sectors], list(m1.sectors), m1.sign)
    a.sumTo(b)
    b.finalize()
    both = run_sp(case, [m0, m1], sqr=False)
    assert rel_err(b.get_sign_times_M_r_w(), both.get_sign_times_M_r_w()) <= 1e-13


def test_sp_single_measurement_matches_oracle(oracle_lib):
    """Stamping (the reference's stamping_period() > 0): after each accumulate the handle also holds
    that measurement's own f(tau); its M(r, w) equals the oracle's for an accumulator fed only that
    measurement, clearSingleMeasurement zeroes it, and the running sum is unchanged."""
    from dca_b200.accumulators import LogicError, SpAccumulator
    case, _ = golden("c1_mag")
    p = case.sp_params(stamping=True)
    acc = SpAccumulator(p)
    acc.resetAccumulation()
    ms = case.measurements[:3]
    for m in ms:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        ora = oracle_lib.OracleSp(case.sp_params())
        ora.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        ora.finalize()
        assert rel_err(acc.get_single_measurement_sign_times_MFunction(), ora.get()) <= SP_TOL
    ft = acc.get_single_measurement_sign_times_MFunction_time()
    assert ft.shape == (2, p.n_bands ** 2 * p.n_sites, 8 * p.n_sp_freq + 16) and np.any(ft != 0)
    acc.clearSingleMeasurement()
    assert not np.any(acc.get_single_measurement_sign_times_MFunction_time())
    acc.finalize()
    ref = run_sp(case, ms, sqr=False)  # shared-memory atomics: equal up to summation order
    assert rel_err(acc.get_sign_times_M_r_w(), ref.get_sign_times_M_r_w()) <= 1e-13
    plain = SpAccumulator(case.sp_params())
    with pytest.raises(LogicError):  # no stamping
        plain.clearSingleMeasurement()


def test_sp_errors():
    from dca_b200.accumulators import LogicError, SpAccumulator
    case, _ = golden("c1_mag")
    acc = SpAccumulator(case.sp_params())
    m = case.measurements[0]
    with pytest.raises(LogicError):
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), 1.0)
    acc.resetAccumulation()
    acc.finalize()
    with pytest.raises(LogicError):  # M^2 was not accumulated
        acc.get_sign_times_M_r_w_sqr()
    with pytest.raises(LogicError):  # already finalized
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), 1.0)
