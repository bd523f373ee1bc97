"""Failure detection on the GPU, without a GPU fault: a bounded device wait made to run out
(the host reads an error status and the context stays usable), and device / pinned allocations
made to fail inside dcaacc_tp_create (DCAACC_OOM, nothing left allocated).  The reference has no
device-side failure detection on this path; its CPU accumulator throws std::bad_alloc on an
allocation failure (tp_accumulator_gpu.hpp:314-317), which DCAACC_OOM stands for here."""

import time

import numpy as np
import pytest

from helpers import case_from_workload, golden, rel_err
from dca_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _small_c3(n_range=(40, 80)):
    import dataclasses
    return dataclasses.replace(W.WORKLOADS["c3"], n_range=n_range)


def _feed(acc, ms):
    for m in ms:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)


@pytest.mark.parametrize("stop_step", [0, 5])
def test_bounded_wait_runs_out_and_the_handle_recovers(stop_step):
    """The tensor-core direct G4 term's first block stops feeding its consumers before pipeline
    step stop_step, so their bounded wait (2^14 polls here) runs out: finalize reports
    DCAACC_DEVICE_INDEX_ERR within seconds, and after resetAccumulation the same handle on the same
    GPU accumulates correctly again."""
    from dca_b200.accumulators import TpAccumulator
    case = case_from_workload(_small_c3(), 16)
    ms = case.measurements
    acc = TpAccumulator(case.G0, case.tp_params(precision=1, max_batch=8))
    acc.set_graphs(False)
    acc.resetAccumulation(0)
    acc.set_fault_injection(stop_step, 1 << 14)
    _feed(acc, ms)
    t0 = time.time()
    with pytest.raises(RuntimeError, match="DEVICE_INDEX_ERR.*timed out"):
        acc.finalize()
    assert time.time() - t0 < 20
    acc.set_fault_injection(-1, 0)
    acc.resetAccumulation(1)
    _feed(acc, ms)
    acc.finalize()
    ref = TpAccumulator(case.G0, case.tp_params(precision=1, max_batch=8))
    ref.set_graphs(False)
    ref.resetAccumulation(0)
    _feed(ref, ms)
    ref.finalize()
    for a, b in zip(acc.get_G4(), ref.get_G4()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [0, 1])
def test_allocation_failure_in_create_returns_oom_and_leaks_nothing(precision):
    """Every device or pinned allocation of a c3-sized handle (G4 537 MB, mixed-path workspace of
    several GB) is made to fail in turn: each create raises MemoryError (DCAACC_OOM), the device's
    free memory returns to where it was, and the handle created afterwards works."""
    import torch

    from dca_b200 import _native as N
    from dca_b200.accumulators import TpAccumulator
    case = case_from_workload(_small_c3((40, 60)), 2)
    params = case.tp_params(precision=precision, max_batch=8)
    warm = TpAccumulator(case.G0, params)  # loads the kernels creation launches
    del warm
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    try:
        for nth in range(1, 400):
            N.lib.dcaacc_set_allocation_failure(nth)
            try:
                acc = TpAccumulator(case.G0, params)
            except MemoryError as e:
                assert "injected allocation failure" in str(e)
                failures += 1
                torch.cuda.synchronize()
                assert free0 - torch.cuda.mem_get_info()[0] <= (4 << 20), nth
                continue
            break
    finally:
        N.lib.dcaacc_set_allocation_failure(0)
    assert failures >= 20
    acc.resetAccumulation(0)
    _feed(acc, case.measurements)
    acc.finalize()
    exact = TpAccumulator(case.G0, case.tp_params(precision=0, max_batch=1))
    exact.resetAccumulation(0)
    _feed(exact, case.measurements)
    exact.finalize()
    for a, b in zip(acc.get_G4(), exact.get_G4()):
        assert rel_err(a, b) <= (1e-12 if precision == 0 else 1e-6)
    del acc, exact
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] <= (4 << 20)
