"""Two-particle accumulator on the GPU, through the C ABI, against the oracle / reference outputs."""

import numpy as np
import pytest

from conftest import GOLDEN_CASES
from helpers import case_from_workload, golden, rel_err
from dca_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12   # plain FP64 path vs the FP64 reference
MIXED_TOL = 1e-6   # mixed-precision path vs FP64 (relative Frobenius error per channel)


def run_gpu(case, measurements=None, **kw):
    from dca_b200.accumulators import TpAccumulator
    acc = TpAccumulator(case.G0, case.tp_params(**kw))
    acc.resetAccumulation(0)
    for m in (measurements if measurements is not None else case.measurements):
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    acc.finalize()
    return acc


def run_oracle(oracle_lib, case, measurements=None, **kw):
    acc = oracle_lib.OracleTp(case.G0, case.tp_params(**kw))
    for m in (measurements if measurements is not None else case.measurements):
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    return acc


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fp64_matches_reference_golden(name):
    case, ref = golden(name)
    acc = run_gpu(case)
    for got, want in zip(acc.get_G4(), ref.g4):
        assert rel_err(got, want) <= FP64_TOL


@pytest.mark.parametrize("name", ["sq2_all", "mb3_all", "sq4_q5"])
def test_fp64_g_matches_oracle(oracle_lib, name):
    case, _ = golden(name)
    m = case.measurements[-1]
    acc = run_gpu(case, [m])
    ora = run_oracle(oracle_lib, case, [m])
    for spin in range(2):
        assert rel_err(acc.get_G(spin), ora.get_G(spin)) <= FP64_TOL


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_mixed_matches_reference_golden(name):
    case, ref = golden(name)
    acc = run_gpu(case, precision=1, max_batch=2)
    for got, want in zip(acc.get_G4(), ref.g4):
        assert rel_err(got, want) <= MIXED_TOL


@pytest.mark.parametrize("wname", ["c2", "c4"])
def test_fp64_full_size_matches_oracle(oracle_lib, wname):
    case = case_from_workload(W.WORKLOADS[wname], 1)
    acc = run_gpu(case)
    ora = run_oracle(oracle_lib, case)
    for got, want in zip(acc.get_G4(), ora.get_G4()):
        assert rel_err(got, want) <= FP64_TOL


def test_mixed_c3_batched_matches_oracle(oracle_lib):
    """Uneven orders in one batch, a partial last batch flushed by finalize."""
    w = W.WORKLOADS["c3"]
    case = case_from_workload(w, 5)
    acc = run_gpu(case, precision=1, max_batch=4)
    ora = run_oracle(oracle_lib, case)
    errs = [rel_err(g, o) for g, o in zip(acc.get_G4(), ora.get_G4())]
    print("mixed c3 relative errors per channel:", errs)
    assert max(errs) <= MIXED_TOL


def test_mixed_equals_fp64_gpu_at_full_batch():
    """Full c3 batch (64 measurements): mixed vs the FP64 GPU path (itself pinned above)."""
    w = W.WORKLOADS["c3"]
    case = case_from_workload(w, 64)
    mixed = run_gpu(case, precision=1, max_batch=64)
    fp64 = run_gpu(case, precision=0, max_batch=1)
    errs = [rel_err(a, b) for a, b in zip(mixed.get_G4(), fp64.get_G4())]
    print("mixed vs FP64, 64 measurements:", errs)
    assert max(errs) <= MIXED_TOL


def _run_timed(case, simt_only, monkeypatch, **kw):
    """Mixed run with stage timing on; DCAACC_TP_SIMT_ONLY selects the update path at creation."""
    from dca_b200.accumulators import TpAccumulator
    monkeypatch.setenv("DCAACC_TP_SIMT_ONLY", "1" if simt_only else "0")
    acc = TpAccumulator(case.G0, case.tp_params(precision=1, **kw))
    acc.enable_timing(True)
    acc.resetAccumulation(0)
    for m in case.measurements:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    acc.finalize()
    return acc


def _small_all_transfers(cluster_kind, freq_transfer):
    """c1-like single-band workloads with every momentum transfer and both PH channels: they take
    the outer-product direct-term kernel at Nc = 4 and 8."""
    import dataclasses
    return dataclasses.replace(W.WORKLOADS["c1"], name=f"all-q {cluster_kind[0]}", cluster_kind=cluster_kind,
                               all_transfers=True, freq_transfer=freq_transfer, channels=(2, 3))


EXTRA_WORKLOADS = {"sq2_allq": _small_all_transfers(("square", 2), 1),
                   "betts8_allq": _small_all_transfers(("betts8",), 0)}


@pytest.mark.parametrize("wname,n_meas,max_batch", [("c1", 6, 4), ("sq2_allq", 5, 4), ("betts8_allq", 5, 4),
                                                     ("c3", 9, 4), ("c3", 70, 72)])
def test_tensor_core_disconnected_terms_match_oracle(oracle_lib, monkeypatch, wname, n_meas, max_batch):
    """The one-band PH update with its disconnected terms on tcgen05 (split FP16, FP32 accumulate)
    against the all-SIMT update and an FP64 reference: the oracle for c1, the FP64 GPU path (pinned
    to the oracle above) for c3.  (c3, 70, 72) takes three K chunks in the GEMM and, in the
    tensor-core direct term (Nc = 16), eight full 8-measurement steps and a partial one, with the
    G4 flush of each tile spread over the next tile's steps; (c3, 9, 4) runs single partial steps
    (batches of 4 and 1), whose flush chunks outnumber the steps.  c1 (M = 64) pads the rows to
    one 128-row tile."""
    case = case_from_workload(EXTRA_WORKLOADS.get(wname) or W.WORKLOADS[wname], n_meas)
    tc = _run_timed(case, False, monkeypatch, max_batch=max_batch)
    simt = _run_timed(case, True, monkeypatch, max_batch=max_batch)
    batches = -(-n_meas // max_batch)
    assert tc.stage_times()["update_g4"][1] == 3 * batches      # planes + GEMM + direct term
    assert simt.stage_times()["update_g4"][1] == batches
    exact = run_oracle(oracle_lib, case) if wname != "c3" else run_gpu(case, precision=0, max_batch=1)
    for got, ref, want in zip(tc.get_G4(), simt.get_G4(), exact.get_G4()):
        print(wname, n_meas, "tensor-core / SIMT relative errors:", rel_err(got, want), rel_err(ref, want))
        assert rel_err(got, want) <= MIXED_TOL
        assert rel_err(ref, want) <= MIXED_TOL


@pytest.mark.parametrize("n_meas,max_batch", [(9, 8), (3, 4)])
def test_half_g_matches_full_g(monkeypatch, n_meas, max_batch):
    """c3 (Nc = 16, all transfers, one band, G0(-k, -w) = conj G0(k, w)) computes only the upper
    frequency half of G and reads the rest as its conjugated mirror, and accumulates only the G4
    tiles with w1 >= Nw/2 (the rest is their mirror, filled at finalize); DCAACC_TP_FULL_G=1
    computes all of G and G4.  Both against the FP64 path, and against each other (with exactly
    conjugate-symmetric inputs the two agree to the last bit)."""
    case = case_from_workload(W.WORKLOADS["c3"], n_meas)
    monkeypatch.setenv("DCAACC_TP_FULL_G", "0")
    half = _run_timed(case, False, monkeypatch, max_batch=max_batch)
    monkeypatch.setenv("DCAACC_TP_FULL_G", "1")
    full = _run_timed(case, False, monkeypatch, max_batch=max_batch)
    exact = run_gpu(case, precision=0, max_batch=1)
    assert half.mirror_mode() == 3 and full.mirror_mode() == 0 and exact.mirror_mode() == 0
    for h, f, want in zip(half.get_G4(), full.get_G4(), exact.get_G4()):
        print("half / full G relative errors:", rel_err(h, want), rel_err(f, want))
        assert rel_err(h, want) <= MIXED_TOL
        assert rel_err(f, want) <= MIXED_TOL
        assert rel_err(h, f) <= MIXED_TOL


def _small(wname, **kw):
    import dataclasses
    return dataclasses.replace(W.WORKLOADS[wname], **kw)


def test_graph_replay_matches_eager(monkeypatch):
    """The mixed path replays each batch shape's kernel sequence from a CUDA graph (captured on the
    shape's second batch): the G4 equals, bit for bit, that of eager launches, and of a handle
    created with DCAACC_TP_GRAPHS=0."""
    from dca_b200.accumulators import TpAccumulator
    w = _small("c3", n_range=(40, 120))
    case = case_from_workload(w, 24)  # 6 batches of 4, three per device input set
    monkeypatch.setenv("DCAACC_TUNE", "0")  # built-in launch shapes: graphs from the second batch on

    def run(graphs, env="1"):
        monkeypatch.setenv("DCAACC_TP_GRAPHS", env)
        acc = TpAccumulator(case.G0, case.tp_params(precision=1, max_batch=4))
        if not graphs:
            acc.set_graphs(False)
        acc.resetAccumulation(0)
        for m in case.measurements:
            acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        acc.finalize()
        return acc

    graph, eager, off = run(True), run(False), run(True, env="0")
    assert graph.graph_stats() == (2, 4)
    assert eager.graph_stats() == (0, 0) and off.graph_stats() == (0, 0)
    assert graph.kernel_launches() == eager.kernel_launches()
    for g, e, o in zip(graph.get_G4(), eager.get_G4(), off.get_G4()):
        assert np.array_equal(g, e) and np.array_equal(g, o)


@pytest.mark.parametrize("wname,precision,max_batch,n_meas", [("c3", 0, 1, 16), ("c3", 1, 4, 64),
                                                              ("c4", 1, 2, 30)])
def test_tuned_launch_shapes_match_builtin(monkeypatch, wname, precision, max_batch, n_meas):
    """The launch-shape tuner times each candidate shape (FP64: row-transform tiles, column-transform
    widths, transfers per G4 CTA; mixed: operand-builder blocks, and for three bands the staged G4
    kernel's entries per thread) on the first batches of a problem shape and keeps the fastest.
    Every candidate gives the same bits, so G4 equals that of the built-in shapes (DCAACC_TUNE=0),
    and every tuned launch has decided."""
    from dca_b200.accumulators import TpAccumulator
    if wname == "c3":
        w = _small("c3", n_range=(40, 60))
    else:
        w = _small("c4", nw_half=4, n_sp=64, n_range=(20, 40), freq_transfer=1)
    case = case_from_workload(w, n_meas)

    def run(tune):
        monkeypatch.setenv("DCAACC_TUNE", tune)
        acc = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=max_batch))
        acc.resetAccumulation(0)
        for m in case.measurements:
            acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        acc.finalize()
        return acc

    tuned, builtin = run("1"), run("0")
    report = [line for line in tuned.tuning_report().splitlines() if line]
    print("\n".join(report))
    assert report and tuned.tuning_settled()
    for line in report:  # "key n=<candidates> choice=<c> ms=<median per candidate>"
        fields = dict(f.split("=", 1) for f in line.split()[1:])
        ms = [float(x) for x in fields["ms"].split(",")]
        assert len(ms) == int(fields["n"]) and min(ms) > 0
        assert ms[int(fields["choice"])] == min(ms)
    assert builtin.tuning_report() == "" and builtin.tuning_settled()
    for a, b in zip(tuned.get_G4(), builtin.get_G4()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [0, 1])
def test_shared_g4_matches_single_handle(precision):
    """Two handles accumulating into one shared G4 (atomic updates, two streams), reset once per
    DCA loop, give the G4 of one handle fed every measurement; a second reset for the same loop
    keeps the sums, a reset for the next loop clears them; sumTo between them moves only signs."""
    from dca_b200.accumulators import TpAccumulator
    case = case_from_workload(_small("c3", n_range=(30, 60)), 6)
    kw = dict(precision=precision, max_batch=2)
    single = run_gpu(case, **kw)
    a = TpAccumulator(case.G0, case.tp_params(**kw))
    b = TpAccumulator(case.G0, case.tp_params(**kw))
    b.share_G4_with(a)
    a.resetAccumulation(7)
    b.resetAccumulation(7)
    for i, m in enumerate(case.measurements):
        (a if i % 2 == 0 else b).accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    a.flush()
    b.flush()
    b.sumTo(a)  # shared G4: only the signs move
    assert a.sign_sum() == (float(sum(m.sign for m in case.measurements)), 6) and b.sign_sum() == (0.0, 0)
    a.finalize()
    # FP64: atomics change only the summation order.  Mixed: the two handles form other batches
    # than the single one, so the FP32 partial sums round differently (about 3e-8 measured).
    tol = 1e-12 if precision == 0 else 1e-7
    for got, want in zip(a.get_G4(), single.get_G4()):
        assert rel_err(got, want) <= tol
    window = a.peek_G4(0, 0, 4096)
    assert np.any(window)
    b.resetAccumulation(7)  # same loop: the shared sums stay
    assert np.array_equal(a.peek_G4(0, 0, 4096), window)
    b.resetAccumulation(8)  # next loop: cleared for both
    assert not np.any(a.peek_G4(0, 0, 4096))


def test_peek_async_matches_peek():
    """peek_G4_async enqueues the read of the running G4 (after the queued measurements) into
    caller memory; after synchronizeCopy it equals the synchronous peek, also with the mirror
    window of the half-G4 path (c3-like)."""
    import torch
    from dca_b200.accumulators import TpAccumulator
    case = case_from_workload(_small("c3", n_range=(40, 80)), 6)
    acc = TpAccumulator(case.G0, case.tp_params(precision=1, max_batch=4))
    acc.resetAccumulation(0)
    outs = []
    for m in case.measurements:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        buf = torch.empty(300, dtype=torch.complex128, pin_memory=True).numpy()
        acc.peek_G4_async(1, 1000, buf)
        outs.append(buf)
    acc.synchronizeCopy()
    assert np.array_equal(outs[-1], acc.peek_G4(1, 1000, 300)) and np.any(outs[-1] != 0)


def test_sign_sum_and_normalized_g4(tmp_path):
    """The handle sums the measurement signs (sumTo moves them with G4); the normalised G4 is
    G4 / (sign sum * beta^2), as the solver divides it, and write_G4 stores it under the
    reference's dataset names in the reference's index order."""
    from dca_b200.accumulators import LogicError, TpAccumulator, write_G4
    case, _ = golden("c1_mag")
    ms = case.measurements
    a = TpAccumulator(case.G0, case.tp_params())
    b = TpAccumulator(case.G0, case.tp_params())
    a.resetAccumulation(0)
    b.resetAccumulation(0)
    for m in ms[:2]:
        a.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    for m in ms[2:]:
        b.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    a.sumTo(b)
    assert a.sign_sum() == (0.0, 0)
    assert b.sign_sum() == (float(sum(m.sign for m in ms)), len(ms))
    b.finalize()
    total = sum(m.sign for m in ms)
    for g, n in zip(b.get_G4(), b.get_G4_normalized()):
        np.testing.assert_allclose(n, g / (total * case.beta ** 2), rtol=1e-15, atol=0)
    path = tmp_path / "g4.npz"
    write_G4(str(path), b)
    with np.load(path) as f:
        assert list(f.keys()) == ["G4_PARTICLE_HOLE_MAGNETIC"]
        stored = f["G4_PARTICLE_HOLE_MAGNETIC"]
    assert stored.shape == b.parameters.g4_shape()
    assert np.array_equal(stored.reshape(-1, order="F"), b.get_G4_normalized()[0])
    a.finalize()
    with pytest.raises(LogicError):  # nothing accumulated: the sign sum is zero
        a.get_G4_normalized()


def test_large_cluster_fp64_matches_oracle(oracle_lib):
    """6x6 single band (Nc = 36): one momentum transfer's k1 x k2 block does not fit the tuned
    single-band kernel's thread block, so the FP64 update takes the general kernel."""
    w = _small("c5", nw_half=2, n_sp=64, n_range=(20, 40))
    case = case_from_workload(w, 2)
    acc = run_gpu(case)
    ora = run_oracle(oracle_lib, case)
    for got, want in zip(acc.get_G4(), ora.get_G4()):
        assert rel_err(got, want) <= FP64_TOL


@pytest.mark.parametrize("channels", [(2,), (2, 3)])
def test_large_cluster_mixed_split_direct_term(oracle_lib, channels):
    """6x6 single band, all 36 momentum transfers, batches of 3: the mixed path takes the
    disconnected terms on the tensor cores and the direct term on the split outer-product kernel
    (three CTAs per frequency tile, 12 rows k1 each).  Against the oracle (FP64), and the G4
    stage must be those three launches per batch."""
    w = _small("c5", nw_half=2, n_sp=64, n_range=(20, 40), channels=channels)
    case = case_from_workload(w, 7)
    from dca_b200.accumulators import TpAccumulator
    acc = TpAccumulator(case.G0, case.tp_params(precision=1, max_batch=3))
    acc.enable_timing(True)
    acc.resetAccumulation(0)
    for m in case.measurements:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    acc.finalize()
    assert acc.stage_times()["update_g4"][1] == 3 * 3  # 3 batches (3 + 3 + 1 measurements)
    ora = run_oracle(oracle_lib, case)
    for got, want in zip(acc.get_G4(), ora.get_G4()):
        print("split direct term, relative error:", rel_err(got, want))
        assert rel_err(got, want) <= MIXED_TOL


@pytest.mark.parametrize("channels", [(4,), (2, 3)])
@pytest.mark.parametrize("precision", [0, 1])
def test_multiband_batched_matches_oracle(oracle_lib, channels, precision):
    """Three bands on the Betts 8 cluster, batches of 3: the staged multi-band update (the G blocks
    of each measurement in shared memory), particle-particle and the two PH channels, in FP64 and
    in the mixed path."""
    w = _small("c4", nw_half=4, n_sp=64, n_range=(20, 40), channels=channels, freq_transfer=1)
    case = case_from_workload(w, 4)
    acc = run_gpu(case, precision=precision, max_batch=3)
    ora = run_oracle(oracle_lib, case)
    tol = FP64_TOL if precision == 0 else MIXED_TOL
    for got, want in zip(acc.get_G4(), ora.get_G4()):
        print("multiband", channels, precision, rel_err(got, want))
        assert rel_err(got, want) <= tol


@pytest.mark.parametrize("all_transfers", [True, False])
def test_pp_multiband_kernel_matches_generic_and_oracle(oracle_lib, monkeypatch, all_transfers):
    """Three bands, particle-particle up-down alone, mixed path: the PP kernel (a thread keeps the
    27 band entries of one (k1, k2, q, b4) over the batch) against the generic staged kernel
    (DCAACC_TP_PP_GENERIC=1) and the oracle.  With all 8 x 2 transfers its items fill three passes
    of the CTA; with one momentum transfer they fill part of one pass."""
    w = _small("c4", nw_half=4, n_sp=64, n_range=(20, 60), channels=(4,), freq_transfer=1,
               all_transfers=all_transfers, k_transfer=3)
    case = case_from_workload(w, 7)
    monkeypatch.setenv("DCAACC_TP_PP_GENERIC", "0")
    pp = run_gpu(case, precision=1, max_batch=4)
    monkeypatch.setenv("DCAACC_TP_PP_GENERIC", "1")
    generic = run_gpu(case, precision=1, max_batch=4)
    ora = run_oracle(oracle_lib, case)
    for a, g, want in zip(pp.get_G4(), generic.get_G4(), ora.get_G4()):
        print("PP kernel / generic staged kernel, relative errors:", rel_err(a, want), rel_err(g, want))
        assert rel_err(a, want) <= MIXED_TOL
        assert rel_err(g, want) <= MIXED_TOL
        assert rel_err(a, g) <= MIXED_TOL


@pytest.mark.parametrize("precision", [0, 1])
def test_sum_to_equals_single_accumulator(precision):
    case, _ = golden("sq2_all")
    from dca_b200.accumulators import TpAccumulator
    a = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=2))
    b = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=2))
    for acc in (a, b):
        acc.resetAccumulation(0)
    ms = case.measurements
    for m in ms[:1]:
        a.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    for m in ms[1:]:
        b.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    a.sumTo(b)
    b.finalize()
    a.finalize()
    whole = run_gpu(case, precision=precision, max_batch=2)
    # FP32 batch partial sums depend on how measurements are grouped into batches.
    tol = 1e-13 if precision == 0 else MIXED_TOL
    for got, want, zero in zip(b.get_G4(), whole.get_G4(), a.get_G4()):
        assert rel_err(got, want) <= tol
        assert np.all(zero == 0)


@pytest.mark.parametrize("precision", [0, 1])
def test_accumulate_batch_equals_single_calls(precision):
    """dcaacc_tp_accumulate_batch stages the same measurements in the same order: identical G4."""
    from dca_b200.accumulators import TpAccumulator
    case = case_from_workload(W.WORKLOADS["c1"], 7)
    single = run_gpu(case, precision=precision, max_batch=3)
    acc = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=3))
    acc.resetAccumulation(0)
    ms = case.measurements
    acc.accumulate_batch([[s.M for s in m.sectors] for m in ms], [list(m.sectors) for m in ms],
                         [m.sign for m in ms])
    acc.finalize()
    for a, b in zip(acc.get_G4(), single.get_G4()):
        assert np.array_equal(a, b)


def test_device_resident_m_matches_host_m():
    import torch
    case, _ = golden("mb3_all")
    from dca_b200.accumulators import TpAccumulator
    host = run_gpu(case)
    acc = TpAccumulator(case.G0, case.tp_params())
    acc.resetAccumulation(0)
    for m in case.measurements:
        Md = [torch.from_numpy(np.ascontiguousarray(s.M.T)).cuda().t() for s in m.sectors]
        acc.accumulate(Md, list(m.sectors), m.sign)
        acc.synchronizeCopy()
    acc.finalize()
    for got, want in zip(acc.get_G4(), host.get_G4()):
        assert rel_err(got, want) <= 1e-14


def test_lifecycle_and_errors():
    from dca_b200.accumulators import LogicError, TpAccumulator
    case, _ = golden("c1_mag")
    acc = TpAccumulator(case.G0, case.tp_params())
    m = case.measurements[0]
    args = ([s.M for s in m.sectors], list(m.sectors), m.sign)
    with pytest.raises(LogicError):          # not ready to measure
        acc.accumulate(*args)
    acc.resetAccumulation(0)
    acc.accumulate(*args)
    with pytest.raises(LogicError):          # bad sign
        acc.accumulate(args[0], args[1], 3)
    bad = W.Sector(m.sectors[0].tau, m.sectors[0].left_band, m.sectors[0].right_band + 1,
                   m.sectors[0].left_site, m.sectors[0].right_site, m.sectors[0].M)
    with pytest.raises(LogicError):          # band out of range
        acc.accumulate([bad.M, m.sectors[1].M], [bad, m.sectors[1]], 1)
    empty = W.Sector(np.zeros(0), *(np.zeros(0, np.int32) for _ in range(4)), np.zeros((0, 0)))
    assert acc.accumulate([empty.M, empty.M], [empty, empty], 1) == 0.0
    acc.finalize()
    one = acc.get_G4()[0].copy()
    with pytest.raises(LogicError):          # finalized: needs resetAccumulation
        acc.accumulate(*args)
    acc.resetAccumulation(1)
    acc.accumulate(*args)
    acc.finalize()
    assert rel_err(acc.get_G4()[0], one) <= 1e-15
    assert acc.kernel_launches() > 0 and acc.deviceFingerprint() > 0


def test_sum_to_across_mirror_modes(monkeypatch):
    """sumTo between handles whose mirror modes differ: a half-G4 mixed handle (c3-like) adds into
    a full-G4 mixed handle (DCAACC_TP_FULL_G=1) and into an FP64 handle (its lower half is filled
    from the mirror first), and a full handle adds into a half one; each sum equals one FP64 handle
    fed every measurement.  Handles of different transfer lists or channels are refused."""
    import dataclasses

    from dca_b200.accumulators import LogicError, TpAccumulator
    case = case_from_workload(_small("c3", n_range=(40, 80)), 6)
    ms = case.measurements

    def make(precision, full=False, **kw):
        monkeypatch.setenv("DCAACC_TP_FULL_G", "1" if full else "0")
        acc = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=4, **kw))
        acc.resetAccumulation(0)
        return acc

    def feed(acc, sub):
        for m in sub:
            acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        return acc

    whole = feed(make(0), ms)
    whole.finalize()
    pairs = [(feed(make(1), ms[:3]), feed(make(1, full=True), ms[3:])),   # half -> full
             (feed(make(1), ms[:3]), feed(make(0), ms[3:])),              # half -> FP64
             (feed(make(1, full=True), ms[:3]), feed(make(1), ms[3:]))]   # full -> half
    assert pairs[0][0].mirror_mode() == 3 and pairs[0][1].mirror_mode() == 0
    for src, dst in pairs:
        src.sumTo(dst)
        dst.finalize()
        for got, want in zip(dst.get_G4(), whole.get_G4()):
            print("sumTo across mirror modes:", src.mirror_mode(), "->", dst.mirror_mode(), rel_err(got, want))
            assert rel_err(got, want) <= MIXED_TOL
    other_q = make(1, k_ex=[0])
    with pytest.raises(LogicError):
        make(1).sumTo(other_q)
    with pytest.raises(LogicError):
        make(1).share_G4_with(make(1, channels=[2]))
    with pytest.raises(LogicError):  # different mirror modes cannot share one G4
        make(1).share_G4_with(make(1, full=True))


def test_share_g4_keeps_what_was_accumulated_before():
    """A handle that has accumulated on its own and then starts sharing another handle's G4 adds
    what it has into the shared one: nothing is dropped, and the sum equals one handle fed every
    measurement."""
    from dca_b200.accumulators import TpAccumulator
    case = case_from_workload(_small("c3", n_range=(30, 60)), 6)
    ms = case.measurements
    single = run_gpu(case, precision=0, max_batch=1)
    a = TpAccumulator(case.G0, case.tp_params(precision=0, max_batch=1))
    b = TpAccumulator(case.G0, case.tp_params(precision=0, max_batch=1))
    a.resetAccumulation(3)
    b.resetAccumulation(3)
    for m in ms[:2]:
        b.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    a.accumulate([s.M for s in ms[2].sectors], list(ms[2].sectors), ms[2].sign)
    b.share_G4_with(a)
    for i, m in enumerate(ms[3:]):
        (a if i % 2 else b).accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    b.sumTo(a)
    a.finalize()
    assert a.sign_sum() == (float(sum(m.sign for m in ms)), 6)
    for got, want in zip(a.get_G4(), single.get_G4()):
        assert rel_err(got, want) <= 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_non_density_vertices_match_oracle(oracle_lib, precision):
    """Vertices whose left and right band / site differ (non-density-density interactions): the rows
    of M are ordered by the right orbital and the columns by the left one
    (cached_ndft_base.hpp:97-103), both sorted on the device.  Three bands on the Betts 8 cluster,
    all four channels, against the oracle."""
    w = _small("c4", nw_half=4, n_sp=64, n_range=(20, 40), freq_transfer=1, channels=(1, 2, 3, 4))
    case = case_from_workload(w, 3)
    rng = np.random.default_rng(5)
    for m in case.measurements:
        for s in m.sectors:
            s.left_band = rng.integers(0, w.nb, s.n).astype(np.int32)
            s.left_site = rng.integers(0, case.nc, s.n).astype(np.int32)
    acc = run_gpu(case, precision=precision, max_batch=2, non_density=True)
    ora = run_oracle(oracle_lib, case, non_density=True)
    tol = FP64_TOL if precision == 0 else MIXED_TOL
    for got, want in zip(acc.get_G4(), ora.get_G4()):
        print("non-density", precision, rel_err(got, want))
        assert rel_err(got, want) <= tol


@pytest.mark.parametrize("precision", [0, 1])
def test_float_m_and_sign_types(precision):
    """accumulate for the reference's other SpScalar / SignType instantiations: float M (host and
    device) gives the G4 of the same M widened to double, a complex sign with zero imaginary part is
    the real sign, and complex M or a complex sign are refused (DCAACC_UNSUPPORTED)."""
    import torch
    from dca_b200.accumulators import LogicError, TpAccumulator
    case = case_from_workload(_small("c3", n_range=(40, 80)), 4)
    ms = case.measurements
    widened = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=2))
    typed = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=2))
    for acc in (widened, typed):
        acc.resetAccumulation(0)
    alive = []  # device M stays valid until the queued batch has run (synchronizeCopy)
    for i, m in enumerate(ms):
        m32 = [np.asfortranarray(s.M.astype(np.float32)) for s in m.sectors]
        widened.accumulate([x.astype(np.float64) for x in m32], list(m.sectors), m.sign)
        if i % 2:  # device float M
            src = [torch.from_numpy(np.ascontiguousarray(x.T)).cuda().t() for x in m32]
        else:
            src = m32
        alive.append(src)
        typed.accumulate_typed(src, list(m.sectors), complex(m.sign, 0.0))
    for acc in (widened, typed):
        acc.finalize()
    for a, b in zip(typed.get_G4(), widened.get_G4()):
        assert rel_err(a, b) <= 1e-15
    # The batched form gives the same bits as one call per measurement.
    batched = TpAccumulator(case.G0, case.tp_params(precision=precision, max_batch=2))
    batched.resetAccumulation(0)
    batched.accumulate_batch_typed([[np.asfortranarray(s.M.astype(np.float32)) for s in m.sectors] for m in ms],
                                   [list(m.sectors) for m in ms], [m.sign for m in ms])
    batched.finalize()
    for a, b in zip(batched.get_G4(), typed.get_G4()):
        assert np.array_equal(a, b)
    typed.resetAccumulation(1)
    m = ms[0]
    with pytest.raises(LogicError, match="UNSUPPORTED"):
        typed.accumulate_typed([s.M.astype(np.complex128) for s in m.sectors], list(m.sectors), 1)
    with pytest.raises(LogicError, match="UNSUPPORTED"):
        typed.accumulate_typed([s.M for s in m.sectors], list(m.sectors), 1j)


def test_large_cluster_half_g_matches_full_g(monkeypatch):
    """6x6 single band (t' = -0.15), Nw = 64, all 36 momentum transfers: the mixed path computes
    the upper frequency half of G and accumulates the G4 tiles with w1 >= Nw/2 only (the split
    direct term reads lower-half blocks as conjugated mirrors with k -> -k); against
    DCAACC_TP_FULL_G=1 and the FP64 GPU path."""
    w = _small("c5", nw_half=32, n_sp=128, n_range=(30, 60))
    case = case_from_workload(w, 5)
    monkeypatch.setenv("DCAACC_TP_FULL_G", "0")
    half = _run_timed(case, False, monkeypatch, max_batch=4)
    monkeypatch.setenv("DCAACC_TP_FULL_G", "1")
    full = _run_timed(case, False, monkeypatch, max_batch=4)
    exact = run_gpu(case, precision=0, max_batch=1)
    assert half.mirror_mode() == 3 and full.mirror_mode() == 0
    for h, f, want in zip(half.get_G4(), full.get_G4(), exact.get_G4()):
        print("6x6 half / full G relative errors:", rel_err(h, want), rel_err(f, want))
        assert rel_err(h, want) <= MIXED_TOL
        assert rel_err(f, want) <= MIXED_TOL


@pytest.mark.parametrize("full_g,fft,mode", [("0", "1", "1"), ("1", "1", "1"), ("0", "0", "1"), ("0", "1", "2"),
                                             ("1", "1", "2")])
def test_factored_column_step_matches_dense(monkeypatch, full_g, fft, mode):
    """One band, Nc = 16: the column step factored by orbital (the column NDFT per orbital, then the
    cluster transform as a 4 x 4 FFT, or with DCAACC_TP_COL_FFT=0 as a 16 x 16 matrix), with
    DCAACC_TP_FACTORED_COL=1 on mma.sync / the CUDA cores and with =2 on tcgen05 with the per-site
    sums in tensor memory, against the dense tensor-core GEMM and the FP64 path, with half G
    (mirror symmetry) and with all of G; an empty spin sector included, orders up to 300 (ten
    32-vertex chunks, sites straddling chunk and 16-vertex step boundaries)."""
    w = _small("c3", n_range=(40, 300))
    case = case_from_workload(w, 9)
    case.measurements[3] = W.make_measurement(w, 3, n_override=(0, 57))
    monkeypatch.setenv("DCAACC_TP_FULL_G", full_g)
    monkeypatch.setenv("DCAACC_TP_COL_FFT", fft)
    monkeypatch.setenv("DCAACC_TP_FACTORED_COL", mode)
    fact = _run_timed(case, False, monkeypatch, max_batch=4)
    monkeypatch.setenv("DCAACC_TP_FACTORED_COL", "0")
    dense = _run_timed(case, False, monkeypatch, max_batch=4)
    exact = run_gpu(case, precision=0, max_batch=1)
    assert fact.mirror_mode() == dense.mirror_mode() == (0 if full_g == "1" else 3)
    for f, d, want in zip(fact.get_G4(), dense.get_G4(), exact.get_G4()):
        print("factored / dense column step, relative errors:", rel_err(f, want), rel_err(d, want))
        assert rel_err(f, want) <= MIXED_TOL
        assert rel_err(d, want) <= MIXED_TOL


@pytest.mark.parametrize("full_g", ["0", "1"])
def test_factored_column_step_6x6_matches_dense(monkeypatch, full_g):
    """One band, 6 x 6 cluster (Nc = 36): the column step factored by orbital on the CUDA cores with
    the 6 x 6 FFT (DCAACC_TP_FACTORED_COL=1) against the dense tensor-core GEMM (the default) and
    the FP64 path, with half G (mirror symmetry) and with all of G.  An empty spin sector, and a
    measurement whose 150 vertices sit on three sites (sites of more than one 32-vertex block)."""
    import dataclasses
    w = _small("c5", nw_half=32, n_sp=128, n_range=(30, 150))
    case = case_from_workload(w, 6)
    case.measurements[2] = W.make_measurement(w, 2, n_override=(0, 57))
    m = W.make_measurement(w, 4, n_override=(150, 41))
    rng = np.random.default_rng(11)
    sites = rng.integers(0, 3, 150).astype(np.int32)
    s0 = dataclasses.replace(m.sectors[0], left_site=sites, right_site=sites.copy())
    case.measurements[4] = W.Measurement(m.sign, (s0, m.sectors[1]))
    monkeypatch.setenv("DCAACC_TP_FULL_G", full_g)
    monkeypatch.setenv("DCAACC_TP_FACTORED_COL", "1")
    fact = _run_timed(case, False, monkeypatch, max_batch=4)
    monkeypatch.delenv("DCAACC_TP_FACTORED_COL")
    dense = _run_timed(case, False, monkeypatch, max_batch=4)
    exact = run_gpu(case, precision=0, max_batch=1)
    assert fact.mirror_mode() == dense.mirror_mode() == (0 if full_g == "1" else 3)
    for f, d, want in zip(fact.get_G4(), dense.get_G4(), exact.get_G4()):
        print("6x6 factored / dense column step, relative errors:", rel_err(f, want), rel_err(d, want))
        assert not np.array_equal(f, d)  # two different column steps ran
        assert rel_err(f, want) <= MIXED_TOL
        assert rel_err(d, want) <= MIXED_TOL
