"""The CPU oracle against the reference's own outputs and against known answers (no GPU)."""

import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN_CASES
from helpers import GOLDEN, case_from_workload, golden, rel_err
from dca_b200 import workloads as W


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_golden(oracle_lib, name):
    """Restatement vs TpAccumulator<CPU> / SpAccumulator<CPU> run from the reference's sources."""
    from oracle import casefile as CF
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        oracle_lib.run_case(os.path.join(GOLDEN, name + ".case"), out)
        mine = CF.read_result(out)
    _, ref = golden(name)
    assert len(mine.g4) == len(ref.g4)
    for a, b in zip(mine.g4, ref.g4):
        assert rel_err(a, b) <= 1e-13
    assert rel_err(mine.mrw, ref.mrw) <= 1e-13
    if ref.mrw_sqr is not None:
        assert rel_err(mine.mrw_sqr, ref.mrw_sqr) <= 1e-13


def _direct_g(case, meas, spin):
    """G of one spin sector from the definition (the direct triple-sum pattern of the reference's
    single_sector_accumulation_test.hpp:226-254), extended to the cluster transform and G0."""
    nb, nc = case.nb, case.nc
    ext = max(abs(w) for w in case.w_ex())
    nwe = 2 * case.nw_half + 2 * ext
    w = W.matsubara(case.beta, nwe // 2)
    sec = meas.sectors[spin]
    # Row vertices use the right band / site, columns the (equal) left ones.
    r_pos = case.r_vecs[sec.right_site] + case.a_vecs[sec.right_band]
    phase = np.exp(1j * (np.outer(w, sec.tau)[:, None, :] +
                         (case.k_vecs @ r_pos.T)[None, :, :]))  # (w, k, i)
    A = np.zeros((nwe, nc, nb, sec.n), complex)
    for b in range(nb):
        A[:, :, b, :] = phase * (sec.right_band == b)[None, None, :]
    A = A.reshape(nwe * nc * nb, sec.n)  # rows (w, k, b) with b fastest
    Gt = A @ sec.M @ A.conj().T / nc
    G0 = case.G0.reshape(2 * case.n_sp, nc, 2, nb, 2, nb)[:, :, spin, :, spin, :]  # (w, k, b2, b1)
    off = case.n_sp - nwe // 2
    G0b = np.transpose(G0[off:off + nwe], (0, 1, 3, 2))  # (w, k, b1, b2)
    D = nwe * nc * nb
    Gt = Gt.reshape(nwe, nc, nb, nwe, nc, nb)
    G = -np.einsum("wkac,wkcxlf,xlfb->wkaxlb", G0b, Gt, G0b)
    for iw in range(nwe):
        for k in range(nc):
            G[iw, k, :, iw, k, :] += case.beta * G0b[iw, k]
    # -> (b1, b2, k1, k2, w1, w2) flattened with b1 fastest.
    return np.transpose(G, (3, 0, 4, 1, 5, 2)).reshape(-1)


@pytest.mark.parametrize("name", ["sq2_all", "mb3_all"])
def test_oracle_g_matches_direct_definition(oracle_lib, name):
    case, _ = golden(name)
    acc = oracle_lib.OracleTp(case.G0, case.tp_params())
    m = case.measurements[0]
    acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    for spin in range(2):
        assert rel_err(acc.get_G(spin), _direct_g(case, m, spin)) <= 1e-12


def test_oracle_ph_charge_minus_magnetic_identity(oracle_lib):
    """charge - magnetic = s/2 [(sum_s G_s)(sum_s G_s) - (G_0 - G_1)(G_0 - G_1)] on the
    disconnected legs: the direct terms cancel (tp_accumulator_cpu.hpp:491-575)."""
    case, _ = golden("sq2_all")
    p = case.tp_params(channels=[W.PH_MAGNETIC, W.PH_CHARGE])
    acc = oracle_lib.OracleTp(case.G0, p)
    m = case.measurements[1]
    acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    mag, charge = acc.get_G4()
    nc, nw = case.nc, 2 * case.nw_half
    ext = max(p.w_ex)
    nwe = nw + 2 * ext
    G = [acc.get_G(s).reshape(nwe, nwe, nc, nc) for s in range(2)]  # [w2, w1, k2, k1] (nb = 1)
    kadd = case.k_add
    expect = np.zeros((len(p.w_ex), len(p.k_ex), nw, nc, nw, nc), complex)
    for iwq, wex in enumerate(p.w_ex):
        for iq, q in enumerate(p.k_ex):
            for w2 in range(nw):
                for k2 in range(nc):
                    for w1 in range(nw):
                        for k1 in range(nc):
                            a = [G[s][w1 + ext + wex, w1 + ext, kadd[k1, q], k1] for s in range(2)]
                            b = [G[s][w2 + ext, w2 + ext + wex, k2, kadd[k2, q]] for s in range(2)]
                            expect[iwq, iq, w2, k2, w1, k1] = 0.5 * m.sign * (
                                (a[0] + a[1]) * (b[0] + b[1]) - (a[0] - a[1]) * (b[0] - b[1]))
    assert rel_err(charge - mag, expect.reshape(-1)) <= 1e-12


def test_oracle_sp_sum_linearity(oracle_lib):
    """Accumulating two measurements equals the sum of accumulating each (sp_accumulator_gpu_test)."""
    case, _ = golden("c1_mag")
    p = case.sp_params()
    parts = []
    for m in case.measurements[:2]:
        a = oracle_lib.OracleSp(p)
        a.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
        a.finalize()
        parts.append(a.get())
    both = oracle_lib.OracleSp(p)
    for m in case.measurements[:2]:
        both.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    both.finalize()
    assert rel_err(both.get(), parts[0] + parts[1]) <= 1e-13


@pytest.mark.parametrize("wname", ["c3", "c5"])
def test_oracle_g_mirror_symmetry(oracle_lib, wname):
    """The identity the mixed path's half-G mode rests on: with real M and G0(-k, -w) =
    conj G0(k, w) (real hopping, t' included), G(-k1 w1', -k2 w2') = conj G(k1 w1; k2 w2) with
    w' = NwExt - 1 - w, on one seeded measurement of the 4x4 and of the 6x6 configuration."""
    import dataclasses
    w = dataclasses.replace(W.WORKLOADS[wname], nw_half=4, n_sp=64, n_range=(20, 40))
    case = case_from_workload(w, 1)
    acc = oracle_lib.OracleTp(case.G0, case.tp_params())
    m = case.measurements[0]
    acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    cl = w.cluster()
    nc = cl.nc
    zero = next(i for i in range(nc) if all(cl.k_add[i, j] == j for j in range(nc)))
    neg = np.array([next(j for j in range(nc) if cl.k_add[k, j] == zero) for k in range(nc)])
    for spin in range(2):
        g = acc.get_G(spin)
        nwe = int(round(np.sqrt(g.size // (nc * nc))))
        g = g.reshape(nwe, nwe, nc, nc)  # [w2][w1][k2][k1] (k1 fastest, one band)
        mirrored = g[::-1, ::-1][:, :, neg][:, :, :, neg]
        assert np.max(np.abs(mirrored - g.conj())) <= 1e-12 * np.max(np.abs(g))


def test_oracle_g4_mirror_symmetry(oracle_lib):
    """The identity behind the half-G4 mode: G4(-k1 w1', -k2 w2', -q, wq = 0) = conj G4(k1 w1, k2 w2,
    q, 0) with w' = Nw - 1 - w, for both particle-hole channels over all momentum transfers of the
    4x4 configuration (three seeded measurements)."""
    import dataclasses
    w = dataclasses.replace(W.WORKLOADS["c3"], nw_half=4, n_sp=64, n_range=(20, 40))
    case = case_from_workload(w, 3)
    acc = oracle_lib.OracleTp(case.G0, case.tp_params())
    for m in case.measurements:
        acc.accumulate([s.M for s in m.sectors], list(m.sectors), m.sign)
    cl = w.cluster()
    nc, nw = cl.nc, 2 * w.nw_half
    assert list(w.exchange_momenta(nc)) == list(range(nc)) and w.exchange_frequencies() == [0]
    zero = next(i for i in range(nc) if all(cl.k_add[i, j] == j for j in range(nc)))
    neg = np.array([next(j for j in range(nc) if cl.k_add[k, j] == zero) for k in range(nc)])
    for g4 in acc.get_G4():
        g = g4.reshape(nc, nw, nc, nw, nc)  # [q][w2][k2][w1][k1] (k1 fastest, one band, one wq)
        mirrored = g[neg][:, ::-1][:, :, neg][:, :, :, ::-1][:, :, :, :, neg]
        assert np.max(np.abs(mirrored - g.conj())) <= 1e-12 * np.max(np.abs(g))
