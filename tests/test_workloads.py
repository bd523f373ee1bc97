"""Host-side logic: cluster tables, G0 layout, case-file round trip (no GPU)."""

import os
import tempfile

import numpy as np
import pytest

from dca_b200 import workloads as W
from helpers import read_case


@pytest.mark.parametrize("cl", [W.square_cluster(2), W.square_cluster(4), W.square_cluster(6),
                                W.betts8_cluster(), W.make_cluster((2, 0), (0, 1))])
def test_cluster_tables_are_group_tables(cl):
    nc = cl.nc
    for t in (cl.r_add, cl.k_add):
        zero = [i for i in range(nc) if all(t[i, j] == j for j in range(nc))]
        assert len(zero) == 1
        for i in range(nc):
            assert sorted(t[i]) == list(range(nc))  # Latin square
    for add, sub in ((cl.r_add, cl.r_sub), (cl.k_add, cl.k_sub)):
        for i in range(nc):
            for j in range(nc):
                assert add[i, sub[i, j]] == j  # x_i + (x_j - x_i) = x_j
    # e^{i k.r} is a character table: rows orthogonal.
    F = np.exp(1j * cl.k_vecs @ cl.r_vecs.T)
    assert np.allclose(F @ F.conj().T, nc * np.eye(nc))


def test_g0_is_inverse_of_bare_hamiltonian():
    w = W.WORKLOADS["c4"]
    cl = w.cluster()
    mu = w.chemical_potential()
    g0 = W.make_g0(w.model, cl, w.beta, mu, 8)
    wn = W.matsubara(w.beta, 8)
    for k in (0, 3):
        for iw in (0, 9):
            g = g0[iw, k, 0, :, 0, :].T
            h = w.model.h0(cl.k_vecs[k])
            assert np.allclose(g @ ((1j * wn[iw] + mu) * np.eye(3) - h), np.eye(3))
    assert np.all(g0[:, :, 0, :, 1, :] == 0)


def test_measurements_are_reproducible_and_well_formed():
    w = W.WORKLOADS["c3"]
    a = W.make_measurements(w, 3, start=5)
    b = W.make_measurement(w, 6)
    assert np.array_equal(a[1].sectors[0].M, b.sectors[0].M)
    for m in a:
        assert m.sign in (-1, 1)
        for s in m.sectors:
            assert w.n_range[0] <= s.n <= w.n_range[1]
            assert np.all((s.tau >= 0) & (s.tau < w.beta))
            assert s.M.flags.f_contiguous


def test_case_file_round_trip():
    from oracle import casefile as CF
    w = W.WORKLOADS["c1"]
    cl = w.cluster()
    g0 = W.make_g0(w.model, cl, w.beta, 0.0, w.n_sp)
    ms = W.make_measurements(w, 2)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c.case")
        CF.write_case(p, w, cl, g0, ms)
        c = read_case(p)
    assert np.array_equal(c.k_add, cl.k_add) and np.array_equal(c.r_sub, cl.r_sub)
    assert np.array_equal(c.G0, g0.reshape(-1))
    assert np.array_equal(c.measurements[1].sectors[1].M, ms[1].sectors[1].M)
