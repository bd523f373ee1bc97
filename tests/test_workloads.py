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


def test_workload_descriptions_name_what_they_are():
    c3 = W.WORKLOADS["c3"].describe()
    assert c3.startswith("c3: single-band Hubbard") and "4x4 cluster (Nc=16)" in c3
    assert "Nw=64" in c3 and "16 q x 1 wq" in c3 and "batch 64" in c3
    c4 = W.WORKLOADS["c4"].describe(with_batch=False)
    assert "three-band Emery" in c4 and "8 q x 4 wq" in c4 and "PARTICLE_PARTICLE_UP_DOWN" in c4
    assert "batch" not in c4


def test_write_g4_uses_reference_names_and_order(tmp_path):
    """write_G4 on a stand-in accumulator (no GPU): one dataset per channel named as DcaData names
    them, shaped (b1, b2, b3, b4, k1, w1, k2, w2, q, wq) in Fortran order."""
    from dca_b200.accumulators import TpParameters, write_G4
    w = W.WORKLOADS["c1"]
    cl = w.cluster()
    p = TpParameters.from_workload(w, cl, channels=(W.PH_MAGNETIC, W.PH_CHARGE))
    shape = p.g4_shape()
    size = int(np.prod(shape))
    rng = np.random.default_rng(3)
    g4 = [rng.standard_normal(size) + 1j * rng.standard_normal(size) for _ in range(2)]

    class StandIn:
        parameters = p

        def get_G4(self):
            return g4

        def get_G4_normalized(self):
            return [g / 2.0 for g in g4]

    path = tmp_path / "g4.npz"
    write_G4(str(path), StandIn())
    with np.load(path) as f:
        assert sorted(f.keys()) == ["G4_PARTICLE_HOLE_CHARGE", "G4_PARTICLE_HOLE_MAGNETIC"]
        mag = f["G4_PARTICLE_HOLE_MAGNETIC"]
    assert mag.shape == shape
    # first index fastest: element (b1..wq) = flat index b1 + nb (b2 + ...)
    assert mag[0, 0, 0, 0, 1, 0, 0, 0, 0, 0] == g4[0][1 * p.n_bands ** 4] / 2.0
    write_G4(str(path), StandIn(), normalized=False)
    with np.load(path) as f:
        assert np.array_equal(f["G4_PARTICLE_HOLE_CHARGE"].reshape(-1, order="F"), g4[1])
