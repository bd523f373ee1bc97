"""Synthetic accumulation workloads: cluster geometry, bare G0, and walker measurements.

There is no Monte Carlo walker here.  Each measurement is generated directly with the shapes,
sizes and value distributions of a CT-AUX / CT-INT measurement, so the accumulators see the
same kind of input the reference's walkers hand to ``TpAccumulator::accumulate`` and
``SpAccumulator::accumulate`` (ctaux_accumulator.hpp:520-523, ctint_accumulator.hpp:234-248):

* per spin sector, an expansion order ``n ~ U[lo, hi]``;
* vertices with ``tau ~ U[0, beta)``, site ``~ U{0..Nc-1}``, band ``~ U{0..nb-1}``
  (a density-density vertex: left and right band / site are equal);
* ``M = (I + A)^-1`` with ``A_ij ~ N(0, 0.1 / n)`` (real, FP64);
* Monte Carlo sign ``+1`` with probability 0.95, else ``-1``.

Measurement ``m`` of a workload with seed ``s`` draws from ``numpy.random.default_rng([s, m])``,
so any subset of a workload is reproducible on its own.

Bare Green's functions:

* single band: ``G0(K, i w) = 1 / (i w + mu - eps_K)`` with
  ``eps_K = -2 t (cos Kx + cos Ky) - 4 t' cos Kx cos Ky``;
* three-band (d, px, py) Emery model: ``G0(K, i w) = ((i w + mu) I - H0(K))^-1`` with the hopping
  matrix elements of the reference's threeband_hubbard.hpp:322-336 (d-px ``-2 i t_pd sin(kx/2)``,
  d-py ``2 i t_pd sin(ky/2)``, px-py ``4 t_pp sin(kx/2) sin(ky/2)``) and on-site energies
  ``eps_d - eps_p = 3.24`` (``eps_p = 0``); band a-vectors (0,0), (1/2,0), (0,1/2)
  (threeband_hubbard.hpp:151-154).

``mu`` is fixed by bisection so that the bare density on a 64 x 64 k mesh at the workload's beta
is 1 per site (single band) or 5 electrons per cell (three band); G0 is an input of the
accumulators, so any documented choice is valid for parity.
"""

from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

# FourPointType values of the reference (include/dca/phys/four_point_type.hpp:27-33).
PH_TRANSVERSE = 1
PH_MAGNETIC = 2
PH_CHARGE = 3
PP_UP_DOWN = 4

CHANNEL_NAMES = {
    PH_TRANSVERSE: "PARTICLE_HOLE_TRANSVERSE",
    PH_MAGNETIC: "PARTICLE_HOLE_MAGNETIC",
    PH_CHARGE: "PARTICLE_HOLE_CHARGE",
    PP_UP_DOWN: "PARTICLE_PARTICLE_UP_DOWN",
}


# ----------------------------------------------------------------------------------------------
# Cluster geometry
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Cluster:
    """A 2D cluster with periodic boundary conditions given by two superlattice vectors."""

    r_vecs: np.ndarray  # (Nc, 2) real-space sites
    k_vecs: np.ndarray  # (Nc, 2) cluster momenta in (-pi, pi]
    r_add: np.ndarray  # (Nc, Nc) int32, [i, j] = index of r_i + r_j
    r_sub: np.ndarray  # (Nc, Nc) int32, [i, j] = index of r_j - r_i
    k_add: np.ndarray
    k_sub: np.ndarray

    @property
    def nc(self) -> int:
        return self.r_vecs.shape[0]


def _reduce_to_bz(k: np.ndarray) -> np.ndarray:
    """Maps each component into (-pi, pi]."""
    out = np.mod(k + math.pi, 2 * math.pi) - math.pi
    out[np.isclose(out, -math.pi, atol=1e-12)] = math.pi
    return out


def make_cluster(R1: Sequence[int], R2: Sequence[int]) -> Cluster:
    """Builds the cluster whose superlattice is spanned by the integer vectors R1, R2.

    Add / subtract tables follow the reference convention (cluster_domain_initializer.hpp:691-765):
    ``add[i, j]`` is the index of ``x_i + x_j`` and ``sub[i, j]`` the index of ``x_j - x_i``,
    both reduced modulo the superlattice (real space) or the reciprocal lattice (momenta).
    """
    Rm = np.array([R1, R2], dtype=float).T  # columns are superlattice vectors
    nc = int(round(abs(np.linalg.det(Rm))))
    Rinv = np.linalg.inv(Rm)

    def reduce_r(r):
        f = Rinv @ r
        f = f - np.floor(f + 1e-9)
        return Rm @ f

    span = int(np.abs(Rm).sum()) + 1
    sites: List[np.ndarray] = []
    for x in range(-span, span + 1):
        for y in range(-span, span + 1):
            r = reduce_r(np.array([x, y], dtype=float))
            if not any(np.allclose(r, s) for s in sites):
                sites.append(r)
    sites.sort(key=lambda v: (round(v[1], 6), round(v[0], 6)))
    r_vecs = np.array(sites)
    assert r_vecs.shape[0] == nc

    # Reciprocal superlattice: K_i . R_j = 2 pi delta_ij.
    Kb = 2 * math.pi * Rinv  # rows are K1, K2
    ks: List[np.ndarray] = []
    for a in range(-nc, nc + 1):
        for b in range(-nc, nc + 1):
            k = _reduce_to_bz(a * Kb[0] + b * Kb[1])
            if not any(np.allclose(k, s) for s in ks):
                ks.append(k)
    ks.sort(key=lambda v: (round(v[1], 6), round(v[0], 6)))
    k_vecs = np.array(ks)
    assert k_vecs.shape[0] == nc

    def index_r(r):
        rr = reduce_r(r)
        for i, s in enumerate(r_vecs):
            if np.allclose(rr, s, atol=1e-8):
                return i
        raise ValueError("site not found")

    def index_k(k):
        kk = _reduce_to_bz(k)
        for i, s in enumerate(k_vecs):
            d = (kk - s) / (2 * math.pi)
            if np.allclose(d, np.round(d), atol=1e-8):
                return i
        raise ValueError("momentum not found")

    r_add = np.zeros((nc, nc), np.int32)
    r_sub = np.zeros((nc, nc), np.int32)
    k_add = np.zeros((nc, nc), np.int32)
    k_sub = np.zeros((nc, nc), np.int32)
    for i in range(nc):
        for j in range(nc):
            r_add[i, j] = index_r(r_vecs[i] + r_vecs[j])
            r_sub[i, j] = index_r(r_vecs[j] - r_vecs[i])
            k_add[i, j] = index_k(k_vecs[i] + k_vecs[j])
            k_sub[i, j] = index_k(k_vecs[j] - k_vecs[i])
    return Cluster(r_vecs, k_vecs, r_add, r_sub, k_add, k_sub)


def square_cluster(L: int) -> Cluster:
    return make_cluster((L, 0), (0, L))


def betts8_cluster() -> Cluster:
    return make_cluster((2, 2), (2, -2))


# ----------------------------------------------------------------------------------------------
# Models and G0
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Model:
    kind: str  # "single" or "threeband"
    t: float = 1.0
    tp: float = 0.0
    U: float = 0.0
    t_pd: float = 1.13
    t_pp: float = 0.49
    eps_d_minus_eps_p: float = 3.24

    @property
    def nb(self) -> int:
        return 1 if self.kind == "single" else 3

    def a_vecs(self) -> np.ndarray:
        if self.kind == "single":
            return np.zeros((1, 2))
        return np.array([[0.0, 0.0], [0.5, 0.0], [0.0, 0.5]])

    def h0(self, k: np.ndarray) -> np.ndarray:
        """H0(k) as an (nb, nb) complex matrix."""
        if self.kind == "single":
            eps = -2 * self.t * (math.cos(k[0]) + math.cos(k[1])) - 4 * self.tp * math.cos(
                k[0]
            ) * math.cos(k[1])
            return np.array([[eps]], dtype=complex)
        I = 1j
        h = np.zeros((3, 3), complex)
        h[0, 0] = self.eps_d_minus_eps_p
        dpx = -2 * I * self.t_pd * math.sin(k[0] / 2)
        dpy = 2 * I * self.t_pd * math.sin(k[1] / 2)
        pxpy = 4 * self.t_pp * math.sin(k[0] / 2) * math.sin(k[1] / 2)
        h[0, 1], h[1, 0] = dpx, -dpx
        h[0, 2], h[2, 0] = dpy, -dpy
        h[1, 2] = h[2, 1] = pxpy
        return h

    def target_density(self) -> float:
        return 1.0 if self.kind == "single" else 5.0


def find_mu(model: Model, beta: float, mesh: int = 64) -> float:
    """Bisection for mu such that the bare density per cell equals model.target_density()."""
    ks = [
        np.array([2 * math.pi * a / mesh, 2 * math.pi * b / mesh])
        for a in range(mesh)
        for b in range(mesh)
    ]
    evals = np.concatenate([np.linalg.eigvalsh(model.h0(k)) for k in ks])

    def density(mu):
        x = np.clip(beta * (evals - mu), -700, 700)
        return 2.0 * np.sum(1.0 / (np.exp(x) + 1.0)) / len(ks)

    lo, hi = evals.min() - 20, evals.max() + 20
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if density(mid) < model.target_density():
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def matsubara(beta: float, n_pos: int) -> np.ndarray:
    """Fermionic Matsubara frequencies pi (2m+1) / beta, m = -n_pos .. n_pos-1.

    Same ordering as the reference's frequency_domain (frequency_domain.cpp:29-47).
    """
    m = np.arange(-n_pos, n_pos)
    return (2 * m + 1) * math.pi / beta


def make_g0(model: Model, cluster: Cluster, beta: float, mu: float, n_sp: int) -> np.ndarray:
    """G0 in the reference layout (b1, s1, b2, s2, k, w), first index fastest.

    Returned as a complex128 array of shape (2 n_sp, Nc, 2, nb, 2, nb) (C order, so the LAST axis
    is fastest and flattening gives the reference's linear order).
    """
    nb = model.nb
    nc = cluster.nc
    w = matsubara(beta, n_sp)
    out = np.zeros((2 * n_sp, nc, 2, nb, 2, nb), complex)
    eye = np.eye(nb)
    for ik, k in enumerate(cluster.k_vecs):
        h = model.h0(k)
        for iw, wn in enumerate(w):
            g = np.linalg.inv((1j * wn + mu) * eye - h)  # g[b1, b2]
            for s in range(2):
                out[iw, ik, s, :, s, :] = g.T  # [b2, b1] so b1 is the fastest index
    return out


# ----------------------------------------------------------------------------------------------
# Workload specifications (the five synthetic configurations)
# ----------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Workload:
    name: str
    model: Model
    cluster_kind: Tuple  # ("square", L), ("rect", R1, R2) or ("betts8",)
    beta: float
    nw_half: int  # four-point fermionic frequencies (Nw = 2 nw_half)
    n_sp: int  # single-particle fermionic frequencies (positive)
    all_transfers: bool
    freq_transfer: int
    k_transfer: int
    channels: Tuple[int, ...]
    n_range: Tuple[int, int]
    batch: int
    seed: int = 42
    mu: Optional[float] = None

    def cluster(self) -> Cluster:
        kind = self.cluster_kind[0]
        if kind == "square":
            return square_cluster(self.cluster_kind[1])
        if kind == "rect":
            return make_cluster(self.cluster_kind[1], self.cluster_kind[2])
        return betts8_cluster()

    @property
    def nb(self) -> int:
        return self.model.nb

    def chemical_potential(self) -> float:
        if self.mu is None:
            if self.model.kind == "single" and self.model.tp == 0.0:
                self.mu = 0.0  # particle-hole symmetric: half filling at mu = 0
            else:
                self.mu = find_mu(self.model, self.beta)
        return self.mu

    # Derived sizes (NwExt = Nw + 2 ext, D = nb Nc NwExt).
    def exchange_frequencies(self) -> List[int]:
        if self.all_transfers:
            return list(range(self.freq_transfer + 1))
        return [self.freq_transfer]

    def exchange_momenta(self, nc: int) -> List[int]:
        if self.all_transfers:
            return list(range(nc))
        return [self.k_transfer]

    def ext(self) -> int:
        return max(abs(w) for w in self.exchange_frequencies())

    def describe(self, with_batch: bool = True) -> str:
        """One line naming the workload by what it is: model, cluster, frequencies, transfers,
        channels, expansion orders and batch."""
        cl = self.cluster()
        if self.model.kind == "single":
            model = f"single-band Hubbard (t={self.model.t:g}, t'={self.model.tp:g}, U={self.model.U:g})"
        else:
            model = f"three-band Emery (U_dd={self.model.U:g})"
        kind = self.cluster_kind[0]
        cluster = f"{self.cluster_kind[1]}x{self.cluster_kind[1]}" if kind == "square" else kind
        chans = " + ".join(CHANNEL_NAMES[c] for c in self.channels)
        s = (f"{self.name}: {model}, {cluster} cluster (Nc={cl.nc}), beta={self.beta:g}, "
             f"Nw={2 * self.nw_half}, {len(self.exchange_momenta(cl.nc))} q x "
             f"{len(self.exchange_frequencies())} wq, {chans}, n~U[{self.n_range[0]},{self.n_range[1]}]")
        return s + (f", batch {self.batch}" if with_batch else "")


WORKLOADS = {
    # 2x2 single-band Hubbard, the reference CPU path's own scale.
    "c1": Workload(
        "c1", Model("single", t=1.0, U=4.0), ("square", 2), 10.0, 8, 64, False, 0, 0,
        (PH_MAGNETIC,), (20, 60), 1),
    # 4x4 single band, unbatched: FP64 vs mixed precision.
    "c2": Workload(
        "c2", Model("single", t=1.0, U=6.0), ("square", 4), 20.0, 32, 512, True, 0, 0,
        (PH_MAGNETIC, PH_CHARGE), (100, 300), 1),
    # 4x4 single band, batched uneven orders (the headline workload).
    "c3": Workload(
        "c3", Model("single", t=1.0, U=6.0), ("square", 4), 20.0, 32, 512, True, 0, 0,
        (PH_MAGNETIC, PH_CHARGE), (50, 400), 64),
    # Three-band Emery model on the Betts 8-site cluster, particle-particle channel.
    "c4": Workload(
        "c4", Model("threeband", U=6.0), ("betts8",), 16.0, 16, 256, True, 3, 0,
        (PP_UP_DOWN,), (100, 500), 32),
    # 6x6 single band with t' = -0.15.
    "c5": Workload(
        "c5", Model("single", t=1.0, tp=-0.15, U=7.0), ("square", 6), 40.0, 64, 512, True, 0, 0,
        (PH_MAGNETIC,), (300, 1000), 128),
}


@dataclasses.dataclass
class Sector:
    tau: np.ndarray  # (n,) float64
    left_band: np.ndarray  # (n,) int32
    right_band: np.ndarray
    left_site: np.ndarray
    right_site: np.ndarray
    M: np.ndarray  # (n, n) float64, Fortran order (column major)

    @property
    def n(self) -> int:
        return self.tau.shape[0]


@dataclasses.dataclass
class Measurement:
    sign: int
    sectors: Tuple[Sector, Sector]


def make_sector(rng: np.random.Generator, n: int, nb: int, nc: int, beta: float) -> Sector:
    tau = rng.uniform(0.0, beta, n)
    site = rng.integers(0, nc, n).astype(np.int32)
    band = rng.integers(0, nb, n).astype(np.int32)
    _hs_spin = rng.choice([-1, 1], n)  # carried by a walker configuration, unused by the math
    A = rng.normal(0.0, math.sqrt(0.1 / max(n, 1)), (n, n))
    M = np.asfortranarray(np.linalg.inv(np.eye(n) + A)) if n else np.zeros((0, 0), order="F")
    return Sector(tau, band.copy(), band.copy(), site.copy(), site.copy(), M)


def make_measurement(w: Workload, index: int, n_override: Optional[Tuple[int, int]] = None
                     ) -> Measurement:
    rng = np.random.default_rng([w.seed, index])
    nc = w.cluster().nc if not hasattr(w, "_nc") else w._nc
    lo, hi = w.n_range
    sectors = []
    for s in range(2):
        n = int(rng.integers(lo, hi + 1)) if n_override is None else n_override[s]
        sectors.append(make_sector(rng, n, w.nb, nc, w.beta))
    sign = 1 if rng.uniform() < 0.95 else -1
    return Measurement(sign, (sectors[0], sectors[1]))


def make_measurements(w: Workload, count: int, start: int = 0) -> List[Measurement]:
    w._nc = w.cluster().nc  # cache for make_measurement
    return [make_measurement(w, start + i) for i in range(count)]
