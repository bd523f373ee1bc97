"""Generates the golden fixtures in this directory.

For each case it writes ``<name>.case`` (a case file, oracle/casefile.hpp) and ``<name>.ref``: the
output of the REFERENCE's own CPU accumulators -- TpAccumulator<Parameters, NONE, CPU> and
SpAccumulator<Parameters, CPU> compiled from the reference sources by oracle/refbuild into
oracle/_ref/tp_ref -- on that case.  The reference's HDF5 G4 baselines are not part of the
reference checkout (.MISSING_LARGE_BLOBS), so these fixtures are what pins the oracle.

Run here (needs the reference sources to build oracle/_ref):  python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dca_b200 import workloads as W  # noqa: E402
from oracle import casefile as CF  # noqa: E402
from oracle import pyoracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ALL_CHANNELS = (W.PH_TRANSVERSE, W.PH_MAGNETIC, W.PH_CHARGE, W.PP_UP_DOWN)


def _non_density_sector(rng, n, nb, nc, beta):
    s = W.make_sector(rng, n, nb, nc, beta)
    s.left_band = rng.integers(0, nb, n).astype(np.int32)
    s.left_site = rng.integers(0, nc, n).astype(np.int32)
    return s


def cases():
    """(name, workload, cluster, measurements, flags)."""
    out = []

    # 1. The 2x2 single-band configuration with PH magnetic, q = 0, wq = 0.
    w = W.WORKLOADS["c1"]
    cl = w.cluster()
    out.append(("c1_mag", w, cl, W.make_measurements(w, 3), 1))

    # 2. 2x2 single band, all four channels, all transfers with frequency transfer 2 (ext = 2).
    w = W.Workload("sq2_all", W.Model("single", t=1.0, U=4.0), ("square", 2), 5.0, 2, 16, True, 2, 0,
                   ALL_CHANNELS, (5, 15), 1, seed=7)
    cl = w.cluster()
    ms = W.make_measurements(w, 3)
    ms[1].sign = -1
    out.append(("sq2_all", w, cl, ms, 1))

    # 3. Three-band Emery model on a 2-site cluster, all channels, frequency transfers 0 and 1.
    w = W.Workload("mb3_all", W.Model("threeband", U=6.0), ("rect", (2, 0), (0, 1)), 4.0, 1, 16, True,
                   1, 0, ALL_CHANNELS, (6, 18), 1, seed=11)
    cl = w.cluster()
    w._nc = cl.nc
    ms = [W.make_measurement(w, i) for i in range(2)]
    out.append(("mb3_all", w, cl, ms, 1))

    # 4. 4x4 single band, one transfer (q index 5, frequency transfer 1), PH magnetic + PP,
    #    with an empty spin sector in the second measurement.
    w = W.Workload("sq4_q5", W.Model("single", t=1.0, U=6.0), ("square", 4), 8.0, 2, 16, False, 1, 5,
                   (W.PH_MAGNETIC, W.PP_UP_DOWN), (10, 30), 1, seed=3)
    cl = w.cluster()
    w._nc = cl.nc
    ms = [W.make_measurement(w, 0), W.make_measurement(w, 1, n_override=(0, 17))]
    out.append(("sq4_q5", w, cl, ms, 0))
    return out


def generate():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "refbuild")], check=True)
    for name, w, cl, ms, flags in cases():
        mu = w.chemical_potential()
        g0 = W.make_g0(w.model, cl, w.beta, mu, w.n_sp)
        case = os.path.join(HERE, name + ".case")
        ref = os.path.join(HERE, name + ".ref")
        CF.write_case(case, w, cl, g0, ms, flags=flags)
        log = pyoracle.run_reference(case, ref)
        print(name, os.path.getsize(case), os.path.getsize(ref), log.strip())


if __name__ == "__main__":
    generate()
