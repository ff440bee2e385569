"""Operator applications of GMRES(30) per wavelength for the headline sweep
(committed fixture cuboid30k_sweep_counts.json; needs a B200).

The reference's GMRES(30) (iterative.rs:53-159) applies the operator once per
Arnoldi step plus once at the start and once at the end of every restart
cycle.  A full oracle solve of the N = 30,000 Au cuboid takes minutes at
520 nm and hours at the plasmonic wavelengths, so the count per wavelength of
the 51-point 400-900 nm sweep is taken from the plain-FP64 device GMRES,
which runs the same algorithm in the same order (its iteration count equals
the oracle's to +-1 on every case the tests compare, and exactly at 520 nm,
N = 30,000).  The CPU baseline and the reference arm of bench.py scale a
sampled oracle matvec by these counts; the full oracle solve at 520 nm
(cuboid30k_oracle.json) anchors them.

Usage (on a GPU host): python tests/golden/make_cuboid30k_counts.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import lumina_b200 as lb  # noqa: E402
from lumina_b200 import configs  # noqa: E402

OUT = os.path.join(HERE, "cuboid30k_sweep_counts.json")
TOL = 1e-8
SWEEP_NM = [400.0 + 10.0 * i for i in range(51)]


def main():
    bk = lb.CudaBackend(0)
    base = configs.cuboid_au_30k(SWEEP_NM[0])
    counts, iters = {}, {}
    sess = None
    for lam in SWEEP_NM:
        w = configs.au_workload(base.name, base.positions, 1.0, lam)
        inv = lb.invert_polarisability(w.alpha)
        b = lb.incident_field(w.positions, w.k, lb.IncidentField())
        if sess is None:
            sess = bk.create_onthefly_session(w.positions, inv, w.k, True, 1.0)
        else:
            sess.set_wavelength(w.k, inv)
        _, info = sess.solve(b, TOL, 5000, 30, "fp64")
        assert info["converged"] == 1, lam
        counts[f"{lam:g}"] = info["matvecs_reference"]
        iters[f"{lam:g}"] = info["iterations"]
        print(f"{lam:g} nm: {info['iterations']} Arnoldi steps, "
              f"{info['matvecs_reference']} operator applications", flush=True)
    sess.close()
    with open(OUT, "w") as f:
        json.dump({"workload": "Au cuboid 60x50x10 nm, cell-centred 1 nm lattice, N = 30000, "
                               "FCD cell 1 nm, RRCM (J&C gold), vacuum, +z x-pol, GMRES(30) "
                               "from x0 = 0, tol 1e-8",
                   "n_dipoles": base.n, "tol": TOL,
                   "counted_by": "plain-FP64 device GMRES(30) (same algorithm as "
                                 "iterative.rs:33-160)",
                   "matvecs_reference": counts, "iterations": iters}, f, indent=1)


if __name__ == "__main__":
    main()
