"""Full FP64 oracle solves of the N = 30,000 Au cuboid (committed fixture).

The oracle (oracle/cda_oracle.cpp, a restatement of matvec_on_the_fly
assembly.rs:209-318 and solve_gmres iterative.rs:33-160) runs GMRES(30) from
x0 = 0 to tol 1e-8 on the FP64 on-the-fly operator with FCD (cell 1 nm) for
the Au cuboid 60 x 50 x 10 nm on the cell-centred 1 nm lattice, +z incidence,
x polarisation.  Each solve takes minutes on a many-core host (one operator
application is ~2.6 s on 16 threads), so the results are stored once:
C_ext / C_abs / C_sca, the iteration and operator-application counts, the
wall time with its thread count and CPU, and the moments of 512 dipoles
spread over the lattice (plus the first and last).  The device solves are
checked against this file at the full size.

Usage: python tests/golden/make_cuboid30k_oracle.py [wavelength_nm ...]
       (default 520; results are merged into cuboid30k_oracle.json)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lumina_b200 import configs  # noqa: E402
from oracle import oracle as orc  # noqa: E402

OUT = os.path.join(HERE, "cuboid30k_oracle.json")
TOL = 1e-8
MAX_ITER = 5000


def sample_indices(n, count=512):
    idx = np.unique(np.concatenate([np.linspace(0, n - 1, count).astype(np.int64), [0, n - 1]]))
    return idx


def cpu_model():
    with open("/proc/cpuinfo") as f:
        for line in f:
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    return "unknown"


def solve(lam):
    w = configs.cuboid_au_30k(lam)
    b = orc.incident_field(w.positions, w.k)
    nt = orc.max_threads()
    t0 = time.perf_counter()
    r = orc.gmres_onthefly(w.positions, w.alpha, b, w.k, True, w.cell_size, tol=TOL,
                           max_iter=MAX_ITER, nthreads=nt)
    secs = time.perf_counter() - t0
    cs = orc.cross_sections(w.positions, w.alpha, r.x, w.k)
    idx = sample_indices(w.n)
    p = r.x.reshape(-1, 3)[idx]
    return {"wavelength_nm": lam, "n_dipoles": w.n, "k": w.k, "tol": TOL,
            "status": int(r.status), "iterations": r.iterations, "matvecs": r.matvecs,
            "rel_residual": r.rel_residual, "c_ext": cs[0], "c_abs": cs[1], "c_sca": cs[2],
            "seconds": secs, "threads": nt, "cpu": cpu_model(),
            "sample_dipoles": idx.tolist(),
            "sample_moments_re": p.real.ravel().tolist(),
            "sample_moments_im": p.imag.ravel().tolist()}


def main():
    lams = [float(v) for v in sys.argv[1:]] or [520.0]
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data.setdefault("workload", "Au cuboid 60x50x10 nm, cell-centred 1 nm lattice, N = 30000, "
                                "FCD cell 1 nm, RRCM (J&C gold), vacuum, +z x-pol, GMRES(30) "
                                "tol 1e-8, FP64 on-the-fly oracle")
    solves = {s["wavelength_nm"]: s for s in data.get("solves", [])}
    for lam in lams:
        s = solve(lam)
        print(f"{lam} nm: status {s['status']} iterations {s['iterations']} matvecs {s['matvecs']} "
              f"C_ext {s['c_ext']:.10e} in {s['seconds']:.0f} s on {s['threads']} threads",
              flush=True)
        solves[lam] = s
        data["solves"] = [solves[k] for k in sorted(solves)]
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
