"""Generates tests/golden/newton_floor_c2.json: the FP64 floor of Newton on the
clamped 2D clustered workload, measured with the compiled reference.

The clustered Diracs of the 2D workload are clamped to the unit box, which
puts pairs of Diracs on the box edges a few 1e-8 apart.  This script runs the
Newton oracle (oracle/newton.py: the reference's update rule with KMT damping,
a direct sparse solve, the compiled reference's masses and CSR Hessian) from
w = 0 towards a relative mass error of 1e-8, and records per size the
relative mass error at each iteration and the smallest distance between two
Diracs, so that the floor the GPU solver meets on the same input is shown to
be the reference's own.  Test infrastructure only (needs the reference
checkout to build oracle/_ref).

    python tests/golden/make_newton_floor.py [n ...]   (default 100000 300000)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import newton, ref  # noqa: E402
from sdot_b200 import workloads  # noqa: E402


def min_pair_distance(p):
    from scipy.spatial import cKDTree

    d, _ = cKDTree(p).query(p, k=2)
    return float(d[:, 1].min())


def main(sizes):
    ref.build()
    out = {"workload": "2D clustered mix (50% uniform + 50% 20 Gaussian clusters sigma 0.02 clamped to the box), "
                       "w0 = 0, targets 1/n, unit box; Newton oracle with the compiled reference and a direct solve",
           "tolerance_asked": 1e-8, "runs": []}
    for n in sizes:
        c = workloads.config2(n=n)
        p = c["positions"]
        r = ref.RefPowerDiagram(p, np.zeros(n))
        r.add_box_shape([0.0, 0.0], [1.0, 1.0])
        trace = []
        t0 = time.perf_counter()
        _, rep = newton.solve(r, np.full(n, 1.0 / n), np.zeros(n), tol=1e-8, max_iter=40, trace=trace)
        out["runs"].append({"n": n, "converged": bool(rep["converged"]), "final_max_rel_mass_error":
                            rep["max_rel_mass_error"], "iterations": rep["iterations"], "trace": trace,
                            "min_pair_distance": min_pair_distance(p), "seconds": time.perf_counter() - t0})
        print(n, rep["converged"], rep["max_rel_mass_error"], rep["iterations"], flush=True)
    with open(os.path.join(HERE, "newton_floor_c2.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main([int(a) for a in sys.argv[1:]] or [100_000, 300_000])
