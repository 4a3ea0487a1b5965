"""Evaluation CLI for profiling runs (not a test module: pytest collects
test_*.py only).

    python tests/profile_case.py CASE REPS [LINEAR_SOLVER TOL]

Builds one named workload and evaluates it REPS times (masses, centroids,
Hessian), printing the stage times of each evaluation; the commands recorded
under profiles/ run this.  CASE is c2_N (the 2D clustered mix at N Diracs),
c3_N (the 2D image + disc-clip workload at N Diracs), c4_N (the 3D mix with
its density) or serving_K (request K < 100 of the seeded 100-request serving
stream, w = 0).  A suffix "_mixed" runs the mixed-precision path.  With
LINEAR_SOLVER ("fp64" or "fp32_refined") and TOL it runs one Newton solve from
w = 0 (the clustered case c2m_N mirrors the clusters at the box faces).
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from sdot_b200 import workloads  # noqa: E402
from sdot_b200.power_diagram import PowerDiagram  # noqa: E402


def main(argv):
    case, reps = argv[0], int(argv[1])
    precision = "fp64"
    if case.endswith("_mixed"):
        case, precision = case[:-6], "mixed"
    density = image = None
    ball = False
    if case.startswith("c2_"):
        c = workloads.config2(n=int(case[3:]))
        p, w = c["positions"], c["weights"]
    elif case.startswith("c2m_"):
        n = int(case[4:])
        rng = np.random.default_rng(workloads.SEED0 + 2)
        p = np.concatenate([workloads.uniform_points(n // 2, 2, rng),
                            workloads.clustered_points(n - n // 2, 2, rng, boundary="reflect")])
        w = np.zeros(n)
    elif case.startswith("c3_"):
        c = workloads.config3(n=int(case[3:]))
        p, w, image, ball = c["positions"], c["weights"], c["image"], True
    elif case.startswith("c4_"):
        c = workloads.config4(n=int(case[3:]))
        p, w, density = c["positions"], c["weights"], c["density"]
    elif case.startswith("serving_"):
        r = workloads.serving_requests(count=100)[int(case[8:])]
        p, w = r["positions"], np.zeros(r["n"])
    else:
        raise SystemExit(f"unknown case {case}")
    dim = p.shape[1]
    g = PowerDiagram(p, w, precision=precision, radial_func="in_ball_w05" if ball else "unit")
    if image is not None:
        g.set_image_density(image)
    else:
        g.add_box_shape(np.zeros(dim), np.ones(dim))
    if density is not None:
        g.set_polynomial_density(density)
    if len(argv) > 2:
        # a Newton solve with the given linear solver ("fp64" or
        # "fp32_refined") to the relative mass tolerance argv[3]
        t = np.full(len(w), (0.8 if image is not None else 1.0) / len(w))
        rep = g.solve_weights(t, rel_mass_tol=float(argv[3]), linear_solver=argv[2], raise_on_failure=False)
        print(case, argv[2], {k: rep[k] for k in ("status", "iterations", "pcg_iterations", "max_rel_mass_error",
                                                 "time_ms")}, flush=True)
        return
    for k in range(reps):
        g.set_weights(w)
        g.evaluate()
        print(case, k, {key: round(float(v), 3) for key, v in g.last_timings().items()}, flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
