"""3D power diagrams on the GPU vs the compiled reference (ConvexPolyhedron3
path of the reference), FP64, unit-cube domain.

Same bounds as the 2D parity tests: volumes, centroids and Hessian values
within RTOL of max(|ref|, mean of the quantity), identical neighbour sets and
CSR patterns.  The 3D volume is summed over faces with the cell's Dirac as
the apex (the reference uses the origin), which changes rounding only.
"""
import numpy as np
import pytest

from sdot_b200 import workloads
from tests.helpers import make_pair
from tests.test_gpu_parity_2d import check_all

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.mark.parametrize("n", [1, 2, 9, 300, 3000])
def test_uniform_unit_cube(gpu_lib, ref_oracle, n):
    rng = np.random.default_rng(300 + n)
    p = rng.random((n, 3))
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle)
    check_all(gpu, ref, n, rtol=RTOL)
    assert abs(gpu.integrals().sum() - 1.0) < 1e-12


def test_weighted_cube(gpu_lib, ref_oracle):
    rng = np.random.default_rng(31)
    n = 4000
    p = rng.random((n, 3))
    w = rng.uniform(-1, 1, n) * 0.2 * (1.0 / n) ** (2 / 3)
    gpu, ref = make_pair(p, w, ref_oracle)
    check_all(gpu, ref, n, rtol=RTOL, rtol_hess=1e-11)


def test_config4_mix(gpu_lib, ref_oracle):
    # 70% uniform + 30% jittered lattice, 20k Diracs
    c = workloads.config4(n=20_000)
    n = len(c["weights"])
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle)
    check_all(gpu, ref, n, rtol=RTOL, rtol_hess=1e-11)


def test_newton_3d(gpu_lib, ref_oracle):
    from oracle import newton

    rng = np.random.default_rng(33)
    n = 1500
    p = rng.random((n, 3))
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle)
    t = np.full(n, 1.0 / n)
    gpu.solve_weights(t, rel_mass_tol=1e-12)
    w_r, rep = newton.solve(ref, t, np.zeros(n), tol=1e-12)
    assert rep["converged"]
    w_g = gpu.get_weights()
    assert np.abs(w_g - w_r).max() <= 1e-10 * np.abs(w_r).max()


def test_clustered_cube(gpu_lib, ref_oracle):
    # 20 Gaussian clusters (sigma 0.02, mirrored at the faces): cells on the
    # clusters' rims reach far into the empty space and have many faces (the
    # larger-capacity passes)
    rng = np.random.default_rng(34)
    n = 30000
    p = workloads.clustered_points(n, 3, rng, boundary="reflect")
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle)
    check_all(gpu, ref, n, rtol=1e-11, rtol_hess=1e-10)


# ---- multilinear density (no reference integrator: the oracle is the qhull
# restatement in oracle/poly3d.py, pinned to the reference at density 1)
def _dict_rows(off, col, val):
    H = {}
    for i in range(len(off) - 1):
        for k in range(off[i], off[i + 1]):
            H[(i, int(col[k]))] = H.get((i, int(col[k])), 0.0) + val[k]
    return H


@pytest.mark.parametrize("coeffs", ["c4", "random"])
def test_polynomial_density_vs_oracle(gpu_lib, coeffs):
    from oracle import poly3d
    from sdot_b200.power_diagram import PowerDiagram

    rng = np.random.default_rng(41)
    n = 400
    p = rng.random((n, 3))
    w = rng.uniform(-1, 1, n) * 0.2 * (1.0 / n) ** (2 / 3)
    if coeffs == "c4":
        a = workloads.C4_DENSITY
    else:
        a = np.concatenate([[1.0], rng.uniform(-0.2, 0.2, 7)])
    g = PowerDiagram(p, w)
    g.add_box_shape(np.zeros(3), np.ones(3), coeff=1.7)
    g.set_polynomial_density(a)
    m_o, c_o, H_o = poly3d.integrate(p, w, poly=a, coeff=1.7)
    m = g.integrals()
    c = g.centroids()
    off, col, val, _ = g.der_integrals_wrt_weights()
    H = _dict_rows(off, col, val)
    np.testing.assert_allclose(m, m_o, rtol=1e-11, atol=1e-12 * m_o.mean())
    np.testing.assert_allclose(c, c_o, rtol=1e-11, atol=1e-12)
    scale = max(abs(v) for v in H_o.values())
    keys = set(H) | set(H_o)
    worst = max(abs(H.get(k, 0.0) - H_o.get(k, 0.0)) for k in keys)
    assert worst < 1e-11 * scale, worst
    assert abs(m.sum() - 1.7 * poly3d.box_integral(a)) < 1e-12 * m.sum()
    assert abs(g.domain_measure() - 1.7 * poly3d.box_integral(a)) < 1e-14


def test_config4_density_newton(gpu_lib):
    # the 3D workload as specified: 200k Diracs, density (1 + 0.3 xyz)
    # normalised, Newton to a relative mass error of 1e-8 from w = 0
    from sdot_b200.power_diagram import PowerDiagram

    c = workloads.config4()
    g = PowerDiagram(c["positions"], c["weights"])
    g.add_box_shape(np.zeros(3), np.ones(3))
    g.set_polynomial_density(c["density"])
    assert abs(g.domain_measure() - 1.0) < 1e-14
    m0 = g.integrals()
    assert abs(m0.sum() - 1.0) < 1e-12
    rep = g.solve_weights(c["target"], rel_mass_tol=1e-8)
    m = g.integrals()
    assert np.max(np.abs(m - c["target"]) / c["target"]) <= 1e-8
    assert rep["iterations"] <= 20
    assert rep["pcg_levels"] >= 4  # the multilevel preconditioner ran (coarse rows of 128)
