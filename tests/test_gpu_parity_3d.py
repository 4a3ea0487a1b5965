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
