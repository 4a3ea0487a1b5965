"""GPU parity at the benchmark workloads' full sizes, against the compiled
reference (one evaluation per arm, the reference on all host threads).

  C2  1,000,000 Diracs, 50% uniform + 50% clamped Gaussian clusters,
      w ~ U[-1e-6, 1e-6], unit box: FP64 path and mixed path
  C3  500,000 Diracs, 512 x 512 image density, disc clip (InBallW05)
  C4  200,000 Diracs in 3D (70% uniform + 30% jittered lattice), unit cube,
      density 1 (the reference integrates no smooth 3D density)

Bounds (relative to max(|ref|, mean of the quantity), as in the smaller
parity tests):
  * C2: the reference and the C restatement of it (oracle/sdot_oracle.c, the
    same cut sequence in plain C) differ on this input by 8.0e-13 in the
    masses and 1.14e-10 in the Hessian values: clamping puts runs of
    collinear Diracs on the box edges, whose bisectors are nearly parallel,
    so a vertex carries an error of eps / sin(angle).  Masses and centroids
    are held to 1e-11 and the Hessian to 1e-9 (ten times that spread).
  * C3: where a cell edge is nearly tangent to the clipping disc, the
    edge-circle intersection is the root of a discriminant at rounding level,
    so inputs that differ by one ulp move it by ~sqrt(eps * r) along the edge.
    The reference and the C restatement differ on this input by 6.8e-10 in
    the masses (54 cells above 1e-11), 1.5e-13 in the centroids and 6.9e-11 in
    the Hessian values: masses and Hessian are held to 1e-9, centroids to
    1e-11.
  * C4: 1e-12 for volumes and centroids, 1e-11 for the Hessian, the bounds of
    the 20k-Dirac 3D test.
Neighbour sets and CSR patterns must match exactly.
"""
import numpy as np
import pytest

from sdot_b200 import workloads
from tests.helpers import make_pair
from tests.test_gpu_parity_2d import check_all

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config2_full_size(gpu_lib, ref_oracle, precision):
    c = workloads.config2()
    n = len(c["weights"])
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle, precision=precision)
    check_all(gpu, ref, n, rtol=1e-11, rtol_hess=1e-9)
    m = gpu.integrals()
    assert (m == 0).sum() > 0.3 * n  # the weight spread empties ~44% of the cells
    assert abs(m.sum() - 1.0) < 1e-11


def test_config3_full_size(gpu_lib, ref_oracle):
    c = workloads.config3()
    n = len(c["weights"])
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle, radial_func="in_ball_w05", image=c["image"])
    check_all(gpu, ref, n, rtol=1e-9, rtol_hess=1e-9, rtol_ctd=1e-11)


def test_config4_geometry_full_size(gpu_lib, ref_oracle):
    c = workloads.config4()
    n = len(c["weights"])
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle)
    check_all(gpu, ref, n, rtol=1e-12, rtol_hess=1e-11)
    assert abs(gpu.integrals().sum() - 1.0) < 1e-11
