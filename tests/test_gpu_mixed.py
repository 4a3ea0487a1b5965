"""Mixed-precision path (SDOT_MIXED): FP32 build of each cell, FP64 re-clip of
its vertices from the FP32 topology, FP64 integration; doubtful cells are
rebuilt in FP64.  Compared with the compiled reference (FP64 oracle).

The target is cell areas within 1e-7 of the FP64 oracle; because every
vertex is recomputed in FP64, the results are held here to the FP64 bounds
of the parity tests (1e-12 of max(|ref|, mean), 1e-11 with disc arcs), and
the neighbour sets must match exactly.
"""
import numpy as np
import pytest

from sdot_b200 import workloads
from tests.helpers import make_pair
from tests.test_gpu_parity_2d import check_all

pytestmark = pytest.mark.gpu


def test_mixed_uniform(gpu_lib, ref_oracle):
    rng = np.random.default_rng(21)
    n = 5000
    p = rng.random((n, 2))
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle, precision="mixed")
    check_all(gpu, ref, n)


def test_mixed_config2_weights(gpu_lib, ref_oracle):
    c = workloads.config2(n=50_000)
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle, precision="mixed")
    check_all(gpu, ref, 50_000, rtol_hess=1e-11)


def test_mixed_clustered_w0(gpu_lib, ref_oracle):
    # clamped clusters: collinear points on the box edges give sliver cells,
    # where the FP64 path already needs 1e-10 on the Hessian
    c = workloads.config2(n=50_000)
    gpu, ref = make_pair(c["positions"], np.zeros(50_000), ref_oracle, precision="mixed")
    check_all(gpu, ref, 50_000, rtol=1e-10, rtol_hess=1e-10)


def test_mixed_disc_clip_image(gpu_lib, ref_oracle):
    c = workloads.config3(n=5000, res=128)
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle, radial_func="in_ball_w05", image=c["image"],
                         precision="mixed")
    check_all(gpu, ref, 5000, rtol=1e-11)


def test_mixed_matches_fp64_path_closely(gpu_lib):
    # the two GPU paths on the 200k-Dirac clustered mix: masses and Hessian
    from sdot_b200.power_diagram import PowerDiagram

    c = workloads.config2(n=200_000)
    out = []
    for prec in ("fp64", "mixed"):
        g = PowerDiagram(c["positions"], c["weights"], precision=prec)
        g.add_box_shape([0, 0], [1, 1])
        out.append((g.integrals(), g.der_integrals_wrt_weights()))
    (m64, h64), (m32, h32) = out
    mean = np.abs(m64).mean()
    assert np.abs(m32 - m64).max() <= 1e-10 * mean
    assert np.array_equal(h64[0], h32[0]) and np.array_equal(h64[1], h32[1])


def test_mixed_newton(gpu_lib):
    # the mixed masses agree with the FP64 ones to round-off, which the
    # inverse Hessian (norm ~ n) amplifies in the solved weights
    from sdot_b200.power_diagram import PowerDiagram

    c = workloads.config1()
    n = len(c["weights"])
    ws = []
    for prec in ("fp64", "mixed"):
        g = PowerDiagram(c["positions"], c["weights"], precision=prec)
        g.add_box_shape([0, 0], [1, 1])
        g.solve_weights(np.full(n, 1.0 / n), rel_mass_tol=1e-12)
        ws.append(g.get_weights())
    assert np.abs(ws[0] - ws[1]).max() <= 1e-8 * np.abs(ws[0]).max()
