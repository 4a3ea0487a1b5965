"""GPU position derivatives (get_der_centroids_and_integrals_wrt_weight_and_positions,
2D) vs the compiled reference oracle.

The CSR over 3 n rows (row 3 i + d: centroid x, centroid y, mass of cell i;
column 3 j + e: x, y, weight of Dirac j) must have the reference's offsets and
columns exactly; values within RTOL of max(|reference value|, the mean |value|
of the rows of the same output), the per-output floor because a block's
rounding error is set by the cell's coordinates, not by the block's size.

The GPU rebuilds each vertex from its two edge lines where the reference
carries the clipped vertices, so the two differ by vertex rounding, which the
centroid rows amplify: they are (d int x - c d mass) / mass in absolute
coordinates, a cancellation of order |c| / cell size.  The reference differs
from itself by as much: the same 20k clustered mix with every coordinate
shifted by (0.125, 0.375), which leaves every block unchanged in exact
arithmetic, moves its centroid rows by up to 3.4e-8 and its mass rows by up to
6.4e-11 (relative, as above).  Hence RTOL_CTD = 1e-7 on the clustered mix and
1e-9 on the uniform inputs; RTOL_MASS = 1e-10 throughout."""
import numpy as np
import pytest

from sdot_b200 import workloads
from sdot_b200.power_diagram import PowerDiagram
from tests.helpers import assert_close, make_pair

pytestmark = pytest.mark.gpu

RTOL_CTD = 1e-9
RTOL_MASS = 1e-10
PERIODIC_T = [(x, y) for x in (-1.0, 0.0, 1.0) for y in (-1.0, 0.0, 1.0) if x or y]


def check_derpos(gpu, ref, n, rtol_ctd=RTOL_CTD, rtol_mass=RTOL_MASS):
    go, gc, gv, gval = gpu.der_centroids_and_integrals_wrt_weight_and_positions()
    ro, rc, rv, rval = ref.der_centroids_and_integrals_wrt_weight_and_positions()
    assert go.shape == (3 * n + 1,)
    assert np.array_equal(go, ro), "CSR offsets differ"
    assert np.array_equal(gc, rc), "CSR columns differ"
    rows = np.repeat(np.arange(3 * n), np.diff(ro))
    floor = np.zeros(len(rv))
    for d in range(3):
        sel = rows % 3 == d
        floor[sel] = max(float(np.nanmean(np.abs(rv[sel]))), 1e-300) if sel.any() else 1.0
    # a void cell's centroid rows are 0 / 0 in the reference (it divides by
    # the mass): NaN on both sides, at the same places
    assert np.array_equal(np.isnan(gv), np.isnan(rv)), "NaN entries differ"
    ok = ~np.isnan(rv)
    gv, rv, floor, rows = gv[ok], rv[ok], floor[ok], rows[ok]
    dv = np.abs(gv - rv)
    e = np.where(dv == 0, 0.0, dv / np.maximum(np.abs(rv), floor))
    for d, rtol in ((0, rtol_ctd), (1, rtol_ctd), (2, rtol_mass)):
        ed = np.where(rows % 3 == d, e, 0.0)
        k = int(np.argmax(ed)) if ed.size else 0
        assert ed.size == 0 or ed.max() <= rtol, \
            f"output {d}: max rel err {ed.max():.3e} at {k} (row {rows[k]}): {gv[k]!r} vs {rv[k]!r}"
    mean_mass = max(float(np.abs(rval[2::3]).mean()), 1e-300)
    assert_close(gval[2::3], rval[2::3], 1e-12, mean_mass, "masses")
    assert_close(gval.reshape(n, 3)[:, :2], rval.reshape(n, 3)[:, :2], 1e-12, 1.0, "centroids")


@pytest.mark.parametrize("n", [1, 2, 7, 100, 3000])
def test_derpos_uniform_box(gpu_lib, ref_oracle, n):
    rng = np.random.default_rng(300 + n)
    p = rng.random((n, 2))
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle)
    check_derpos(gpu, ref, n)


def test_derpos_weighted_clustered(gpu_lib, ref_oracle):
    c = workloads.config2(n=20_000)
    p, w = c["positions"], c["weights"]
    gpu, ref = make_pair(p, w, ref_oracle)
    check_derpos(gpu, ref, len(p), rtol_ctd=1e-7)


def test_derpos_box_with_density(gpu_lib, ref_oracle):
    # a box of density 2.5 and size 3 x 2: the measure carries the density
    rng = np.random.default_rng(310)
    n = 500
    p = rng.random((n, 2)) * [3.0, 2.0] + [-1.0, 0.5]
    shapes = [("add_box_shape", ([-1.0, 0.5], [2.0, 2.5], 2.5))]
    gpu, ref = make_pair(p, rng.uniform(-1e-3, 1e-3, n), ref_oracle, shapes=shapes)
    check_derpos(gpu, ref, n)


def test_derpos_convex_domain(gpu_lib, ref_oracle):
    rng = np.random.default_rng(311)
    n = 2000
    ang = (np.arange(20) + 0.5) * 2 * np.pi / 20
    pts = np.stack([0.5 + 0.5 * np.cos(ang), 0.5 + 0.5 * np.sin(ang)], 1)
    nrm = np.stack([np.cos(ang), np.sin(ang)], 1)
    p = 0.5 + (rng.random((n, 2)) - 0.5) * 0.9
    shapes = [("add_convex_polyhedron_shape", (pts, nrm, 1.0))]
    gpu, ref = make_pair(p, rng.uniform(-1e-5, 1e-5, n), ref_oracle, shapes=shapes)
    check_derpos(gpu, ref, n)


@pytest.mark.parametrize("n", [3, 40, 3000])
def test_derpos_periodic(gpu_lib, ref_oracle, n):
    # small n: a cell meets its own images and several images of one
    # neighbour, so equal columns are merged
    rng = np.random.default_rng(320 + n)
    p = rng.random((n, 2))
    w = rng.uniform(-1e-6, 1e-6, n)
    shapes = [("add_box_shape", ([-1.0, -1.0], [2.0, 2.0], 1.0))]
    gpu, ref = make_pair(p, w, ref_oracle, shapes=shapes)
    gpu.set_translations(PERIODIC_T)
    ref.set_translations(PERIODIC_T)
    check_derpos(gpu, ref, n)


def test_derpos_mixed_precision_context(gpu_lib, ref_oracle):
    # a mixed-precision context: FP32 cell ids, FP64 derivatives
    rng = np.random.default_rng(330)
    n = 2000
    p = rng.random((n, 2))
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle, precision="mixed")
    check_derpos(gpu, ref, n)


def test_derpos_unsupported_cases(gpu_lib):
    rng = np.random.default_rng(340)
    p = rng.random((50, 2))
    g = PowerDiagram(p, np.full(50, 1e-3), radial_func="in_ball_w05")
    g.add_box_shape([0, 0], [1, 1])
    with pytest.raises(Exception, match="disc"):
        g.der_centroids_and_integrals_wrt_weight_and_positions()
    g = PowerDiagram(p, np.zeros(50))
    g.add_box_shape([0, 0], [0.5, 1])
    g.add_box_shape([0.5, 0], [1, 1])
    with pytest.raises(Exception, match="one-shape"):
        g.der_centroids_and_integrals_wrt_weight_and_positions()
    g = PowerDiagram(np.random.default_rng(1).random((20, 3)), np.zeros(20))
    g.add_box_shape([0, 0, 0], [1, 1, 1])
    with pytest.raises(Exception, match="2D"):
        g.der_centroids_and_integrals_wrt_weight_and_positions()


def test_derpos_full_size_properties(gpu_lib):
    # 1M clustered Diracs: v matches the centroids / masses of the evaluation,
    # rows hold their own diagonal block, and the mass rows' weight columns
    # are the Hessian's values
    c = workloads.config2(n=1_000_000)
    g = PowerDiagram(c["positions"], c["weights"])
    g.add_box_shape([0, 0], [1, 1])
    off, col, val, v = g.der_centroids_and_integrals_wrt_weight_and_positions()
    n = len(c["weights"])
    ctd, mas = g.centroids(with_masses=True)
    # the same cells integrated from their rebuilt vertices: equal to rounding
    assert_close(v[2::3], mas, 1e-10, mas.mean(), "masses")
    assert np.allclose(v.reshape(n, 3)[:, :2], ctd, rtol=0, atol=1e-12)
    ho, hc, hv, _ = g.der_integrals_wrt_weights()
    rows = np.repeat(np.arange(3 * n), np.diff(off))
    sel = (rows % 3 == 2) & (col % 3 == 2)
    assert np.array_equal(np.diff(ho), np.diff(off)[2::3] // 3)
    assert np.array_equal(col[sel] // 3, hc)
    np.testing.assert_allclose(val[sel], hv, rtol=1e-9, atol=1e-9 * np.abs(hv).mean())
    # a void cell (config 2 has some) holds only its diagonal block, NaN in
    # its centroid rows as in the reference
    void = np.flatnonzero(mas == 0)
    assert len(void) > 0
    assert np.all(np.diff(off)[3 * void] == 3)
