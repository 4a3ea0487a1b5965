"""Pins the C restatement oracle (oracle/sdot_oracle.c) to the known answers
of the reference's own tests.  CPU only.

Sources (reference tree): tests/test_ConvexPolyhedron2.cpp and
tests/test_scaled_image.cpp; each case below names the TEST_CASE/SECTION it
restates and uses the reference's tolerance.
"""
import math

import numpy as np
import pytest

from oracle.port import Poly, PortPowerDiagram

SQ = math.sqrt


def unit(v):
    v = np.asarray(v, dtype=float)
    return v / (np.linalg.norm(v) + 1e-40)


def test_diam():
    # TEST_CASE( "diam" ) test_ConvexPolyhedron2.cpp:16-49: 8 cuts -> 3.313708499
    cs = Poly.box([-10, -10], [10, 10])
    for y in (-1, 0, 1):
        for x in (-1, 0, 1):
            if x or y:
                n = unit([x, y])
                cs.plane_cut(n, n)
    assert abs(cs.measure() - 3.313708499) < 1e-4


def test_only_sphere():
    # TEST_CASE( "only_sphere" ) :81-95
    cs = Poly.box([-10, -10], [10, 10])
    cs.ball_cut([1, 0], 1)
    assert abs(cs.measure() - math.pi) < 1e-6


@pytest.mark.parametrize("cuts,nb_points", [
    # TEST_CASE( "cases_1" ) :114-154 (vertex counts after plane + ball cuts)
    ([((SQ(0.5), 0.0), (1, 0)), ((SQ(0.6), 0.1), (1, 0))], 2),
    ([((SQ(0.5), 0.0), (1, 0)), ((0.0, 0.0), (0, 1))], 3),
    ([((SQ(0.5), 0.0), (1, 0)), ((0.0, 0.0), (0, -1))], 3),
    ([((SQ(0.5), 0.0), (1, 0)), ((SQ(0.2), 0.1), (1, 0))], 2),
    ([((SQ(0.5), 0.0), (1, 0)), ((SQ(0.6), 0.1), (-1, 0))], 0),
    ([((0.7, 0.0), (1, 0)), ((0.0, 0.7), (0, 1)), ((-0.7, 0.0), (-1, 0)), ((0.0, -0.7), (0, -1))], 4),
])
def test_cases_1(cuts, nb_points):
    for r in range(3):
        off = np.array([r % 3 * 2.5, -(r // 3) * 2.5])
        icp = Poly.box(off - 10, off + 10)
        for p, n in cuts:
            icp.plane_cut(off + np.array(p), unit(n))
        icp.ball_cut(off, 1)
        assert icp.nb_points() == nb_points


def _kv(cuts, expect_area, expect_nb=None):
    icp = Poly.box([-10, -10], [10, 10])
    for p, n in cuts:
        icp.plane_cut(p, n)
    icp.ball_cut([0.0, 0.0], 1)
    if expect_nb is not None:
        assert icp.nb_points() == expect_nb
    assert abs(icp.measure() - expect_area) < 1e-7


def test_known_values():
    # TEST_CASE( "known_values" ) :156-263, tolerance 1e-7
    _kv([], math.pi)                                                               # full
    _kv([((1.0, 0.0), (1, 0))], math.pi, 0)                                        # no modification
    _kv([((1.0, 0.0), (-1, 0))], 0.0, 0)                                           # full removal
    for i in range(12):                                                            # 1 intersection, middle
        a = 2 * math.pi * i / 12
        _kv([((0.0, 0.0), (math.cos(a), math.sin(a)))], math.pi / 2, 2)
    _kv([((SQ(0.5), 0.0), (1, 0))], 3 * math.pi / 4 + 0.5, 2)                      # at the right
    _kv([((-SQ(0.5), 0.0), (1, 0))], math.pi / 4 - 0.5, 2)                         # at the left
    _kv([((-SQ(0.5), 0.0), (-1, 0)), ((SQ(0.5), 0.0), (1, 0))], math.pi / 2 + 1.0, 4)
    _kv([((-SQ(0.5), 0.0), (-1, 0)), ((SQ(0.5), 0.0), (-1, 0))], math.pi / 4 - 0.5, 2)
    _kv([((-SQ(0.5), 0.0), (-1, 0)), ((-0.9, 0.0), (-1, 0))], 3 * math.pi / 4 + 0.5, 2)
    _kv([((0.0, 0.0), (-1, 0)), ((0.0, 0.0), (0, 1))], math.pi / 4, 3)
    _kv([((0.0, 0.0), (-1, 0)), ((0.0, 0.0), (0, -1))], math.pi / 4, 3)
    _kv([((0.2, 0.0), (1, 0)), ((0.0, 0.2), (0, 1)), ((-0.2, 0.0), (-1, 0)), ((0.0, -0.2), (0, -1))], 0.16, 4)
    _kv([((0.0, -1.0), (1, 0)), ((0.0, -1.0), tuple(unit([1, 1])))], math.pi / 4 - 0.5)   # degeneracies


def _ctd(cuts, r):
    icp = Poly.box([-10, -10], [10, 10])
    for p, n in cuts:
        icp.plane_cut(p, n)
    icp.ball_cut([0.0, 0.0], r)
    return icp.centroid()


def test_centroid():
    # TEST_CASE( "centroid" ) :265-311
    c = _ctd([], 1)
    assert abs(c[0]) < 1e-6 and abs(c[1]) < 1e-6
    c = _ctd([((0.0, 0.0), (1, 0))], 1)
    assert abs(-0.424413 - c[0]) < 1e-4 and abs(c[1]) < 1e-4
    c = _ctd([((0.0, 0.0), (1, 0)), ((0.0, 0.0), (0, 1))], 1)
    assert abs(-0.424413 - c[0]) < 1e-4 and abs(-0.424413 - c[1]) < 1e-4
    c = _ctd([((0.0, 0.0), (1, 0)), ((0.0, 0.0), (0, 1))], 0.5)
    assert abs(-0.212207 - c[0]) < 1e-4 and abs(-0.212207 - c[1]) < 1e-4
    c = _ctd([((1, 0), (1, 0)), ((0, 1), (0, 1)), ((-1, 0), (-1, 0)), ((0, -1), (0, -1))], 10)
    assert abs(c[0]) < 1e-6 and abs(c[1]) < 1e-6


def test_integration_only_lines_unit():
    # TEST_CASE( "integration_only_lines" ) :313-339, Unit parts
    icp = Poly.box([0, 0], [2, 1])
    assert abs(icp.measure() - 2.0) < 1e-5
    c = icp.centroid()
    assert abs(c[0] - 1.0) < 1e-5 and abs(c[1] - 0.5) < 1e-5
    scp = Poly.box([0, 0], [3, 3])
    scp.ball_cut([0, 0], 2)
    assert abs(scp.measure() - math.pi) < 1e-5
    sph = Poly.box([0, 0], [8, 8])
    sph.ball_cut([4, 4], 2)
    assert abs(sph.measure() - 4 * math.pi) < 1e-5


def test_scaled_image_1():
    # TEST_CASE( "scaled image 1" ) test_scaled_image.cpp:56-70: 1 pixel, nb_coeffs 6 -> 11
    pd = PortPowerDiagram(np.array([[0.5, 0.5]]), np.array([1.0]))
    pd.set_image_density(np.array([2, 3, 4, 5, 6, 7], dtype=float).reshape(6, 1, 1), nb_coeffs=6)
    assert abs(pd.integrals()[0] - 11) < 1e-6


def test_scaled_image_2():
    # TEST_CASE( "scaled image 2" ) test_scaled_image.cpp:72-92
    pd = PortPowerDiagram(np.array([[0.25, 0.25], [0.75, 0.25], [0.25, 0.75], [0.75, 0.75]]), np.ones(4))
    pd.set_image_density(np.array([2, 3, 4, 5, 6, 7], dtype=float).reshape(6, 1, 1), nb_coeffs=6)
    m = pd.integrals()
    for got, exp in zip(m, [1.28125, 2.46875, 2.84375, 4.40625]):
        assert abs(got - exp) < 1e-6


def test_uniform_areas_sum_to_one():
    rng = np.random.default_rng(11)
    n = 2000
    pd = PortPowerDiagram(rng.random((n, 2)))
    pd.add_box_shape([0, 0], [1, 1])
    m = pd.integrals()
    assert abs(m.sum() - 1) < 1e-12
    assert (m > 0).all()
    off, ids = pd.neighbors()
    # symmetric adjacency on a non-degenerate Voronoi diagram
    nbs = [set(int(j) for j in ids[off[i]:off[i + 1]] if j >= 0) for i in range(n)]
    assert all(i in nbs[j] for i in range(n) for j in nbs[i])


def test_hessian_rows_sum_to_zero():
    # Unit density on a single box: each row of d mass / d w sums to zero
    rng = np.random.default_rng(12)
    n = 1500
    pd = PortPowerDiagram(rng.random((n, 2)), rng.uniform(-1e-4, 1e-4, n))
    pd.add_box_shape([0, 0], [1, 1])
    err, off, col, val, m = pd.der_integrals_wrt_weights()
    sums = np.add.reduceat(val, off[:-1])
    assert np.abs(sums).max() < 1e-9 * np.abs(val).max()


def test_hessian_matches_finite_differences():
    # derivative-consistency pattern of tests/test_der_pos.cpp:17-101, restated
    # in FP64 with central differences
    rng = np.random.default_rng(13)
    n = 60
    p = rng.random((n, 2))
    w = rng.uniform(-1e-3, 1e-3, n)
    pd = PortPowerDiagram(p, w)
    pd.add_box_shape([0, 0], [1, 1])
    err, off, col, val, m = pd.der_integrals_wrt_weights()
    H = np.zeros((n, n))
    for i in range(n):
        H[i, col[off[i]:off[i + 1]]] = val[off[i]:off[i + 1]]
    eps = 1e-7
    for j in range(0, n, 7):
        wp, wm = w.copy(), w.copy()
        wp[j] += eps
        wm[j] -= eps
        a = PortPowerDiagram(p, wp)
        a.add_box_shape([0, 0], [1, 1])
        b = PortPowerDiagram(p, wm)
        b.add_box_shape([0, 0], [1, 1])
        fd = (a.integrals() - b.integrals()) / (2 * eps)
        assert np.abs(fd - H[:, j]).max() < 1e-5 * np.abs(H).max()
