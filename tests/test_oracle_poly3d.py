"""The 3D multilinear-density oracle (oracle/poly3d.py): pinned against the
compiled reference at density 1 (volumes, centroids, Hessian rows), and its
polynomial integrals against closed forms."""
import numpy as np

from oracle import poly3d

C4 = np.array([1.0, 0, 0, 0, 0, 0, 0, 0.3])


def _csr_to_dict(off, col, val):
    H = {}
    for i in range(len(off) - 1):
        for k in range(off[i], off[i + 1]):
            H[(i, int(col[k]))] = H.get((i, int(col[k])), 0.0) + val[k]
    return H


def test_simplex_moments_known_values():
    # unit tetrahedron (0, e1, e2, e3): int x = 1/24, int xyz = 1/720, int x^2 = 1/60
    V = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]], float)
    vol = 1.0 / 6
    assert np.isclose(vol * poly3d.simplex_monomial(V, [0])[0], 1 / 24, rtol=1e-14)
    assert np.isclose(vol * poly3d.simplex_monomial(V, [0, 1, 2])[0], 1 / 720, rtol=1e-14)
    assert np.isclose(vol * poly3d.simplex_monomial(V, [0, 0])[0], 1 / 60, rtol=1e-14)
    assert np.isclose(vol * poly3d.simplex_monomial(V, [0, 0, 1, 2])[0], 2 / 5040, rtol=1e-14)
    # unit right triangle in the z = 0 plane: int x y dA = 1/24
    T = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], float)
    assert np.isclose(0.5 * poly3d.simplex_monomial(T, [0, 1])[0], 1 / 24, rtol=1e-14)


def test_single_cell_is_the_box():
    m, c, H = poly3d.integrate(np.array([[0.3, 0.6, 0.2]]), poly=C4)
    assert np.isclose(m[0], 1 + 0.3 / 8, rtol=1e-13)
    # int x (1 + 0.3 xyz) = 1/2 + 0.3/12 over the unit cube
    assert np.allclose(c[0], (0.5 + 0.3 / 12) / (1 + 0.3 / 8), rtol=1e-13)
    assert H[(0, 0)] == 0.0


def test_two_cells_split_at_a_plane():
    # Diracs mirrored about x = 0.4: cells [0, 0.4] and [0.4, 1] in x
    p = np.array([[0.3, 0.5, 0.5], [0.5, 0.5, 0.5]])
    m, c, H = poly3d.integrate(p, poly=C4)
    a = 0.4
    assert np.isclose(m[0], a + 0.3 * (a * a / 2) / 4, rtol=1e-13)
    assert np.isclose(m[1], (1 - a) + 0.3 * ((1 - a * a) / 2) / 4, rtol=1e-13)
    # shared face x = 0.4: int (1 + 0.3 * 0.4 y z) dy dz = 1 + 0.3 * 0.4 / 4, over |x_0 - x_1| = 0.2
    f = 1 + 0.3 * a / 4
    assert np.isclose(H[(0, 1)], -0.5 * f / 0.2, rtol=1e-13)
    assert np.isclose(H[(0, 0)], 0.5 * f / 0.2, rtol=1e-13)


def test_masses_sum_to_the_box_integral():
    rng = np.random.default_rng(7)
    p = rng.random((120, 3))
    w = rng.uniform(-1e-3, 1e-3, 120)
    m, c, H = poly3d.integrate(p, w, poly=C4)
    assert np.isclose(m.sum(), poly3d.box_integral(C4), rtol=1e-13)
    # rows of the Hessian sum to zero (no domain faces in the rows)
    rows = np.zeros(120)
    for (i, j), v in H.items():
        rows[i] += v
    assert np.max(np.abs(rows)) < 1e-11 * max(abs(v) for v in H.values())


def test_density_one_matches_the_compiled_reference(ref_oracle):
    rng = np.random.default_rng(11)
    n = 300
    p = rng.random((n, 3))
    w = rng.uniform(-2e-3, 2e-3, n)
    m, c, H = poly3d.integrate(p, w)
    r = ref_oracle.RefPowerDiagram(p, w, dim=3)
    r.add_box_shape(np.zeros(3), np.ones(3))
    rm = r.integrals()
    rc = r.centroids()
    err, off, col, val, _ = r.der_integrals_wrt_weights()
    assert err == 0
    np.testing.assert_allclose(m, rm, rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(c, rc, rtol=1e-10, atol=1e-13)
    RH = _csr_to_dict(off, col, val)
    scale = max(abs(v) for v in RH.values())
    keys = set(RH) | set(H)
    worst = max(abs(RH.get(k, 0.0) - H.get(k, 0.0)) for k in keys)
    assert worst < 1e-10 * scale, worst


def test_convex_shape_planes_vs_reference(ref_oracle):
    # the half-space extension of the qhull oracle (a convex shape: its box
    # cut by planes) against the compiled reference on one convex shape
    from oracle import poly3d

    rng = np.random.default_rng(307)
    p = rng.random((2000, 3))
    p = p[p.sum(1) < 2.15][:300]
    n = len(p)
    pts, nrm = [], []
    for d in range(3):
        for side in (0.0, 1.0):
            q = [0.5, 0.5, 0.5]
            q[d] = side
            v = [0.0, 0.0, 0.0]
            v[d] = 1.0 if side else -1.0
            pts.append(q)
            nrm.append(v)
    pts.append([2.2 / 3] * 3)
    nrm.append([1.0, 1.0, 1.0])
    pts, nrm = np.array(pts), np.array(nrm)
    r = ref_oracle.RefPowerDiagram(p, np.zeros(n))
    r.add_convex_polyhedron_shape(pts, nrm)
    m_r = r.integrals()
    c_r = r.centroids()
    nn = nrm / np.linalg.norm(nrm, axis=1)[:, None]
    planes = np.hstack([nn, np.sum(nn * pts, 1)[:, None]])
    lo, hi = pts.min(0), pts.max(0)
    m_o, c_o, H_o = poly3d.integrate(p, lo=lo - (hi - lo), hi=hi + (hi - lo), planes=planes)
    np.testing.assert_allclose(m_o, m_r, rtol=1e-11, atol=1e-12 * m_r.mean())
    np.testing.assert_allclose(c_o, c_r, rtol=1e-11, atol=1e-12)
    _, off, col, val, _ = r.der_integrals_wrt_weights()
    H_r = {}
    for i in range(n):
        for k in range(off[i], off[i + 1]):
            H_r[(i, int(col[k]))] = H_r.get((i, int(col[k])), 0.0) + val[k]
    scale = max(abs(v) for v in H_r.values())
    keys = set(H_r) | set(H_o)
    assert max(abs(H_r.get(k, 0.0) - H_o.get(k, 0.0)) for k in keys) < 1e-10 * scale
