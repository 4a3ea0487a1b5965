"""The oracle's position derivatives (the compiled reference's
get_der_centroids_and_integrals_wrt_weight_and_positions) against central
finite differences of its own centroids and masses: pins the derivative
blocks before the GPU is compared with them.  CPU only."""
import numpy as np
import pytest


def dense(off, col, val, n3):
    m = np.zeros((n3, n3))
    for r in range(n3):
        m[r, col[off[r]:off[r + 1]]] += val[off[r]:off[r + 1]]
    return m


def values(ref_mod, p, w, translations=None, lo=(0.0, 0.0), hi=(1.0, 1.0)):
    r = ref_mod.RefPowerDiagram(p, w)
    r.add_box_shape(np.array(lo), np.array(hi))
    if translations is not None:
        r.set_translations(translations)
    c, m = r.centroids(with_masses=True)
    return np.concatenate([c, m[:, None]], 1).ravel(), r


@pytest.mark.parametrize("periodic", [False, True])
def test_der_pos_matches_finite_differences(ref_oracle, periodic):
    rng = np.random.default_rng(5 + periodic)
    n = 24
    p = rng.random((n, 2))
    w = rng.uniform(-2e-3, 2e-3, n)
    tr = None
    lo, hi = (0.0, 0.0), (1.0, 1.0)
    if periodic:
        tr = [(x, y) for x in (-1.0, 0.0, 1.0) for y in (-1.0, 0.0, 1.0) if x or y]
        lo, hi = (-1.0, -1.0), (2.0, 2.0)
    v0, r = values(ref_oracle, p, w, tr, lo, hi)
    off, col, val, v = r.der_centroids_and_integrals_wrt_weight_and_positions()
    assert np.allclose(v, v0, rtol=0, atol=1e-14)
    d = dense(off, col, val, 3 * n)
    h = 1e-6
    for j in range(0, n, 5):
        for e in range(3):
            pp, ww = p.copy(), w.copy()
            pm, wm = p.copy(), w.copy()
            if e < 2:
                pp[j, e] += h
                pm[j, e] -= h
            else:
                ww[j] += h
                wm[j] -= h
            fd = (values(ref_oracle, pp, ww, tr, lo, hi)[0] - values(ref_oracle, pm, wm, tr, lo, hi)[0]) / (2 * h)
            # centroid rows: the reference divides by the mass; mass rows as is
            np.testing.assert_allclose(d[:, 3 * j + e], fd, rtol=0, atol=1e-7 * max(1.0, np.abs(fd).max()),
                                       err_msg=f"column {3 * j + e}")
