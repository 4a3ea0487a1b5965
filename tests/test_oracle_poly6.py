"""Piecewise-quadratic image densities (ScaledImage with nb_coeffs = 6): the
C restatement (oracle/sdot_oracle.c) against the compiled reference on the
same inputs -- masses, centroids and Hessian -- so that the restatement is
pinned before it checks anything.  Runs on the CPU."""
import numpy as np
import pytest

from oracle.port import PortPowerDiagram
from tests.helpers import assert_close, compare_csr


def poly6_image(ny, nx, rng):
    """Coefficient planes (6, ny, nx) of a positive piecewise-quadratic density."""
    c = rng.uniform(-0.3, 0.3, (6, ny, nx))
    c[0] += 2.0
    return c


def run_pair(ref_mod, p, w, img):
    r = ref_mod.RefPowerDiagram(p, w)
    r.set_image_density(img)
    q = PortPowerDiagram(p, w)
    q.set_image_density(img, nb_coeffs=6)
    return r, q


@pytest.mark.parametrize("n,res", [(300, (8, 8)), (2000, (32, 48))])
def test_poly6_restatement_vs_reference(ref_oracle, n, res):
    rng = np.random.default_rng(600 + n)
    p = rng.random((n, 2))
    w = rng.uniform(-1e-4, 1e-4, n) / n
    img = poly6_image(res[0], res[1], rng)
    r, q = run_pair(ref_oracle, p, w, img)
    m_r, m_q = r.integrals(), q.integrals()
    mean = np.abs(m_r).mean()
    assert_close(m_q, m_r, 1e-12, mean, "masses")
    c_r, mc_r = r.centroids(with_masses=True)
    c_q, mc_q = q.centroids(with_masses=True)
    assert_close(mc_q, mc_r, 1e-12, mean, "centroid masses")
    assert_close(c_q, c_r, 1e-12, 1.0, "centroids")
    e, ro, rc, rv, rm = r.der_integrals_wrt_weights()
    _, qo, qc, qv, qm = q.der_integrals_wrt_weights()
    compare_csr((qo, qc, qv), (ro, rc, rv), 1e-11, np.abs(rv).mean())


def test_poly6_domain_measure(ref_oracle):
    # ScaledImage::measure with nb_coeffs = 6 (ScaledImage.tcc:45-62)
    rng = np.random.default_rng(606)
    img = poly6_image(5, 7, rng)
    r = ref_oracle.RefPowerDiagram(rng.random((10, 2)), np.zeros(10))
    r.set_image_density(img)
    q = PortPowerDiagram(rng.random((10, 2)))
    q.set_image_density(img, nb_coeffs=6)
    assert abs(q.domain_measure() - r.domain_measure()) <= 1e-13 * abs(r.domain_measure())
