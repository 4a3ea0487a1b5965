"""The tree build and the weight refresh replay CUDA graphs captured on the
first build of a context (keyed on the Dirac count, the input buffers and the
leaf size): a context that changes its Dirac count, its positions or only its
weights between evaluations gives bitwise the results of a fresh context."""
import numpy as np
import pytest

from sdot_b200.power_diagram import PowerDiagram

pytestmark = pytest.mark.gpu


def fresh(p, w):
    g = PowerDiagram(p, w)
    g.add_box_shape([0, 0], [1, 1])
    return g.integrals(), g.der_integrals_wrt_weights()


def same(a, b):
    assert np.array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)


def test_reused_context_matches_fresh(gpu_lib):
    rng = np.random.default_rng(900)
    sizes = [20_000, 7_000, 20_000, 150_000, 20_000]
    probs = [(rng.random((n, 2)), rng.uniform(-1e-6, 1e-6, n)) for n in sizes]
    g = PowerDiagram(probs[0][0], probs[0][1])
    g.add_box_shape([0, 0], [1, 1])
    for p, w in probs:
        g.set_positions_and_weights(p, w)
        got = (g.integrals(), g.der_integrals_wrt_weights())
        same(got, fresh(p, w))
        # weights alone: the refresh graph
        w2 = w + rng.uniform(-1e-7, 1e-7, len(w))
        g.set_weights(w2)
        got = (g.integrals(), g.der_integrals_wrt_weights())
        same(got, fresh(p, w2))
