"""The Newton oracle (oracle/newton.py) on known answers, CPU only."""
import numpy as np
import pytest

from oracle import newton, port


def two_cells(target0):
    # Diracs at x = 0.25 and x = 0.75 in the unit box: the power bisector is the
    # vertical line x = 0.5 + w0 - w1, so the left cell has mass 0.5 + w0 - w1
    p = np.array([[0.25, 0.5], [0.75, 0.5]])
    pd = port.PortPowerDiagram(p, np.zeros(2))
    pd.add_box_shape([0.0, 0.0], [1.0, 1.0])
    return pd, np.array([target0, 1.0 - target0])


@pytest.mark.parametrize("rule", ["damped", "reference"])
def test_two_cells_known_weights(rule):
    pd, t = two_cells(0.3)
    w, rep = newton.solve(pd, t, np.zeros(2), tol=1e-14, rule=rule)
    assert rep["converged"]
    assert abs((w[0] - w[1]) - (-0.2)) < 1e-14
    # the gauge fix (H[0][0] doubled) keeps the weight of Dirac 0 at its start
    assert abs(w[0]) < 1e-14


def test_damped_keeps_cells_non_empty():
    # a far target: the full step empties a cell, the damped rule halves it
    pd, t = two_cells(0.02)
    w, rep = newton.solve(pd, t, np.zeros(2), tol=1e-13, rule="damped")
    assert rep["converged"]
    assert abs((w[0] - w[1]) - (-0.48)) < 1e-13


def test_uniform_grid_is_fixed_point():
    # a regular grid already has equal masses: zero iterations
    g = (np.arange(8) + 0.5) / 8
    p = np.stack(np.meshgrid(g, g), -1).reshape(-1, 2)
    pd = port.PortPowerDiagram(p, np.zeros(64))
    pd.add_box_shape([0.0, 0.0], [1.0, 1.0])
    w, rep = newton.solve(pd, np.full(64, 1 / 64), np.zeros(64), tol=1e-12)
    assert rep["converged"] and rep["iterations"] == 0
