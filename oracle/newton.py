"""Test infrastructure only: the Newton oracle on the weights.

Restates OptimalTransportSolver::solve (src/sdot/Solvers/OptimalTransportSolver.tcc:27-119)
in Python over any CPU power-diagram oracle that returns the reference CSR
(oracle/ref.py RefPowerDiagram, or oracle/port.py PortPowerDiagram):

  * per iteration: masses + CSR Hessian at the current weights
    (get_der_integrals_wrt_weights, .tcc:59);
  * gauge fix: the first CSR value (entry (0, 0)) doubled when there is no
    ball cut (.tcc:62-63);
  * rule "reference": on an empty cell, w = 0.9 w_old + 0.1 w and retry
    (.tcc:72-79); otherwise the full step w -= dw (.tcc:106-109);
  * rule "damped": the Kitagawa-Merigot-Thibert step halving (tau halves
    until min mass >= eps0 and |m - t| <= (1 - tau / 2) |m_0 - t|, with
    eps0 = min(min target, min starting mass) / 2; a step that reaches the
    tolerance is always taken), the rule the device solver uses by default;
  * the linear solve is scipy.sparse.linalg.spsolve (a direct solve, as the
    reference's SimplicialCholesky, EigenSolver.cpp:9-41, whose Eigen
    dependency is absent here);
  * it stops on the relative mass error max_i |m_i - t_i| / t_i <= tol
    instead of the reference's max |dw| < 1e-6 (.tcc:111-112).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _stats(m, t):
    d = m - t
    return float(np.max(np.abs(d) / t)), float(m.min()), float(np.dot(d, d))


def solve(diagram, target, w0, tol=1e-10, max_iter=150, rule="damped", ball_cut=False, trace=None):
    """diagram: an oracle power diagram (set_weights / der_integrals_wrt_weights);
    w0: starting weights.  Returns (weights, report).  trace (a list, may be
    None) receives the relative mass error at the start of each iteration."""
    t = np.asarray(target, dtype=np.float64)
    n = t.shape[0]
    w = np.array(w0, dtype=np.float64)

    def der(wv):
        diagram.set_weights(wv)
        err, off, col, val, m = diagram.der_integrals_wrt_weights()
        return off, col, val.copy(), m

    off, col, val, m = der(w)
    e = _stats(m, t)
    w_old = w.copy()
    eps0 = 0.5 * min(t.min(), e[1])
    rep = {"iterations": 0, "evaluations": 1}
    for it in range(max_iter + 1):
        rep["max_rel_mass_error"], rep["min_mass"] = e[0], e[1]
        if trace is not None:
            trace.append(e[0])
        if e[0] <= tol:
            rep["converged"] = True
            return w, rep
        if it >= max_iter:
            break
        rep["iterations"] = it + 1
        if rule == "reference" and not e[1] > 0:
            w = 0.9 * w_old + 0.1 * w
            off, col, val, m = der(w)
            rep["evaluations"] += 1
            e = _stats(m, t)
            continue
        w_old = w.copy()
        if len(val) and not ball_cut:
            val[0] *= 2
        H = sp.csr_matrix((val, col, off), shape=(n, n))
        dw = spla.spsolve(H.tocsc(), m - t)
        tau = 1.0
        for _ in range(41):
            w = w_old - tau * dw
            off2, col2, val2, m2 = der(w)
            rep["evaluations"] += 1
            e2 = _stats(m2, t)
            if rule == "reference" or e2[0] <= tol or (e2[1] >= eps0 and
                                                        np.sqrt(e2[2]) <= (1 - 0.5 * tau) * np.sqrt(e[2])):
                break
            tau *= 0.5
        else:
            w = w_old
            break
        off, col, val, m, e = off2, col2, val2, m2, e2
    rep["converged"] = False
    return w, rep
