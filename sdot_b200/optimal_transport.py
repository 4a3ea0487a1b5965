"""``OptimalTransport``: semi-discrete optimal transport by Newton on the weights.

Mirrors the Python surface the reference's example script uses
(weights.py:1-15): ``OptimalTransport(positions)``, the ``verbosity``
attribute, ``adjust_weights()``, ``get_positions()`` and ``get_weights()``.
The solve is OptimalTransportSolver::solve (OptimalTransportSolver.tcc:27-119)
on the device: fused cell evaluation, CSR Hessian with the reference's gauge
fix, Jacobi-preconditioned conjugate gradients in place of the sparse
Cholesky of EigenSolver::solve (EigenSolver.cpp:9-41), and a damped step.

Defaults when the caller gives none: the unit box [0, 1]^dim with density 1
as the domain, equal target masses (domain measure / n) and zero starting
weights (the Voronoi diagram, where no cell of distinct points is empty).
"""
import numpy as np

from .power_diagram import PowerDiagram


class OptimalTransport:
    def __init__(self, positions=None, masses=None, weights=None, domain=None, radial_func="unit",
                 precision="fp64", rel_mass_tol=1e-10, verbosity=0):
        self.verbosity = verbosity
        self.rel_mass_tol = rel_mass_tol
        self.radial_func = radial_func
        self.precision = precision
        self._positions = None
        self._weights = None
        self._masses = None
        self._domain = domain
        self.pd = None
        self.last_report = None
        if positions is not None:
            self.set_positions(positions)
        if weights is not None:
            self.set_weights(weights)
        if masses is not None:
            self.set_masses(masses)

    # ------------------------------------------------------------ inputs
    def set_positions(self, positions):
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64))
        if p.ndim != 2:
            raise ValueError("positions must have shape (n, dim)")
        self._positions = p
        if self._weights is None or self._weights.shape[0] != p.shape[0]:
            self._weights = np.zeros(p.shape[0])
        self.pd = None

    def get_positions(self):
        return self._positions

    def set_weights(self, weights):
        self._weights = np.ascontiguousarray(np.asarray(weights, dtype=np.float64)).copy()
        if self.pd is not None:
            self.pd.set_weights(self._weights)

    def get_weights(self):
        return self._weights

    def set_masses(self, masses):
        self._masses = np.ascontiguousarray(np.asarray(masses, dtype=np.float64))

    def get_masses(self):
        return self._masses

    def set_domain(self, domain):
        """domain: a callable ``f(power_diagram)`` that adds the shapes (or the
        image density) to a PowerDiagram, e.g. ``lambda pd: pd.add_box_shape(a, b)``."""
        self._domain = domain
        self.pd = None

    # ------------------------------------------------------------- solve
    def _diagram(self):
        if self.pd is None:
            if self._positions is None:
                raise ValueError("no positions")
            dim = self._positions.shape[1]
            pd = PowerDiagram(self._positions, self._weights, precision=self.precision,
                              radial_func=self.radial_func)
            if self._domain is None:
                pd.add_box_shape(np.zeros(dim), np.ones(dim))
            else:
                self._domain(pd)
            self.pd = pd
        return self.pd

    def adjust_weights(self, initial_weights=None, damping=True, max_iter=150):
        """Solves for the weights that give every cell its target mass; the
        relative mass error at the end is at most ``rel_mass_tol``."""
        if initial_weights is not None:
            self.set_weights(initial_weights)
        pd = self._diagram()
        n = self._positions.shape[0]
        masses = self._masses
        if masses is None:
            masses = np.full(n, pd.domain_measure() / n)
        rep = pd.solve_weights(masses, rel_mass_tol=self.rel_mass_tol, max_iter=max_iter, damping=damping,
                               verbosity=self.verbosity)
        self._weights = pd.get_weights()
        self.last_report = rep
        return rep

    def get_centroids(self):
        return self._diagram().centroids()

    def get_integrals(self):
        return self._diagram().integrals()
