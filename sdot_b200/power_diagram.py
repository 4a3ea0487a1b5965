"""Python facade of the power-diagram path, mirroring sdot's PowerDiagram surface.

Reference surface (the pybind11 sources are not part of the reference tree;
the names come from its README and its example script):
  * ``PowerDiagram`` with cumulative ``add_..._shape`` domain calls
    (README.md:7-9);
  * ``OptimalTransport(positions)``, ``verbosity``, ``adjust_weights()``,
    ``get_positions()``, ``get_weights()`` (weights.py:1-15);
  * images are given as numpy arrays whose last axis is x
    (ScaledImage.h:12: ``sizes[d] = img.shape(img.ndim() - 1 - d)``).

Every numeric result comes from libsdot_b200.so (CUDA, sm_100a).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import SDOT_DEVICE, SDOT_FP64, SDOT_HOST, SDOT_MIXED, SdotError


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if shape is not None:
        a = a.reshape(shape)
    return a


class PowerDiagram:
    """Laguerre (power) diagram of weighted Diracs clipped to a domain.

    positions: (n, dim) array; weights: (n,) array (default zeros).
    precision: "fp64" or "mixed".  radial_func: "unit" (FunctionEnum::Unit)
    or "in_ball_w05" (FunctionEnum::InBallW05: cells clipped by the disc of
    radius sqrt(w_i)).
    """

    def __init__(self, positions=None, weights=None, dim=None, precision="fp64", radial_func="unit",
                 max_diracs_per_cell=11, device=-1):
        self._lib = _lib.load()
        if dim is None:
            dim = np.asarray(positions).shape[1] if positions is not None else 2
        self.dim = int(dim)
        prec = {"fp64": SDOT_FP64, "mixed": SDOT_MIXED}[precision]
        opt = _lib.SdotOptions(int(max_diracs_per_cell), None, int(device))
        self._ctx = self._lib.sdot_create(self.dim, prec, ctypes.byref(opt))
        if not self._ctx:
            raise SdotError(_lib.SDOT_CUDA_ERROR, "sdot_create failed (no CUDA device?)")
        self.precision = precision
        self._positions = None
        self._weights = None
        self.set_radial_func(radial_func)
        if positions is not None:
            self.set_positions_and_weights(positions, weights)

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx:
            self._lib.sdot_destroy(ctx)
            self._ctx = None

    # ------------------------------------------------------------------ misc
    def _check(self, st, allow=()):
        if st != _lib.SDOT_OK and st not in allow:
            raise SdotError(st, self._lib.sdot_last_error(self._ctx).decode())
        return st

    # -------------------------------------------------------------- diracs
    def set_positions_and_weights(self, positions, weights=None):
        p = _f64(positions)
        if p.ndim != 2 or p.shape[1] != self.dim:
            raise ValueError(f"positions must have shape (n, {self.dim})")
        n = p.shape[0]
        w = np.zeros(n) if weights is None else _f64(weights, (n,))
        self._positions, self._weights = p, w
        self._check(self._lib.sdot_set_diracs(self._ctx, _ptr(p), _ptr(w), n, SDOT_HOST))

    def set_weights(self, weights):
        w = _f64(weights, (self._positions.shape[0],))
        self._weights = w
        self._check(self._lib.sdot_set_weights(self._ctx, _ptr(w), SDOT_HOST))

    def get_positions(self):
        return self._positions

    def get_weights(self):
        return self._weights

    @property
    def nb_diracs(self):
        return 0 if self._positions is None else self._positions.shape[0]

    # -------------------------------------------------------------- domain
    def add_box_shape(self, p0, p1, coeff=1.0):
        a, b = _f64(p0), _f64(p1)
        self._check(self._lib.sdot_add_box_shape(self._ctx, _ptr(a), _ptr(b), float(coeff)))

    def add_convex_polyhedron_shape(self, points, normals, coeff=1.0):
        pts = _f64(points, (-1, self.dim))
        nrm = _f64(normals, pts.shape)
        self._check(self._lib.sdot_add_convex_polyhedron_shape(self._ctx, _ptr(pts), _ptr(nrm), pts.shape[0],
                                                               float(coeff)))

    def add_simplex_shape(self, points, coeff=1.0):
        pts = _f64(points, (self.dim + 1, self.dim))
        self._check(self._lib.sdot_add_simplex_shape(self._ctx, _ptr(pts), float(coeff)))

    def set_image_density(self, image, min_pt=None, max_pt=None, nb_coeffs=None):
        """image: numpy array of shape (ny, nx) (last axis is x) for a
        piecewise-constant density, or (6, ny, nx) for a piecewise-quadratic
        one (nb_coeffs = 6: per pixel c0 + c1 x + c2 y + c3 x^2 + c4 x y +
        c5 y^2 in absolute coordinates, plane k holding c_k; the layout of
        ScaledImage's data)."""
        img = _f64(image)
        if nb_coeffs is None:
            nb_coeffs = img.shape[0] if img.ndim == self.dim + 1 else 1
        spatial = img.shape[1:] if nb_coeffs > 1 else img.shape
        sizes = np.array(spatial[::-1], dtype=np.int64)
        mn = _f64(min_pt if min_pt is not None else np.zeros(self.dim))
        mx = _f64(max_pt if max_pt is not None else np.ones(self.dim))
        self._check(self._lib.sdot_set_image_density(self._ctx, _ptr(mn), _ptr(mx), _ptr(img), _ptr(sizes),
                                                     int(nb_coeffs)))

    def set_polynomial_density(self, coeffs):
        """3D: multiplies the domain's density by c0 + c1 x + c2 y + c3 z +
        c4 xy + c5 xz + c6 yz + c7 xyz (8 coefficients; 1 coefficient
        restores a constant factor).  Integrated exactly."""
        c = _f64(coeffs).reshape(-1)
        self._check(self._lib.sdot_set_polynomial_density(self._ctx, _ptr(c), int(c.size)))

    def clear_domain(self):
        self._check(self._lib.sdot_clear_domain(self._ctx))

    def normalize_domain(self):
        self._check(self._lib.sdot_normalize_domain(self._ctx))

    def domain_measure(self):
        out = np.zeros(1)
        self._check(self._lib.sdot_domain_measure(self._ctx, _ptr(out)))
        return float(out[0])

    def set_translations(self, translations):
        """Periodic copies of the Diracs (SpZGrid::translations): a list of
        translation vectors; each cell is also cut by the images of every
        Dirac under them.  An empty list removes them."""
        t = _f64(np.asarray(translations, dtype=np.float64).reshape(-1, self.dim))
        self._check(self._lib.sdot_set_translations(self._ctx, _ptr(t) if t.size else None, int(t.shape[0])))

    def set_radial_func(self, name):
        on = {"unit": 0, "in_ball_w05": 1}[name]
        self.radial_func = name
        self._check(self._lib.sdot_set_ball_cut(self._ctx, on))

    # ------------------------------------------------------------- results
    def integrals(self):
        out = np.empty(self.nb_diracs)
        self._check(self._lib.sdot_get_integrals(self._ctx, _ptr(out), SDOT_HOST))
        return out

    def centroids(self, with_masses=False):
        c = np.empty((self.nb_diracs, self.dim))
        m = np.empty(self.nb_diracs)
        self._check(self._lib.sdot_get_centroids(self._ctx, _ptr(c), _ptr(m), SDOT_HOST))
        return (c, m) if with_masses else c

    def der_integrals_wrt_weights(self, stop_if_void=False):
        """Returns (offsets, columns, values, masses): the CSR Hessian
        d mass_i / d w_j and the masses, like get_der_integrals_wrt_weights."""
        nnz = ctypes.c_int64(0)
        self._check(self._lib.sdot_get_der_integrals_wrt_weights(self._ctx, None, None, None, None,
                                                                 ctypes.byref(nnz), int(stop_if_void), SDOT_HOST))
        n = self.nb_diracs
        offsets = np.empty(n + 1, dtype=np.int64)
        columns = np.empty(nnz.value, dtype=np.int64)
        values = np.empty(nnz.value)
        masses = np.empty(n)
        st = self._lib.sdot_get_der_integrals_wrt_weights(self._ctx, _ptr(offsets), _ptr(columns), _ptr(values),
                                                          _ptr(masses), ctypes.byref(nnz), int(stop_if_void),
                                                          SDOT_HOST)
        self._check(st, allow=(_lib.SDOT_VOID_CELL,))
        if st == _lib.SDOT_VOID_CELL:
            raise SdotError(st, "void cell")
        return offsets, columns, values, masses

    def neighbors(self):
        """Per cell, the cut ids of its final boundary in vertex order
        (Dirac index, -1 domain edge, -2 disc arc), as CSR (offsets, ids)."""
        cnt = ctypes.c_int64(0)
        self._check(self._lib.sdot_get_neighbors(self._ctx, None, None, ctypes.byref(cnt), SDOT_HOST))
        offsets = np.empty(self.nb_diracs + 1, dtype=np.int64)
        ids = np.empty(cnt.value, dtype=np.int64)
        self._check(self._lib.sdot_get_neighbors(self._ctx, _ptr(offsets), _ptr(ids), ctypes.byref(cnt),
                                                 SDOT_HOST))
        return offsets, ids

    def der_centroids_and_integrals_wrt_weight_and_positions(self):
        """get_der_centroids_and_integrals_wrt_weight_and_positions (2D): CSR
        (offsets, columns, values) over 3 n rows and columns -- row 3 i + d is
        output d (centroid x, centroid y, mass) of cell i, column 3 j + e input
        e (x, y, weight) of Dirac j -- and the values (3 n: centroid, mass)."""
        fn = self._lib.sdot_get_der_centroids_and_integrals_wrt_weight_and_positions
        nnz = ctypes.c_int64(0)
        self._check(fn(self._ctx, None, None, None, None, ctypes.byref(nnz), SDOT_HOST))
        n3 = 3 * self.nb_diracs
        off = np.empty(n3 + 1, dtype=np.int64)
        col = np.empty(nnz.value, dtype=np.int64)
        val = np.empty(nnz.value)
        v = np.empty(n3)
        self._check(fn(self._ctx, _ptr(off), _ptr(col), _ptr(val), _ptr(v), ctypes.byref(nnz), SDOT_HOST))
        return off, col, val, v

    def image_integrals(self, min_pt, max_pt, nb_pixels):
        """get_image_integrals: for the raster of nb_pixels = (nx, ny) pixels
        over [min_pt, max_pt], an array (ny, nx, 3) holding per pixel
        (sum m_i x_i, sum m_i y_i, sum m_i), m_i the integral of cell i over
        the pixel."""
        mn, mx = _f64(min_pt), _f64(max_pt)
        nbp = np.array(nb_pixels, dtype=np.int64)
        out = np.empty((int(nbp[1]), int(nbp[0]), 3))
        self._check(self._lib.sdot_get_image_integrals(self._ctx, _ptr(mn), _ptr(mx), _ptr(nbp), _ptr(out), SDOT_HOST))
        return out

    def image_of_cell_nums(self, min_pt, max_pt, nb_pixels):
        """get_image_of_cell_nums: an int64 array (ny, nx) holding per pixel the
        index of a cell of non-zero integral over it (the largest such index),
        -1 where there is none."""
        mn, mx = _f64(min_pt), _f64(max_pt)
        nbp = np.array(nb_pixels, dtype=np.int64)
        out = np.empty((int(nbp[1]), int(nbp[0])), dtype=np.int64)
        self._check(self._lib.sdot_get_image_of_cell_nums(self._ctx, _ptr(mn), _ptr(mx), _ptr(nbp), _ptr(out),
                                                          SDOT_HOST))
        return out

    def solve_weights(self, target_masses, rel_mass_tol=1e-10, max_iter=150, damping=True, pcg_rel_tol=1e-12,
                      pcg_max_iter=20000, verbosity=0, preconditioner="multilevel", linear_solver=None,
                      raise_on_failure=True):
        """Newton on the weights so that every cell mass reaches its target
        (OptimalTransportSolver::solve, OptimalTransportSolver.tcc:27-119).
        Updates the weights of this diagram and returns the solver report as
        a dict; raises SdotError when the tolerance is not reached.
        preconditioner: "multilevel" (V-cycle over Morton aggregates) or
        "jacobi".  linear_solver: "fp64" (FP64 PCG) or "fp32_refined" (FP32
        PCG with FP64 iterative refinement); by default "fp32_refined" for a
        mixed-precision diagram and "fp64" otherwise.  raise_on_failure=False
        returns the report (its "status" field set) instead of raising when the
        tolerance is not reached."""
        t = _f64(target_masses, (self.nb_diracs,))
        if linear_solver is None:
            linear_solver = "fp32_refined" if self.precision == "mixed" else "fp64"
        opt = _lib.SdotNewtonOptions(int(max_iter), float(rel_mass_tol), int(pcg_max_iter), float(pcg_rel_tol),
                                     int(bool(damping)), int(verbosity),
                                     {"multilevel": 0, "jacobi": 1}[preconditioner],
                                     {"fp64": 0, "fp32_refined": 1}[linear_solver])
        rep = _lib.SdotNewtonReport()
        st = self._lib.sdot_solve(self._ctx, _ptr(t), SDOT_HOST, ctypes.byref(opt), ctypes.byref(rep))
        w = np.empty(self.nb_diracs)
        self._check(self._lib.sdot_get_weights(self._ctx, _ptr(w), SDOT_HOST))
        self._weights = w
        report = {f: getattr(rep, f) for f, _ in rep._fields_}
        report["status"] = st
        if raise_on_failure or st not in (_lib.SDOT_OK, _lib.SDOT_NOT_CONVERGED):
            self._check(st)
        return report

    def evaluate(self):
        """Fused evaluation kept on the device (timing helper)."""
        self._check(self._lib.sdot_evaluate(self._ctx))

    def last_timings(self):
        t = np.zeros(3)
        self._lib.sdot_last_timings(self._ctx, _ptr(t))
        return {"tree_ms": t[0], "cells_ms": t[1], "hessian_ms": t[2]}

    def last_overflow_count(self):
        c = ctypes.c_int64(0)
        self._lib.sdot_last_overflow_count(self._ctx, ctypes.byref(c))
        return c.value


def csr_solve(offsets, columns, values, b, gauge_fix=True, rel_tol=1e-12, max_iter=20000):
    """Solves H x = b for a CSR matrix on the device (EigenSolver::solve,
    EigenSolver.cpp:9-41, by Jacobi-preconditioned conjugate gradients).
    Returns (x, iterations, relative residual); raises SdotError on failure."""
    lib = _lib.load()
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    col = np.ascontiguousarray(columns, dtype=np.int64)
    val = _f64(values)
    rhs = _f64(b)
    n = rhs.shape[0]
    x = np.zeros(n)
    it = ctypes.c_int64(0)
    res = ctypes.c_double(0)
    msg = ctypes.create_string_buffer(512)
    st = lib.sdot_csr_solve(_ptr(off), _ptr(col), _ptr(val), n, _ptr(rhs), _ptr(x), int(bool(gauge_fix)),
                            float(rel_tol), int(max_iter), SDOT_HOST, ctypes.byref(it), ctypes.byref(res), msg,
                            len(msg))
    if st != _lib.SDOT_OK:
        raise SdotError(st, msg.value.decode())
    return x, it.value, res.value
