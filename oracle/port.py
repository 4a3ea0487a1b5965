"""Test infrastructure only: ctypes wrapper of the C restatement oracle.

oracle/libsdot_oracle.so is built from oracle/sdot_oracle.c (plain C, no
reference sources needed), so it is available wherever gcc is.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsdot_oracle.so")

_lib = None


def build(force=False):
    src = os.path.join(HERE, "sdot_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(src) > os.path.getmtime(LIB):
        subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(LIB)
    P, I64, D, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
    sig = {
        "or_poly_box": (P, [D, D, D, D, I64]),
        "or_poly_simplex": (P, [P, I64]),
        "or_poly_copy": (P, [P]),
        "or_poly_free": (None, [P]),
        "or_poly_plane_cut": (I, [P, D, D, D, D, I64, I]),
        "or_poly_ball_cut": (None, [P, D, D, D, I64]),
        "or_poly_intersect_with": (None, [P, P]),
        "or_poly_nb_points": (I, [P]),
        "or_poly_points": (None, [P, P, P, P]),
        "or_poly_measure": (D, [P]),
        "or_poly_centroid": (None, [P, D, P, P]),
        "or_poly_integrate_poly6": (D, [P, P]),
        "or_poly_sphere_radius": (D, [P]),
        "or_domain_new": (P, []),
        "or_domain_free": (None, [P]),
        "or_domain_add_box": (None, [P, P, P, D]),
        "or_domain_add_simplex": (None, [P, P, D]),
        "or_domain_add_convex_polyhedron": (None, [P, P, P, I64, D]),
        "or_domain_set_image": (None, [P, P, P, P, P, I]),
        "or_domain_normalize": (None, [P]),
        "or_domain_measure": (D, [P]),
        "or_power_diagram_2d": (I, [I64, P, P, P, I, P, P, P, P, P, P, I64, P, P, I64]),
    }
    for k, (r, a) in sig.items():
        f = getattr(L, k)
        f.restype = r
        f.argtypes = a
    _lib = L
    return L


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class Poly:
    """One ConvexPolyhedron2 (the reference's single-polygon API)."""

    def __init__(self, handle):
        self.L = load()
        self.h = ctypes.c_void_p(handle)

    @classmethod
    def box(cls, p0, p1, cut_id=-1):
        return cls(load().or_poly_box(p0[0], p0[1], p1[0], p1[1], cut_id))

    @classmethod
    def simplex(cls, pts, cut_id=-1):
        a = _f(pts).reshape(-1)
        return cls(load().or_poly_simplex(_p(a), cut_id))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_poly_free(self.h)
            self.h = None

    def plane_cut(self, origin, normal, cut_id=-1, normalized=True):
        return self.L.or_poly_plane_cut(self.h, origin[0], origin[1], normal[0], normal[1], cut_id, int(normalized))

    def ball_cut(self, center, radius, cut_id=-1):
        self.L.or_poly_ball_cut(self.h, center[0], center[1], radius, cut_id)

    def nb_points(self):
        return self.L.or_poly_nb_points(self.h)

    def measure(self):
        return self.L.or_poly_measure(self.h)

    def centroid(self, coeff=1.0):
        c = np.zeros(2)
        m = np.zeros(1)
        self.L.or_poly_centroid(self.h, coeff, _p(c), _p(m))
        return c

    def integrate_poly6(self, coeffs):
        c = _f(coeffs)
        return self.L.or_poly_integrate_poly6(self.h, _p(c))


class PortPowerDiagram:
    """The C restatement driven with the same calls as the product."""

    def __init__(self, positions, weights=None, radial_func="unit"):
        self.L = load()
        self.pos = _f(positions)
        n = self.pos.shape[0]
        self.w = np.zeros(n) if weights is None else _f(weights)
        self.ball = radial_func == "in_ball_w05"
        self.dom = ctypes.c_void_p(self.L.or_domain_new())
        self._res = None

    def __del__(self):
        if getattr(self, "dom", None):
            self.L.or_domain_free(self.dom)
            self.dom = None

    @property
    def n(self):
        return self.pos.shape[0]

    def set_weights(self, w):
        self.w = _f(w)
        self._res = None

    def add_box_shape(self, p0, p1, coeff=1.0):
        a, b = _f(p0), _f(p1)
        self.L.or_domain_add_box(self.dom, _p(a), _p(b), float(coeff))
        self._res = None

    def add_simplex_shape(self, pts, coeff=1.0):
        a = _f(pts).reshape(-1)
        self.L.or_domain_add_simplex(self.dom, _p(a), float(coeff))
        self._res = None

    def add_convex_polyhedron_shape(self, pts, nrm, coeff=1.0):
        p = _f(pts).reshape(-1, 2)
        q = _f(nrm).reshape(p.shape)
        self.L.or_domain_add_convex_polyhedron(self.dom, _p(p), _p(q), p.shape[0], float(coeff))
        self._res = None

    def set_image_density(self, image, min_pt=None, max_pt=None, nb_coeffs=1):
        img = _f(image)
        if nb_coeffs == 1:
            sizes = np.array(img.shape[::-1], dtype=np.int64)
        else:
            sizes = np.array(img.shape[1:][::-1], dtype=np.int64)
        mn = _f(min_pt if min_pt is not None else [0.0, 0.0])
        mx = _f(max_pt if max_pt is not None else [1.0, 1.0])
        self._img = img
        self.L.or_domain_set_image(self.dom, _p(mn), _p(mx), _p(img), _p(sizes), int(nb_coeffs))
        self._res = None

    def normalize_domain(self):
        self.L.or_domain_normalize(self.dom)
        self._res = None

    def domain_measure(self):
        return self.L.or_domain_measure(self.dom)

    def _run(self):
        if self._res is not None:
            return self._res
        n = self.n
        cap = 64 * max(n, 1)
        mass, mc = np.zeros(n), np.zeros(n)
        ctd = np.zeros((n, 2))
        off = np.zeros(n + 1, dtype=np.int64)
        cols = np.zeros(cap, dtype=np.int64)
        vals = np.zeros(cap)
        nbo = np.zeros(n + 1, dtype=np.int64)
        nbi = np.zeros(cap, dtype=np.int64)
        st = self.L.or_power_diagram_2d(n, _p(self.pos), _p(self.w), self.dom, int(self.ball), _p(mass), _p(ctd),
                                        _p(mc), _p(off), _p(cols), _p(vals), cap, _p(nbo), _p(nbi), cap)
        if st != 0:
            raise RuntimeError("oracle buffers too small")
        self._res = dict(mass=mass, mass_c=mc, ctd=ctd, off=off, cols=cols[:off[-1]], vals=vals[:off[-1]],
                         nbo=nbo, nbi=nbi[:nbo[-1]])
        return self._res

    def integrals(self):
        return self._run()["mass"].copy()

    def centroids(self, with_masses=False):
        r = self._run()
        return (r["ctd"].copy(), r["mass_c"].copy()) if with_masses else r["ctd"].copy()

    def der_integrals_wrt_weights(self, stop_if_void=False):
        r = self._run()
        err = int(stop_if_void and bool((r["mass"] == 0).any()))
        return err, r["off"].copy(), r["cols"].copy(), r["vals"].copy(), r["mass"].copy()

    def neighbors(self):
        r = self._run()
        return r["nbo"].copy(), r["nbi"].copy()
