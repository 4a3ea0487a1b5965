"""Test infrastructure only: ctypes wrapper of the compiled reference oracle.

oracle/_ref/libsdot_ref.so is the UNMODIFIED reference sdot path (SpZGrid +
get_integrals / get_centroids / get_der_integrals_wrt_weights over
ConvexPolyhedronAssembly or ScaledImage bounds), compiled by oracle/Makefile
from the reference sources with the driver oracle/ref_driver.cpp.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
parity reference and the timed CPU baseline.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libsdot_ref.so")
# The reference checkout: $SDOT_REFERENCE_DIR, else a checkout named
# "reference" beside this repository's root directory.
REF_TREE = os.environ.get("SDOT_REFERENCE_DIR") or os.path.join(os.path.dirname(HERE), os.pardir, "reference")

_lib = None


def build(force=False):
    """Compile oracle/_ref/libsdot_ref.so when the reference tree is present."""
    if os.path.exists(REF_LIB) and not force:
        return REF_LIB
    if not os.path.isdir(REF_TREE):
        return None
    subprocess.run(["make", "-C", HERE, "ref", f"REF={REF_TREE}"], check=True, capture_output=True)
    return REF_LIB


def available():
    return os.path.exists(REF_LIB)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise ImportError("oracle/_ref/libsdot_ref.so is not built")
    L = ctypes.CDLL(REF_LIB)
    P, I64, D, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
    sig = {
        "ref_init_threads": (None, [I]),
        "ref_nb_threads": (I, []),
        "ref_create": (P, [I, I64]),
        "ref_destroy": (None, [P]),
        "ref_set_diracs": (None, [P, I64, P, P]),
        "ref_set_ball_cut": (None, [P, I]),
        "ref_add_box": (None, [P, P, P, D]),
        "ref_add_convex_polyhedron": (None, [P, I64, P, P, D]),
        "ref_add_simplex": (None, [P, P, D]),
        "ref_normalize": (None, [P]),
        "ref_domain_measure": (D, [P]),
        "ref_set_image": (None, [P, P, P, P, P, I64]),
        "ref_update": (None, [P]),
        "ref_get_integrals": (None, [P, P]),
        "ref_get_centroids": (None, [P, P, P]),
        "ref_get_der_integrals_wrt_weights": (I, [P, I]),
        "ref_der_nnz": (I64, [P]),
        "ref_der_copy": (None, [P, P, P, P, P]),
        "ref_neighbors": (I64, [P]),
        "ref_neighbors_copy": (None, [P, P, P]),
        "ref_timings": (None, [P, P]),
        "ref_get_image_integrals": (None, [P, P, P, P, P]),
        "ref_set_translations": (None, [P, P, I64]),
        "ref_der_pos": (I64, [P]),
        "ref_der_pos_copy": (None, [P, P, P, P, P]),
        "ref_get_image_of_cell_nums": (None, [P, P, P, P, P]),
    }
    for k, (r, a) in sig.items():
        f = getattr(L, k)
        f.restype = r
        f.argtypes = a
    _lib = L
    return L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class RefPowerDiagram:
    """The reference's own CPU path, driven with the same calls as the product."""

    def __init__(self, positions, weights=None, dim=None, radial_func="unit", max_diracs_per_cell=11, threads=0):
        self.L = load()
        if threads:
            self.L.ref_init_threads(int(threads))
        self.pos = _f(positions)
        self.dim = dim or self.pos.shape[1]
        n = self.pos.shape[0]
        self.w = np.zeros(n) if weights is None else _f(weights)
        self.h = ctypes.c_void_p(self.L.ref_create(self.dim, int(max_diracs_per_cell)))
        self.L.ref_set_diracs(self.h, n, _p(self.pos), _p(self.w))
        self.L.ref_set_ball_cut(self.h, 1 if radial_func == "in_ball_w05" else 0)
        self._updated = False

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    @property
    def n(self):
        return self.pos.shape[0]

    def set_weights(self, w):
        self.w = _f(w)
        self.L.ref_set_diracs(self.h, self.n, _p(self.pos), _p(self.w))
        self._updated = False

    def add_box_shape(self, p0, p1, coeff=1.0):
        a, b = _f(p0), _f(p1)
        self.L.ref_add_box(self.h, _p(a), _p(b), float(coeff))

    def add_convex_polyhedron_shape(self, points, normals, coeff=1.0):
        pts = _f(points).reshape(-1, self.dim)
        nrm = _f(normals).reshape(pts.shape)
        self.L.ref_add_convex_polyhedron(self.h, pts.shape[0], _p(pts), _p(nrm), float(coeff))

    def add_simplex_shape(self, points, coeff=1.0):
        a = _f(points).reshape(-1)
        self.L.ref_add_simplex(self.h, _p(a), float(coeff))

    def normalize_domain(self):
        self.L.ref_normalize(self.h)

    def domain_measure(self):
        return self.L.ref_domain_measure(self.h)

    def set_image_density(self, image, min_pt=None, max_pt=None, nb_coeffs=None):
        """image: (ny, nx) values, or (6, ny, nx) coefficient planes (nb_coeffs = 6)."""
        img = _f(image)
        if nb_coeffs is None:
            nb_coeffs = img.shape[0] if img.ndim == self.dim + 1 else 1
        spatial = img.shape[1:] if nb_coeffs > 1 else img.shape
        sizes = np.array(spatial[::-1], dtype=np.int64)
        mn = _f(min_pt if min_pt is not None else np.zeros(self.dim))
        mx = _f(max_pt if max_pt is not None else np.ones(self.dim))
        self._img = img
        self.L.ref_set_image(self.h, _p(mn), _p(mx), _p(img), _p(sizes), int(nb_coeffs))

    def update(self):
        self.L.ref_update(self.h)
        self._updated = True

    def _ensure(self):
        if not self._updated:
            self.update()

    def integrals(self):
        self._ensure()
        out = np.zeros(self.n)
        self.L.ref_get_integrals(self.h, _p(out))
        return out

    def centroids(self, with_masses=False):
        self._ensure()
        c = np.zeros((self.n, self.dim))
        m = np.zeros(self.n)
        self.L.ref_get_centroids(self.h, _p(c), _p(m))
        return (c, m) if with_masses else c

    def der_integrals_wrt_weights(self, stop_if_void=False):
        self._ensure()
        err = self.L.ref_get_der_integrals_wrt_weights(self.h, int(stop_if_void))
        nnz = self.L.ref_der_nnz(self.h)
        off = np.zeros(self.n + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int64)
        val = np.zeros(nnz)
        mas = np.zeros(self.n)
        if err == 0:
            self.L.ref_der_copy(self.h, _p(off), _p(col), _p(val), _p(mas))
        return err, off, col, val, mas

    def neighbors(self):
        self._ensure()
        cnt = self.L.ref_neighbors(self.h)
        off = np.zeros(self.n + 1, dtype=np.int64)
        ids = np.zeros(cnt, dtype=np.int64)
        self.L.ref_neighbors_copy(self.h, _p(off), _p(ids))
        return off, ids

    def der_centroids_and_integrals_wrt_weight_and_positions(self):
        """get_der_centroids_and_integrals_wrt_weight_and_positions: CSR over
        (dim + 1) n rows and columns (offsets, columns, values) and the
        values (centroid, mass) per Dirac."""
        self._ensure()
        nnz = self.L.ref_der_pos(self.h)
        if nnz < 0:
            raise RuntimeError("void cell")
        k = self.dim + 1
        off = np.zeros(k * self.n + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int64)
        val = np.zeros(nnz)
        v = np.zeros(k * self.n)
        self.L.ref_der_pos_copy(self.h, _p(off), _p(col), _p(val), _p(v))
        return off, col, val, v

    def set_translations(self, translations):
        t = _f(np.asarray(translations, dtype=np.float64).reshape(-1, self.dim))
        self.L.ref_set_translations(self.h, _p(t), t.shape[0])
        self._updated = False

    def image_integrals(self, min_pt, max_pt, nb_pixels):
        """get_image_integrals: (ny, nx, 3) per pixel (sum m x, sum m y, sum m)."""
        self._ensure()
        mn, mx = _f(min_pt), _f(max_pt)
        nbp = np.array(nb_pixels, dtype=np.int64)
        out = np.zeros((int(nbp[1]), int(nbp[0]), 3))
        self.L.ref_get_image_integrals(self.h, _p(mn), _p(mx), _p(nbp), _p(out))
        return out

    def image_of_cell_nums(self, min_pt, max_pt, nb_pixels):
        """get_image_of_cell_nums: (ny, nx) int64, -1 where no cell."""
        self._ensure()
        mn, mx = _f(min_pt), _f(max_pt)
        nbp = np.array(nb_pixels, dtype=np.int64)
        out = np.zeros((int(nbp[1]), int(nbp[0])), dtype=np.int64)
        self.L.ref_get_image_of_cell_nums(self.h, _p(mn), _p(mx), _p(nbp), _p(out))
        return out

    def timings(self):
        t = np.zeros(4)
        self.L.ref_timings(self.h, _p(t))
        return {"update_s": t[0], "integrals_s": t[1], "centroids_s": t[2], "der_s": t[3]}
