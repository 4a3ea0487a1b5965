"""3D power-diagram cells with a multilinear density: a CPU restatement for
tests only (the oracle; nothing in the product imports it).

The reference's 3D densities are piecewise constant (ScaledImage with
nb_coeffs = 1, src/sdot/Domains/ScaledImage.tcc:36-69; Polynomial.h:53-58),
so no reference integrator exists for a smooth 3D density.  This oracle
builds each cell independently of the device kernels and of the reference:

  * cell i = {x in box : (x_j - x_i) . x <= (|x_j|^2 - |x_i|^2 + w_i - w_j)/2
    for every j}, the power cell of SpZGrid::for_each_laguerre_cell
    (src/sdot/Grids/SpZGrid.tcc:506-522), as a qhull half-space intersection
    (scipy.spatial.HalfspaceIntersection) from a Chebyshev centre;
  * its boundary triangulated by qhull (ConvexHull), each triangle assigned
    to the half-space it lies on (neighbour j, or a box face);
  * integrals of monomials exact on every tetrahedron (interior point +
    boundary triangle) and every boundary triangle by the simplex moment
    formula  int_T prod_{m=1..k} L_m = |T| d! / (d+k)! sum over ordered
    vertex tuples (a_1..a_k) of prod_i (mult_i)! prod_m L_m(v_{a_m})
    (from int_T lambda^alpha = |T| d! alpha! / (d + |alpha|)!).

Outputs follow the reference's definitions: mass = coeff int rho,
centroid = int rho x / int rho (get_centroids.h:13-56), Hessian row
-1/2 coeff int_{F_ij} rho / |x_i - x_j| per neighbour, the diagonal their
sum (get_der_integrals_wrt_weights.h:43-88, ConvexPolyhedron3 boundary
measures).  Pinned against the compiled reference at density 1 by the tests.
"""
import itertools
import math

import numpy as np
from scipy.optimize import linprog
from scipy.spatial import ConvexHull, HalfspaceIntersection

# multilinear basis: (1, x, y, z, xy, xz, yz, xyz) as coordinate lists
MONOMIALS = ([], [0], [1], [2], [0, 1], [0, 2], [1, 2], [0, 1, 2])


def _tuple_table(nv, k):
    """Ordered vertex tuples of length k over nv vertices and their weight
    prod_i (mult_i)!."""
    tab = []
    for t in itertools.product(range(nv), repeat=k):
        wgt = 1
        for a in set(t):
            wgt *= math.factorial(t.count(a))
        tab.append((t, wgt))
    return tab


_TABLES = {}


def simplex_monomial(V, coords):
    """int over each simplex of prod_m x_{coords[m]}, divided by its measure.
    V: (T, nv, 3) vertices (nv = 4 tetrahedra, 3 triangles)."""
    nv = V.shape[1]
    d = nv - 1
    k = len(coords)
    key = (nv, k)
    if key not in _TABLES:
        _TABLES[key] = _tuple_table(nv, k)
    acc = np.zeros(V.shape[0])
    for t, wgt in _TABLES[key]:
        p = np.full(V.shape[0], float(wgt))
        for m, a in enumerate(t):
            p = p * V[:, a, coords[m]]
        acc += p
    return acc * math.factorial(d) / math.factorial(d + k)


def _chebyshev_centre(A, b):
    """A point deep inside {x : A x <= b}, or None if the set is (nearly) empty."""
    nrm = np.linalg.norm(A, axis=1)
    c = np.zeros(A.shape[1] + 1)
    c[-1] = -1.0
    res = linprog(c, A_ub=np.hstack([A, nrm[:, None]]), b_ub=b, bounds=[(None, None)] * A.shape[1] + [(0, None)],
                  method="highs")
    if res.status != 0 or res.x[-1] <= 1e-12:
        return None
    return res.x[:-1]


class Cell:
    """One cell: boundary triangles (T, 3, 3), the id of each triangle's plane
    (a Dirac index, or -1 - face for box faces) and an interior point."""

    def __init__(self, tris, ids, centre):
        self.tris = tris
        self.ids = ids
        self.centre = centre


def build_cell(i, pos, w, lo, hi, cand=None, planes=None):
    """Power cell of Dirac i in the box [lo, hi] cut by the half-spaces
    planes[k, :3] . x <= planes[k, 3] (ids -7 - k; None: the box alone),
    None when empty."""
    n = len(pos)
    js = np.arange(n) if cand is None else np.asarray(cand)
    js = js[js != i]
    V = pos[js] - pos[i]
    P4 = np.zeros((0, 4)) if planes is None else np.asarray(planes, float).reshape(-1, 4)
    A = np.vstack([V, -np.eye(3), np.eye(3), P4[:, :3]])
    b = np.concatenate([0.5 * (np.sum(pos[js] ** 2, 1) - np.sum(pos[i] ** 2) + w[i] - w[js]),
                        -np.asarray(lo, float), np.asarray(hi, float), P4[:, 3]])
    ids = np.concatenate([js, -1 - np.arange(6), -7 - np.arange(len(P4))])
    x0 = _chebyshev_centre(A, b)
    if x0 is None:
        return None
    hs = HalfspaceIntersection(np.hstack([A, -b[:, None]]), x0)
    P = hs.intersections
    hull = ConvexHull(P)
    tris = P[hull.simplices]
    # plane of each triangle: the half-space its three vertices lie on
    nrm = np.linalg.norm(A, axis=1)
    dist = np.abs(np.einsum("tvk,hk->tvh", tris, A) - b[None, None, :]) / nrm[None, None, :]
    h = np.argmin(dist.max(axis=1), axis=1)
    scale = max(1.0, float(np.max(np.abs(P))))
    if np.max(dist.max(axis=1)[np.arange(len(h)), h]) > 1e-9 * scale:
        raise RuntimeError(f"cell {i}: a boundary triangle lies on no half-space")
    return Cell(tris, ids[h], x0)


def cells(pos, w=None, lo=(0, 0, 0), hi=(1, 1, 1), planes=None):
    """All cells; candidates grow from nearest neighbours until no other Dirac
    can cut (its bisector is farther than the cell's farthest vertex)."""
    pos = np.asarray(pos, float)
    n = len(pos)
    w = np.zeros(n) if w is None else np.asarray(w, float)
    out = [None] * n
    for i in range(n):
        d2 = np.sum((pos - pos[i]) ** 2, 1)
        near = np.argsort(d2)
        k = min(n, 48)
        while True:
            c = build_cell(i, pos, w, lo, hi, near[:k], planes)
            if c is None or k == n:
                break
            r = np.max(np.linalg.norm(c.tris.reshape(-1, 3) - pos[i], axis=1))
            rest = near[k:]
            d = np.sqrt(d2[rest])
            with np.errstate(divide="ignore", invalid="ignore"):
                reach = (d2[rest] + w[i] - w[rest]) / (2 * d)  # bisector distance from x_i
            if not np.any((d == 0) | (reach <= r * (1 + 1e-9))):
                break
            k = min(n, 2 * k)
        out[i] = c
    return out


def integrate(pos, w=None, poly=None, coeff=1.0, lo=(0, 0, 0), hi=(1, 1, 1), planes=None):
    """Masses (n), centroids (n, 3) and the Hessian as {(i, j): value} for
    density coeff * sum_m poly[m] * MONOMIALS[m] (poly None: constant) over
    the box [lo, hi] cut by `planes` (see build_cell)."""
    pos = np.asarray(pos, float)
    n = len(pos)
    w = np.zeros(n) if w is None else np.asarray(w, float)
    poly = np.array([1.0, 0, 0, 0, 0, 0, 0, 0]) if poly is None else np.asarray(poly, float)
    cs = cells(pos, w, lo, hi, planes)
    mass = np.zeros(n)
    ctd = np.zeros((n, 3))
    H = {}
    for i, c in enumerate(cs):
        if c is None:
            H[(i, i)] = 0.0
            continue
        T = len(c.tris)
        tet = np.concatenate([np.broadcast_to(c.centre, (T, 1, 3)), c.tris], axis=1)
        e1, e2, e3 = (tet[:, k] - tet[:, 0] for k in (1, 2, 3))
        vol = np.abs(np.einsum("tk,tk->t", e1, np.cross(e2, e3))) / 6
        m = 0.0
        mom = np.zeros(3)
        for a, cl in zip(poly, MONOMIALS):
            if a == 0:
                continue
            m += a * np.sum(vol * simplex_monomial(tet, cl))
            for d in range(3):
                mom[d] += a * np.sum(vol * simplex_monomial(tet, cl + [d]))
        mass[i] = coeff * m
        ctd[i] = mom / m if m != 0 else 0.0
        area = 0.5 * np.linalg.norm(np.cross(c.tris[:, 1] - c.tris[:, 0], c.tris[:, 2] - c.tris[:, 0]), axis=1)
        face = np.zeros(T)
        for a, cl in zip(poly, MONOMIALS):
            if a != 0:
                face += a * area * simplex_monomial(c.tris, cl)
        diag = 0.0
        for j in np.unique(c.ids):
            if j < 0:
                continue
            v = 0.5 * coeff * np.sum(face[c.ids == j]) / np.linalg.norm(pos[j] - pos[i])
            H[(i, int(j))] = -v
            diag += v
        H[(i, i)] = diag
    return mass, ctd, H


def box_integral(poly, lo=(0, 0, 0), hi=(1, 1, 1)):
    """Exact integral of the multilinear density over a box."""
    res = 0.0
    for a, cl in zip(poly, MONOMIALS):
        t = a
        for d in range(3):
            t *= 0.5 * (hi[d] ** 2 - lo[d] ** 2) if d in cl else hi[d] - lo[d]
        res += t
    return res


def integrate_shapes(pos, shapes, w=None, poly=None):
    """A domain of several convex shapes (ConvexPolyhedronAssembly: each
    cell is intersected with every shape and the pieces summed,
    ConvexPolyhedronAssembly.tcc:132-142).  shapes: list of (lo, hi, planes,
    coeff).  Returns masses, centroids and the Hessian dict like integrate."""
    pos = np.asarray(pos, float)
    n = len(pos)
    mass = np.zeros(n)
    mom = np.zeros((n, 3))
    H = {}
    for lo, hi, planes, coeff in shapes:
        m, c, h = integrate(pos, w, poly, coeff, lo, hi, planes)
        mass += m
        mom += c * m[:, None]
        for k, v in h.items():
            H[k] = H.get(k, 0.0) + v
    ctd = np.where(mass[:, None] != 0, mom / np.where(mass == 0, 1.0, mass)[:, None], 0.0)
    return mass, ctd, H
