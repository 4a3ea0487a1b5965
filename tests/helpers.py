"""Comparison helpers shared by the parity tests."""
import numpy as np

from sdot_b200.power_diagram import PowerDiagram


def make_pair(positions, weights, ref_mod, domain="unit_box", radial_func="unit", image=None, shapes=None,
              precision="fp64"):
    """Build the product PowerDiagram and the reference oracle on the same inputs."""
    gpu = PowerDiagram(positions, weights, precision=precision, radial_func=radial_func)
    ref = ref_mod.RefPowerDiagram(positions, weights, radial_func=radial_func)
    dim = positions.shape[1]
    if image is not None:
        gpu.set_image_density(image)
        ref.set_image_density(image)
    elif shapes is not None:
        for kind, args in shapes:
            getattr(gpu, kind)(*args)
            getattr(ref, kind)(*args)
    elif domain == "unit_box":
        gpu.add_box_shape(np.zeros(dim), np.ones(dim))
        ref.add_box_shape(np.zeros(dim), np.ones(dim))
    return gpu, ref


def rel_err(a, b, floor):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    return np.where(d == 0, 0.0, d / np.maximum(np.abs(b), max(float(floor), 1e-300)))


def assert_close(a, b, rtol, floor, what):
    e = rel_err(np.asarray(a), np.asarray(b), floor)
    k = int(np.argmax(e)) if e.size else 0
    assert e.size == 0 or e.max() <= rtol, f"{what}: max rel err {e.max():.3e} at {k}: {np.ravel(a)[k]!r} vs {np.ravel(b)[k]!r}"


def csr_rows(off, col, val):
    return [(col[off[i]:off[i + 1]], val[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


def compare_csr(g, r, rtol, floor):
    """g, r: (offsets, columns, values).  Same sparsity pattern, values within rtol."""
    go, gc, gv = g
    ro, rc, rv = r
    assert np.array_equal(go, ro), "CSR offsets differ"
    assert np.array_equal(gc, rc), "CSR columns differ"
    assert_close(gv, rv, rtol, floor, "CSR values")


def neighbor_sets(off, ids):
    return [frozenset(int(x) for x in ids[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


def neighbor_set_mismatches(off_a, ids_a, off_b, ids_b):
    """Rows whose sets of ids differ (vectorised: one unique-sort of
    (row, id) keys per side).  Returns the sorted array of those rows."""
    n = len(off_a) - 1
    assert len(off_b) - 1 == n

    def keys(off, ids):
        rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
        return np.unique(rows * (np.int64(n) + 8) + (np.asarray(ids, dtype=np.int64) + 4))

    ka, kb = keys(off_a, ids_a), keys(off_b, ids_b)
    only = np.setxor1d(ka, kb, assume_unique=True)
    return np.unique(only // (np.int64(n) + 8))
