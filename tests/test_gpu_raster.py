"""Rasterisation of the diagram on the GPU against the compiled reference:
get_image_integrals (get_image_integrals.h:16-78) and get_image_of_cell_nums
(get_image_of_cell_nums.h:13-80).

Image integrals: per pixel (sum m_i x_i, sum m_i y_i, sum m_i); the GPU adds
the cells' contributions to a pixel atomically, in no fixed order, so the sums
agree with the reference's to rounding: within 1e-12 of max(|ref|, the mean
pixel value of that component).
Cell numbers: where several cells meet a pixel the reference keeps the one
its work order wrote last and the GPU the largest index; both must mark the
same pixels as covered, the GPU's index is never below the reference's (the
reference's is one of the covering cells), and where they differ the GPU's
cell borders the reference's one.
"""
import numpy as np
import pytest

from sdot_b200 import workloads
from tests.helpers import assert_close, make_pair

pytestmark = pytest.mark.gpu


def check_integrals(gpu, ref, lo, hi, nbp):
    g = gpu.image_integrals(lo, hi, nbp)
    r = ref.image_integrals(lo, hi, nbp)
    for k in range(3):
        assert_close(g[..., k], r[..., k], 1e-12, np.abs(r[..., k]).mean(), f"image integrals component {k}")
    return g, r


@pytest.mark.parametrize("radial_func", ["unit", "in_ball_w05"])
def test_image_integrals_box(gpu_lib, ref_oracle, radial_func):
    rng = np.random.default_rng(71)
    n = 2000
    p = rng.random((n, 2))
    w = np.full(n, 0.3 / n) * rng.uniform(0.5, 2.0, n) if radial_func != "unit" else rng.uniform(-1e-5, 1e-5, n)
    gpu, ref = make_pair(p, w, ref_oracle, radial_func=radial_func)
    g, _ = check_integrals(gpu, ref, [0.0, 0.0], [1.0, 1.0], (64, 48))
    assert abs(g[..., 2].sum() - gpu.integrals().sum()) < 1e-12


def test_image_integrals_clustered(gpu_lib, ref_oracle):
    c = workloads.config2(n=100_000)
    gpu, ref = make_pair(c["positions"], c["weights"], ref_oracle)
    check_integrals(gpu, ref, [0.0, 0.0], [1.0, 1.0], (256, 256))


def test_image_integrals_several_shapes(gpu_lib, ref_oracle):
    rng = np.random.default_rng(72)
    n = 1500
    p = rng.random((n, 2)) * [2.0, 1.0]
    shapes = [("add_box_shape", ([0.0, 0.0], [1.0, 1.0], 1.0)),
              ("add_box_shape", ([1.0, 0.0], [2.0, 1.0], 0.5))]
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle, shapes=shapes)
    check_integrals(gpu, ref, [0.0, 0.0], [2.0, 1.0], (80, 40))


def test_image_of_cell_nums(gpu_lib, ref_oracle):
    rng = np.random.default_rng(73)
    n = 300
    p = rng.random((n, 2))
    gpu, ref = make_pair(p, np.zeros(n), ref_oracle)
    nbp = (200, 160)
    g = gpu.image_of_cell_nums([0.0, 0.0], [1.0, 1.0], nbp)
    r = ref.image_of_cell_nums([0.0, 0.0], [1.0, 1.0], nbp)
    assert ((g < 0) == (r < 0)).all()
    assert (g >= r).all()
    # where they differ, the pixel meets several cells (pixels are ~1/100 of
    # a cell): the GPU's cell is then a neighbour of the reference's one, or
    # a neighbour of one of its neighbours (a pixel over a short edge meets
    # the two cells on either side of it, which do not touch)
    off, ids = ref.neighbors()
    nb = [set(int(j) for j in ids[off[i]:off[i + 1]] if j >= 0) for i in range(n)]
    diff = np.argwhere(g != r)
    assert len(diff) < 0.2 * g.size
    for iy, ix in diff:
        a, b = int(r[iy, ix]), int(g[iy, ix])
        assert b in nb[a] or any(b in nb[k] for k in nb[a]), (iy, ix, a, b)
