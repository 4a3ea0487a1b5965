"""Pins the C restatement oracle against the golden fixtures of tests/golden/
(generated from the compiled reference by tests/golden/make_golden.py) and,
when oracle/_ref is built, against the compiled reference on larger seeded
inputs.  CPU only.

Tolerances as in tests/test_gpu_parity_2d.py: errors are measured against
max(|reference|, the mean of the quantity over all cells), RTOL = 1e-12.
"""
import glob
import os

import numpy as np
import pytest

from oracle.port import PortPowerDiagram
from sdot_b200 import workloads
from tests.helpers import assert_close, neighbor_sets

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-12

SHAPES = {
    "two_boxes_simplex_300": [("add_box_shape", ([0.0, 0.0], [1.0, 1.0], 1.0)),
                              ("add_box_shape", ([1.0, 0.0], [2.0, 1.0], 0.5)),
                              ("add_simplex_shape", ([[0.2, 0.2], [0.9, 0.3], [0.4, 0.8]], 2.0))],
}


def load_case(path):
    d = dict(np.load(path, allow_pickle=False))
    d["radial"] = str(d["radial"])
    return d


def port_for(name, d):
    pd = PortPowerDiagram(d["positions"], d["weights"], radial_func=d["radial"])
    if "image" in d:
        pd.set_image_density(d["image"])
    elif name in SHAPES:
        for kind, args in SHAPES[name]:
            getattr(pd, kind)(*args)
    else:
        pd.add_box_shape([0.0, 0.0], [1.0, 1.0])
    return pd


def compare(pd, ref, n, rtol=RTOL):
    """ref: dict with masses, centroids, centroid_masses, offsets, columns, values, nb_offsets, nb_ids."""
    m = pd.integrals()
    mean = max(float(np.abs(ref["masses"]).mean()), 1e-300)
    assert_close(m, ref["masses"], rtol, mean, "masses")
    c, mc = pd.centroids(with_masses=True)
    assert_close(mc, ref["centroid_masses"], rtol, mean, "centroid masses")
    assert_close(c, ref["centroids"], rtol, 1.0, "centroids")
    err, off, col, val, _ = pd.der_integrals_wrt_weights()
    assert np.array_equal(off, ref["offsets"]) and np.array_equal(col, ref["columns"])
    rows = np.repeat(np.arange(n), np.diff(ref["offsets"]))
    diag = np.abs(ref["values"][ref["columns"] == rows]).mean()
    assert_close(val, ref["values"], rtol, diag, "Hessian")
    no, ni = pd.neighbors()
    assert neighbor_sets(no, ni) == neighbor_sets(ref["nb_offsets"], ref["nb_ids"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))), ids=os.path.basename)
def test_port_matches_golden(path):
    name = os.path.basename(path)[:-4]
    d = load_case(path)
    compare(port_for(name, d), d, len(d["weights"]))


def _ref_dict(r):
    m = r.integrals()
    c, mc = r.centroids(with_masses=True)
    err, off, col, val, _ = r.der_integrals_wrt_weights()
    no, ni = r.neighbors()
    return dict(masses=m, centroids=c, centroid_masses=mc, offsets=off, columns=col, values=val, nb_offsets=no,
                nb_ids=ni)


@pytest.mark.parametrize("case", ["config1", "disc_3000", "image_disc_5000"])
def test_port_matches_compiled_reference(ref_oracle, case):
    if case == "config1":
        c = workloads.config1()
        p, w, kw = c["positions"], c["weights"], {}
    elif case == "disc_3000":
        rng = np.random.default_rng(3)
        p = rng.random((3000, 2))
        w = np.full(3000, (0.5 / np.sqrt(3000)) ** 2) * rng.uniform(0.5, 2.0, 3000)
        kw = {"radial": "in_ball_w05"}
    else:
        c = workloads.config3(n=5000, res=128)
        p, w, kw = c["positions"], c["weights"], {"radial": "in_ball_w05", "image": c["image"]}
    r = ref_oracle.RefPowerDiagram(p, w, radial_func=kw.get("radial", "unit"))
    q = PortPowerDiagram(p, w, radial_func=kw.get("radial", "unit"))
    for pd in (r, q):
        if "image" in kw:
            pd.set_image_density(kw["image"])
        else:
            pd.add_box_shape([0.0, 0.0], [1.0, 1.0])
    compare(q, _ref_dict(r), len(w), rtol=RTOL if case == "config1" else 1e-11)
