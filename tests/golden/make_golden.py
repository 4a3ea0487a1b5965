"""Generates the golden fixtures of tests/golden/ from the compiled reference.

    python tests/golden/make_golden.py

Needs oracle/_ref/libsdot_ref.so (the unmodified reference path compiled
by `make -C oracle ref`, which needs the reference tree).  Each fixture is a
small seeded case: inputs, cell masses (get_integrals), centroids and masses
(get_centroids), the CSR Hessian (get_der_integrals_wrt_weights, stop_if_void
= false) and the boundary cut ids of every cell.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from sdot_b200 import workloads  # noqa: E402


def cases():
    rng = np.random.default_rng(20261203)
    yield "uniform_500", dict(p=rng.random((500, 2)), w=np.zeros(500))
    rng = np.random.default_rng(20261204)
    p = np.concatenate([rng.random((400, 2)), workloads.clustered_points(400, 2, rng, nb_clusters=4, sigma=0.05)])
    yield "clustered_weights_800", dict(p=p, w=rng.uniform(-1e-4, 1e-4, 800))
    rng = np.random.default_rng(20261205)
    n = 400
    yield "disc_clip_400", dict(p=rng.random((n, 2)), w=np.full(n, (0.5 / np.sqrt(n)) ** 2) * rng.uniform(0.5, 2, n),
                                radial="in_ball_w05")
    rng = np.random.default_rng(20261206)
    c = workloads.config3(n=400, res=32)
    yield "image_disc_400", dict(p=c["positions"], w=c["weights"], radial="in_ball_w05", image=c["image"])
    rng = np.random.default_rng(20261207)
    yield "two_boxes_simplex_300", dict(
        p=rng.random((300, 2)) * [2, 1], w=np.zeros(300),
        shapes=[("add_box_shape", ([0.0, 0.0], [1.0, 1.0], 1.0)), ("add_box_shape", ([1.0, 0.0], [2.0, 1.0], 0.5)),
                ("add_simplex_shape", ([[0.2, 0.2], [0.9, 0.3], [0.4, 0.8]], 2.0))])


def build_pd(cls, case):
    pd = cls(case["p"], case["w"], radial_func=case.get("radial", "unit"))
    if "image" in case:
        pd.set_image_density(case["image"])
    elif "shapes" in case:
        for kind, args in case["shapes"]:
            getattr(pd, kind)(*args)
    else:
        pd.add_box_shape([0.0, 0.0], [1.0, 1.0])
    return pd


def main():
    ref.build()
    for name, case in cases():
        pd = build_pd(ref.RefPowerDiagram, case)
        m = pd.integrals()
        c, mc = pd.centroids(with_masses=True)
        err, off, col, val, mas = pd.der_integrals_wrt_weights()
        no, ni = pd.neighbors()
        extra = {}
        if "image" in case:
            extra["image"] = case["image"]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), positions=case["p"], weights=case["w"],
                            radial=case.get("radial", "unit"), masses=m, centroids=c, centroid_masses=mc,
                            offsets=off, columns=col, values=val, nb_offsets=no, nb_ids=ni, **extra)
        print(name, len(case["w"]), "nnz", len(col))


if __name__ == "__main__":
    main()
