"""Serving loop: each result is the same alone and in the mix.

A mixed stream of 2D and 3D requests of uneven sizes is solved by a 3-slot
server (requests overlap on the GPU) and again one request at a time
(1 slot); the solved weights must agree within 1e-12 of max |w| (the kernels
and reductions are deterministic, so they agree bitwise in practice), and
every request must meet the mass tolerance.
"""
import numpy as np
import pytest

from sdot_b200 import workloads

pytestmark = pytest.mark.gpu


def requests():
    rng = np.random.default_rng(55)
    out = []
    for k, (dim, n) in enumerate([(2, 3000), (3, 1500), (2, 20000), (2, 1000), (3, 4000), (2, 8000)]):
        if dim == 2 and k % 2:
            p = np.concatenate([rng.random((n // 2, 2)), workloads.clustered_points(n - n // 2, 2, rng)])
        else:
            p = rng.random((n, dim))
        out.append((p, np.full(n, 1.0 / n)))
    return out


def solve_all(slots, reqs):
    from sdot_b200.serving import Server

    srv = Server(slots=slots, hbm_budget_bytes=4 << 30, rel_mass_tol=1e-10)
    ids = [srv.submit(p, t) for p, t in reqs]
    srv.drain()
    res = [srv.result(i) for i in ids]
    srv.close()
    return res


def test_same_result_alone_and_in_the_mix(gpu_lib):
    reqs = requests()
    mix = solve_all(3, reqs)
    alone = solve_all(1, reqs)
    for (wm, rm), (wa, ra) in zip(mix, alone):
        assert rm["max_rel_mass_error"] <= 1e-10 and ra["max_rel_mass_error"] <= 1e-10
        assert np.abs(wm - wa).max() <= 1e-12 * np.abs(wa).max()
    # in the mix, requests overlapped in time
    spans = sorted((r["start_ms"], r["end_ms"]) for _, r in mix)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_budget_admits_oversized_request_alone(gpu_lib):
    from sdot_b200.serving import Server

    srv = Server(slots=2, hbm_budget_bytes=1 << 20, rel_mass_tol=1e-8)  # smaller than any request
    rng = np.random.default_rng(56)
    ids = [srv.submit(rng.random((2000, 2)), np.full(2000, 1 / 2000)) for _ in range(3)]
    srv.drain()
    reps = [srv.result(i)[1] for i in ids]
    srv.close()
    spans = sorted((r["start_ms"], r["end_ms"]) for r in reps)
    assert all(spans[i + 1][0] >= spans[i][1] for i in range(len(spans) - 1))  # one at a time
