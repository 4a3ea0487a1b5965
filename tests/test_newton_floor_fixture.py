"""The FP64 floor of Newton on the clamped 2D clustered workload, as the
compiled reference meets it (fixture tests/golden/newton_floor_c2.json, made
by tests/golden/make_newton_floor.py with the Newton oracle over the compiled
reference and a direct sparse solve).

Clamping the clustered Diracs to the unit box puts pairs of them on the box
edges a few 1e-8 apart; their shared edge cannot be placed finely enough in
FP64 for a relative mass error of 1e-8, so the reference itself stalls above
it, and the floor grows with n.  The GPU solver's runs on the same input are
held to what the reference reaches (tests/test_gpu_newton.py)."""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def test_reference_newton_floor_on_clamped_mix():
    with open(os.path.join(HERE, "golden", "newton_floor_c2.json")) as f:
        d = json.load(f)
    runs = sorted(d["runs"], key=lambda r: r["n"])
    assert len(runs) >= 2
    for r in runs:
        assert not r["converged"]
        assert r["final_max_rel_mass_error"] > 1e-7
        assert r["min_pair_distance"] < 1e-7  # the clamped near-coincident pairs
        # the error stopped decreasing: the last iterations gained less than 10x
        tr = r["trace"]
        assert min(tr) > 0.1 * tr[-1] or len(tr) < 3
    # the floor does not improve with n
    assert runs[-1]["final_max_rel_mass_error"] >= runs[0]["final_max_rel_mass_error"]
