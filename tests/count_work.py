"""Operation count of the 2D cell stage on the benchmark workload, measured.

    python tests/count_work.py            (needs a GPU; the counting build
                                            sdot_b200/libsdot_b200_count.so is
                                            compiled first when missing)

Runs one evaluation of the 1M-Dirac 2D clustered mix with the counting build
(-DSDOT_COUNT), which adds up the work of the fast tier's walks: cut attempts,
vertices classified at each attempt, node (eviction) tests and the vertices
tested at each (up to the first that fails, as the reference's all_pos
stops), effective cuts, final vertices.  With the operation weights of
the reference algorithm (FMA = 2 flops: bisector setup 12 per attempt, signed
distance 5 per vertex per attempt, eviction test 12 per vertex tested, area +
centroid 20 and boundary + Hessian term 15 per final vertex) it writes the
per-cell flop count to profiles/work_counts_c2_1M.json, which bench.py uses as
the roofline numerator.  Cells of the warp tier (about 0.1%) are not counted;
the count per cell is the fast tier's mean.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "profiles", "work_counts_c2_1M.json")

CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, {root!r})
from sdot_b200 import workloads, _lib
from sdot_b200.power_diagram import PowerDiagram
L = _lib.load()
c = workloads.config2()
g = PowerDiagram(c["positions"], c["weights"])
g.add_box_shape([0, 0], [1, 1])
g.evaluate()  # the first evaluation also tunes the block size (extra runs)
cnt = (ctypes.c_uint64 * 8)()
L.sdot_debug_work_counts(cnt, 1)
g.set_weights(c["weights"])
g.evaluate()
L.sdot_debug_work_counts(cnt, 0)
print(json.dumps([int(v) for v in cnt]))
"""


def main():
    sys.path.insert(0, ROOT)
    from sdot_b200 import build

    lib = build.build_counting()
    env = dict(os.environ, SDOT_B200_LIB=lib)
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                       check=True)
    a = json.loads(r.stdout.strip().splitlines()[-1])
    attempts, v_cut, tests, v_test, eff, final, cells = a[:7]
    flops = 12 * attempts + 5 * v_cut + 12 * v_test + 35 * final
    out = {"workload": "2D clustered mix, 1M Diracs, w ~ U[-1e-6, 1e-6] (the bench workload)",
           "cells_counted": cells, "cut_attempts": attempts, "vertices_at_cut_attempts": v_cut,
           "node_tests": tests, "vertices_at_node_tests": v_test, "effective_cuts": eff, "final_vertices": final,
           "per_cell": {"cut_attempts": attempts / cells, "vertices_per_attempt": v_cut / max(attempts, 1),
                        "node_tests": tests / cells, "vertices_per_test": v_test / max(tests, 1),
                        "final_vertices": final / cells},
           "flops_per_cell": flops / cells,
           "weights": "12 per attempt + 5 per vertex per attempt + 12 per vertex per node test + 35 per final vertex",
           "command": "python tests/count_work.py"}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
