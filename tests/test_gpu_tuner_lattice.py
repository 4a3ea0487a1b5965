"""The fast 2D kernels tune their block size on the first evaluation of at
least 131,072 cells in a process, by running the fast tier three times on
that evaluation's cells.  On a regular lattice most cells of the mixed path
are handed to the warp tier (FP32 ties on every bisector), so each trial run
appends most cells to the overflow list: the counters must start from zero
before every trial, or the list would be written past its end.

Each case runs in a fresh process so that the tuner runs on the lattice.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CODE = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
from sdot_b200.power_diagram import PowerDiagram
k = 512
g = (np.arange(k) + 0.5) / k
p = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
n = len(p)
d = PowerDiagram(p, np.zeros(n), precision={prec!r})
d.add_box_shape([0.0, 0.0], [1.0, 1.0])
m = d.integrals()
off, col, val, _ = d.der_integrals_wrt_weights()
ovf = d.last_overflow_count()
# every cell is a square of area 1/n; every Hessian row sums to zero
assert np.abs(m - 1.0 / n).max() <= 1e-12 / n, np.abs(m - 1.0 / n).max() * n
rows = np.repeat(np.arange(n), np.diff(off))
diag = np.zeros(n)
diag[rows[col == rows]] = val[col == rows]
assert (diag > 0).all()
assert np.abs(np.bincount(rows, weights=val, minlength=n)).max() <= 1e-12 * diag.max()
print("lattice ok", n, "overflow", ovf)
"""


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_block_size_tuner_on_a_lattice(cuda_ok, precision):
    from sdot_b200 import build

    build.build()
    r = subprocess.run([sys.executable, "-c", CODE.format(root=ROOT, prec=precision)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "lattice ok" in r.stdout
