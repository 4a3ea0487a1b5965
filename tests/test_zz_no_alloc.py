"""sdot_csr_solve_noalloc (the allocation-free CSR solve) against sdot_csr_solve.

Collected last on purpose (file name): it must pass both alone in a fresh
process and after every other test.  Device buffers are created here by the
test (torch); the entry point itself allocates nothing.
"""
import ctypes

import numpy as np
import pytest

from sdot_b200 import workloads

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the parity tests' relative bound


def hessian_c1(n):
    from sdot_b200.power_diagram import PowerDiagram

    c = workloads.config1(n=n)
    g = PowerDiagram(c["positions"], c["weights"])
    g.add_box_shape([0.0, 0.0], [1.0, 1.0])
    off, col, val, m = g.der_integrals_wrt_weights()
    b = m - 1.0 / n + np.random.default_rng(5).normal(0.0, 1e-6, n)
    return off, col, val, b


def solve_existing(lib, off, col, val, b):
    from sdot_b200._lib import SDOT_HOST

    n = b.shape[0]
    x = np.zeros(n)
    it = ctypes.c_int64(0)
    res = ctypes.c_double(0)
    msg = ctypes.create_string_buffer(256)
    st = lib.sdot_csr_solve(off.ctypes.data, col.ctypes.data, val.ctypes.data, n, b.ctypes.data, x.ctypes.data, 1,
                            1e-13, 20000, SDOT_HOST, ctypes.byref(it), ctypes.byref(res), msg, len(msg))
    assert st == 0, msg.value
    return x


def solve_noalloc(lib, d_off, d_col, d_val, d_b, d_x, n, stream):
    it = ctypes.c_int64(0)
    res = ctypes.c_double(0)
    msg = ctypes.create_string_buffer(256)
    st = lib.sdot_csr_solve_noalloc(d_off.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), n, d_b.data_ptr(),
                                    d_x.data_ptr(), 1, 1e-13, 20000, ctypes.c_void_p(stream), ctypes.byref(it),
                                    ctypes.byref(res), msg, len(msg))
    return st, msg.value.decode(), it.value, res.value


def check_two_calls(gpu_lib, n):
    """Solves one Hessian twice in a row through the allocation-free entry
    point; both results must match sdot_csr_solve, and the second call must
    leave the device's free memory unchanged (an allocation made inside the
    library would not pass through torch's caching allocator, but it would
    show up in cudaMemGetInfo at the driver's granularity)."""
    import torch

    off, col, val, b = hessian_c1(n)
    x_ref = solve_existing(gpu_lib, off, col, val, b)
    dev = torch.device("cuda", 0)
    d_off = torch.from_numpy(off).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    stream = torch.cuda.Stream(device=dev)
    scale = np.abs(x_ref).max()
    d_xs = [torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
    for call in range(2):  # two calls in a row reuse the same scratch
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        st, msg, it, res = solve_noalloc(gpu_lib, d_off, d_col, d_val, d_b, d_xs[call], n, stream.cuda_stream)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info(dev)[0]
        assert st == 0, msg
        assert res <= 1e-13 and it > 0
        if call == 1:
            assert free1 == free0, f"free device memory changed by {free0 - free1} bytes during the call"
        x = d_xs[call].cpu().numpy()
        err = np.abs(x - x_ref).max() / scale
        assert err <= RTOL, f"call {call}: max difference {err:.3e} of max |x|"


def test_noalloc_solve_matches_existing_entry_point(gpu_lib):
    check_two_calls(gpu_lib, 10_000)


def test_noalloc_solve_at_the_row_limit(gpu_lib):
    """n = SDOT_NOALLOC_MAX_ROWS: every work vector of the scratch array in use."""
    check_two_calls(gpu_lib, 65_536)


def test_noalloc_rejects_rows_beyond_the_limit(gpu_lib):
    import torch

    from sdot_b200._lib import SDOT_BAD_ARG

    dev = torch.device("cuda", 0)
    small = torch.zeros(4, dtype=torch.float64, device=dev)
    small_i = torch.zeros(4, dtype=torch.int64, device=dev)
    st, msg, _, _ = solve_noalloc(gpu_lib, small_i, small_i, small, small, small, 65537, 0)
    assert st == SDOT_BAD_ARG
    assert "65536" in msg and "65537" in msg
