"""ctypes binding of libsdot_b200.so (the C ABI of include/sdot_gpu.h).

The shared library is built in-tree by sdot_b200/build.py.  There is no
CPU fallback: if the library is missing or cannot be loaded, importing the
product raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# SDOT_B200_LIB selects another build of the same sources (e.g. a debug build)
LIB_PATH = os.environ.get("SDOT_B200_LIB") or os.path.join(_HERE, "libsdot_b200.so")

SDOT_OK = 0
SDOT_VOID_CELL = 1
SDOT_CAPACITY = 2
SDOT_NOT_CONVERGED = 3
SDOT_ITER_CAP = 4
SDOT_OOM = 5
SDOT_BAD_ARG = 6
SDOT_CUDA_ERROR = 7
SDOT_UNSUPPORTED = 8
SDOT_PENDING = 9
STATUS_NAMES = {0: "OK", 1: "VOID_CELL", 2: "CAPACITY", 3: "NOT_CONVERGED", 4: "ITER_CAP", 5: "OOM",
                6: "BAD_ARG", 7: "CUDA_ERROR", 8: "UNSUPPORTED", 9: "PENDING"}

SDOT_HOST = 0
SDOT_DEVICE = 1
SDOT_FP64 = 0
SDOT_MIXED = 1


class SdotOptions(ctypes.Structure):
    _fields_ = [("max_diracs_per_cell", ctypes.c_int64), ("stream", ctypes.c_void_p), ("device", ctypes.c_int)]


class SdotNewtonOptions(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int),
        ("rel_mass_tol", ctypes.c_double),
        ("pcg_max_iter", ctypes.c_int),
        ("pcg_rel_tol", ctypes.c_double),
        ("damping", ctypes.c_int),
        ("verbosity", ctypes.c_int),
        ("preconditioner", ctypes.c_int),
        ("pcg_fp32", ctypes.c_int),
    ]


class SdotNewtonReport(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("pcg_iterations", ctypes.c_int64),
        ("max_rel_mass_error", ctypes.c_double),
        ("min_mass", ctypes.c_double),
        ("time_ms", ctypes.c_double),
        ("evaluations", ctypes.c_int),
        ("pcg_levels", ctypes.c_int),
    ]


class SdotServerOptions(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_int64), ("device", ctypes.c_int),
                ("newton", SdotNewtonOptions)]


class SdotRequestReport(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("submit_ms", ctypes.c_double), ("start_ms", ctypes.c_double),
                ("end_ms", ctypes.c_double), ("iterations", ctypes.c_int), ("max_rel_mass_error", ctypes.c_double)]


_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.c_int64

# name -> (restype, argtypes); every symbol here must be declared in include/sdot_gpu.h
SIGNATURES = {
    "sdot_create": (_P, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(SdotOptions)]),
    "sdot_destroy": (None, [_P]),
    "sdot_last_error": (ctypes.c_char_p, [_P]),
    "sdot_set_diracs": (ctypes.c_int, [_P, _P, _P, _I64, ctypes.c_int]),
    "sdot_set_weights": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "sdot_add_box_shape": (ctypes.c_int, [_P, _P, _P, ctypes.c_double]),
    "sdot_add_convex_polyhedron_shape": (ctypes.c_int, [_P, _P, _P, _I64, ctypes.c_double]),
    "sdot_add_simplex_shape": (ctypes.c_int, [_P, _P, ctypes.c_double]),
    "sdot_set_image_density": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int]),
    "sdot_set_polynomial_density": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "sdot_clear_domain": (ctypes.c_int, [_P]),
    "sdot_set_stream": (ctypes.c_int, [_P, _P]),
    "sdot_normalize_domain": (ctypes.c_int, [_P]),
    "sdot_domain_measure": (ctypes.c_int, [_P, _P]),
    "sdot_set_ball_cut": (ctypes.c_int, [_P, ctypes.c_int]),
    "sdot_set_translations": (ctypes.c_int, [_P, _P, _I64]),
    "sdot_get_integrals": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "sdot_get_centroids": (ctypes.c_int, [_P, _P, _P, ctypes.c_int]),
    "sdot_get_der_integrals_wrt_weights": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int]),
    "sdot_get_neighbors": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int]),
    "sdot_get_image_integrals": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int]),
    "sdot_get_der_centroids_and_integrals_wrt_weight_and_positions": (ctypes.c_int, [_P, _P, _P, _P, _P, _P,
                                                                                     ctypes.c_int]),
    "sdot_get_image_of_cell_nums": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int]),
    "sdot_solve": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.POINTER(SdotNewtonOptions),
                                  ctypes.POINTER(SdotNewtonReport)]),
    "sdot_get_weights": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "sdot_csr_solve": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_int, _P, _P, ctypes.c_char_p, _I64]),
    "sdot_csr_solve_noalloc": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                              _P, _P, _P, ctypes.c_char_p, _I64]),
    "sdot_server_create": (_P, [ctypes.POINTER(SdotServerOptions)]),
    "sdot_server_submit": (_I64, [_P, ctypes.c_int, _I64, _P, _P, _P, _P, _P]),
    "sdot_server_poll": (ctypes.c_int, [_P, _I64, _P, ctypes.POINTER(SdotRequestReport)]),
    "sdot_server_drain": (ctypes.c_int, [_P]),
    "sdot_server_destroy": (None, [_P]),
    "sdot_evaluate": (ctypes.c_int, [_P]),
    "sdot_last_timings": (ctypes.c_int, [_P, _P]),
    "sdot_last_overflow_count": (ctypes.c_int, [_P, _P]),
    "sdot_kernel_launches": (ctypes.c_int, [_P]),
    "sdot_measure_fma_peaks": (ctypes.c_int, [_P]),
    "sdot_debug_checks": (ctypes.c_int, [_P]),
    "sdot_debug_work_counts": (ctypes.c_int, [_P, ctypes.c_int]),
}

_lib = None


def load():
    """Load libsdot_b200.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libsdot_b200.so is not built (run `python -m sdot_b200.build`); the power-diagram path has no CPU fallback"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class SdotError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"sdot: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status
