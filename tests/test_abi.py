"""The C ABI library loads on a CPU-only machine and exports every entry point
that include/sdot_gpu.h declares (no compute call is made)."""
import ctypes
import os
import re

from sdot_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "sdot_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sdot_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_loads():
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    assert lib is not None


def test_every_declared_symbol_is_exported():
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_the_header():
    assert set(declared_symbols()) == set(_lib.SIGNATURES), "sdot_b200/_lib.py SIGNATURES out of sync with the header"


def test_bad_arguments_fail_loudly_without_gpu():
    lib = _lib.load()
    # a null context is rejected without touching the device
    assert lib.sdot_set_ball_cut(None, 1) == _lib.SDOT_BAD_ARG
    assert lib.sdot_last_error(None) == b"null context"
