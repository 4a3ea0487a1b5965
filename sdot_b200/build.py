"""Build recipe for libsdot_b200.so (sm_100a) -- compiled in-tree with nvcc.

    python -m sdot_b200.build          # or sdot_b200.build.build()

The library is a plain shared object exposing the C ABI declared in
include/sdot_gpu.h; Python binds it with ctypes (sdot_b200/_lib.py).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsdot_b200.so")
SOURCES = ["prims.cu", "tree.cu", "cell2d.cu", "cell3d.cu", "csr.cu", "solve.cu", "api.cu", "server.cu", "peaks.cu",
           "noalloc.cu", "derpos.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_rebuild():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "sdot_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, obj, extra):
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", "-o", obj, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r


def build(force=False, verbose=False, extra=(), lib=None):
    """Compiles every source to an object file (in parallel, one nvcc per
    file), then links the shared library.  lib/extra: another output (e.g.
    the counting build, -DSDOT_COUNT) with extra compiler flags; its objects
    go to a folder of their own."""
    lib = lib or LIB
    if lib == LIB and not force and not needs_rebuild():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(HERE, "_build" if lib == LIB else "_build_" + os.path.basename(lib).split(".")[0])
    os.makedirs(objdir, exist_ok=True)
    jobs = [(os.path.join(CSRC, s), os.path.join(objdir, s.replace(".cu", ".o"))) for s in SOURCES]
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda j: _compile(j[0], j[1], extra), jobs))
    failed = False
    for cmd, r in results:
        if verbose:
            print(" ".join(cmd), flush=True)
        if r.returncode != 0:
            failed = True
            sys.stderr.write(r.stdout + r.stderr)
        elif verbose and (r.stdout or r.stderr):
            sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError("nvcc failed building libsdot_b200.so")
    cmd = [nvcc(), *ARCH, "-shared", "-o", lib + ".tmp", *[o for _, o in jobs]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking " + os.path.basename(lib))
    os.replace(lib + ".tmp", lib)
    return lib


COUNT_LIB = os.path.join(HERE, "libsdot_b200_count.so")


def build_counting(force=False):
    """The counting build (-DSDOT_COUNT): the same library with the work
    counters of the 2D fast tier compiled in (sdot_debug_work_counts)."""
    if not force and os.path.exists(COUNT_LIB) and os.path.getmtime(COUNT_LIB) >= os.path.getmtime(LIB):
        return COUNT_LIB
    return build(force=True, extra=["-DSDOT_COUNT"], lib=COUNT_LIB)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=["-Xptxas", "-v"] if "-v" in sys.argv else [])
