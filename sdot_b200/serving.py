"""Continuously batched OT solves (the sdot_server_* C ABI).

    srv = Server(slots=4, hbm_budget_bytes=8 << 30)
    rid = srv.submit(positions, target)          # 2D or 3D, unit box by default
    srv.drain()
    weights, report = srv.result(rid)

Each request is one Newton solve (OptimalTransportSolver::solve,
OptimalTransportSolver.tcc:27-119) on its own worker, contexts and CUDA
stream; `slots` requests run at once and their device work overlaps.
slots=1 solves the requests one after the other (the sequential baseline).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import SDOT_OK, SDOT_PENDING, SdotError


class Server:
    def __init__(self, slots=4, hbm_budget_bytes=16 << 30, device=-1, rel_mass_tol=1e-8, max_iter=150,
                 damping=True, pcg_rel_tol=1e-12, pcg_max_iter=20000):
        self._lib = _lib.load()
        newton = _lib.SdotNewtonOptions(int(max_iter), float(rel_mass_tol), int(pcg_max_iter), float(pcg_rel_tol),
                                        int(bool(damping)), 0)
        opt = _lib.SdotServerOptions(int(slots), int(hbm_budget_bytes), int(device), newton)
        self._srv = self._lib.sdot_server_create(ctypes.byref(opt))
        if not self._srv:
            raise SdotError(_lib.SDOT_CUDA_ERROR, "sdot_server_create failed")
        self._n = {}

    def submit(self, positions, target, weights=None, box_lo=None, box_hi=None):
        p = np.ascontiguousarray(positions, dtype=np.float64)
        n, dim = p.shape
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(n)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64).reshape(n)
        lo = None if box_lo is None else np.ascontiguousarray(box_lo, dtype=np.float64)
        hi = None if box_hi is None else np.ascontiguousarray(box_hi, dtype=np.float64)

        def ptr(a):
            return None if a is None else ctypes.c_void_p(a.ctypes.data)

        rid = self._lib.sdot_server_submit(self._srv, dim, n, ptr(p), ptr(w), ptr(t), ptr(lo), ptr(hi))
        if rid < 0:
            raise SdotError(-rid, "sdot_server_submit failed")
        self._n[rid] = n
        return rid

    def poll(self, rid):
        """(done, weights or None, report dict)."""
        w = np.empty(self._n[rid])
        rep = _lib.SdotRequestReport()
        st = self._lib.sdot_server_poll(self._srv, rid, ctypes.c_void_p(w.ctypes.data), ctypes.byref(rep))
        report = {f: getattr(rep, f) for f, _ in rep._fields_}
        if st == SDOT_PENDING:
            return False, None, report
        return True, w, report

    def result(self, rid):
        done, w, report = self.poll(rid)
        if not done:
            raise RuntimeError("request still pending")
        if report["status"] != SDOT_OK:
            raise SdotError(report["status"], f"request {rid} failed")
        return w, report

    def drain(self):
        self._lib.sdot_server_drain(self._srv)

    def close(self):
        if getattr(self, "_srv", None):
            self._lib.sdot_server_destroy(self._srv)
            self._srv = None

    def __del__(self):
        self.close()
