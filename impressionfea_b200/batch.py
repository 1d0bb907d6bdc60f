"""Many independent forging cases stepped together on one GPU, and the launch-parameter tuner (csrc/batch.cpp).

The reference runs independent cases with Parallel.For (ThreeD/MeshConvergence.cs:117). Here every case keeps its
own context (streams, captured graphs); ``ForgingBatch.step`` drives them from a pool of host threads so that the
GPU runs many cases' kernels side by side. ``autotune`` picks the factorisation's tensor-core row threshold and the
solves' multi-CTA front height for a case by timing them, cached per size class.
"""
import ctypes as C

import numpy as np

from ._lib import StepInfo, lib, raise_for


class ForgingBatch:
    def __init__(self, solvers3d=(), solvers2d=(), threads=0):
        L = lib()
        self._L = L
        self.s3, self.s2 = list(solvers3d), list(solvers2d)
        a3 = (C.c_void_p * max(1, len(self.s3)))(*[s._h.value for s in self.s3])
        a2 = (C.c_void_p * max(1, len(self.s2)))(*[s._h.value for s in self.s2])
        h = C.c_void_p()
        raise_for(L.ifea_batch_create(len(self.s3), a3, len(self.s2), a2, int(threads), C.byref(h)), "ifea_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.ifea_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def step(self, increments=1):
        """Advance every case by `increments`; returns (per case a list of step-info dicts, per case status)."""
        n = len(self.s3) + len(self.s2)
        infos = (StepInfo * (n * increments))()
        status = np.zeros(n, np.int32)
        self._L.ifea_batch_step(self._h, int(increments), infos, status.ctypes.data_as(C.POINTER(C.c_int32)))
        out = []
        for c in range(n):
            out.append([{f: getattr(infos[c * increments + k], f) for f, _ in StepInfo._fields_} for k in range(increments)])
        return out, status


def autotune(solver, use_cache=True):
    """Tune a Forging3DSolver's factorisation and solve launch parameters on its next matrix (call after
    set_scalar("factor_fp32", ...)). Returns {"tc_rows", "wide_front_rows", "best_ms"} (best_ms -1: from cache)."""
    L = lib()
    t, w, ms = C.c_double(), C.c_double(), C.c_double()
    solver._check(L.ifea3d_autotune(solver._h, int(use_cache), C.byref(t), C.byref(w), C.byref(ms)))
    return {"tc_rows": t.value, "wide_front_rows": w.value, "best_ms": ms.value}
