"""ForgingSolver (2D axisymmetric / plane strain) on the B200: host-side mirror of Solver/ForgingSolver.cs over
the C ABI. ``step()`` is ForgingSolver.Advance; the Q4 kernel, band assembly and band Cholesky run on the GPU.
"""
import ctypes as C
import math

import numpy as np

from ._lib import Params2D, StepInfo, lib, raise_for

_DT = {1: np.uint8, 4: np.int32, 8: np.float64}


class ForgingSolver2D:
    def __init__(self, cfg):
        L = lib()
        self._L = L
        self.cfg = cfg
        p = Params2D(cfg.C, cfg.N, cfg.M, cfg.eps0, cfg.friction, cfg.ram, cfg.ds, cfg.tol, cfg.max_iter,
                     int(cfg.axisymmetric), cfg.length, cfg.radius, cfg.height, cfg.nx, cfg.nz)
        b = np.ascontiguousarray(cfg.bottom_profile, np.float64).ravel()
        t = np.ascontiguousarray(cfg.top_profile, np.float64).ravel()
        h = C.c_void_p()
        raise_for(L.ifea2d_create(C.byref(p), len(b) // 2, _dp(b), len(t) // 2, _dp(t), C.byref(h)),
                  "ifea2d_create rejected the configuration")
        self._h = h

    def _check(self, status):
        if status != 0:
            raise_for(status, self._L.ifea2d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.ifea2d_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def TotalStroke(self):
        return self.scalar("gap0")

    @property
    def NominalSteps(self):
        return int(math.ceil(self.scalar("gap0") / self.cfg.ds))

    @property
    def IsFinished(self):
        return self.scalar("gap") <= 1e-9

    def step(self, cancel=None):
        info = StepInfo()
        flag = C.byref(cancel) if cancel is not None else None
        self._check(self._L.ifea2d_step(self._h, C.byref(info), flag))
        return {f: getattr(info, f) for f, _ in StepInfo._fields_}

    def prepare(self):
        self._check(self._L.ifea2d_prepare(self._h))

    def assemble(self, matrix, newton, v=None):
        e, p = C.c_double(), C.c_double()
        vp = None
        if v is not None:
            v = np.ascontiguousarray(v, np.float64)
            vp = _dp(v)
        self._check(self._L.ifea2d_assemble(self._h, int(matrix), int(newton), vp, C.byref(e), C.byref(p)))
        return e.value, p.value

    def solve_velocity(self, picard_fallback=False):
        it, conv = C.c_int32(), C.c_int32()
        self._check(self._L.ifea2d_solve_velocity(self._h, int(picard_fallback), C.byref(it), C.byref(conv)))
        return it.value, bool(conv.value)

    def array(self, name):
        n, b = C.c_int64(), C.c_int32()
        self._check(self._L.ifea2d_array_size(self._h, name.encode(), C.byref(n), C.byref(b)))
        out = np.zeros(n.value, _DT[b.value])
        self._check(self._L.ifea2d_get_array(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), n.value))
        return out

    def scalar(self, name):
        v = C.c_double()
        self._check(self._L.ifea2d_get_scalar(self._h, name.encode(), C.byref(v)))
        return v.value


def band_factor_solve(band, half_bandwidth, rhs):
    """SymmetricBandMatrix.Factorize + Solve on the GPU: returns (L band, x); raises on a non-positive pivot."""
    L = lib()
    a = np.array(band, np.float64).ravel()
    x = np.array(rhs, np.float64).ravel()
    row, piv = C.c_int32(), C.c_double()
    st = L.ifea_band_factor_solve(len(x), half_bandwidth, _dp(a), _dp(x), C.byref(row), C.byref(piv))
    raise_for(st, f"Stiffness matrix not positive definite at equation {row.value} (pivot {piv.value:.3E}).")
    return a, x


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))
