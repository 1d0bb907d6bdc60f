"""Forging3DSolver on the B200: the host-side mirror of ThreeD/Forging3DSolver.cs over the C ABI.

Stepping API as in the reference (IForgingStepper, Simulation/SimulationEngine.cs:18-34): ``TotalStroke``,
``NominalSteps``, ``StepIndex``, ``IsFinished``, ``step()``. Each ``step()`` is one increment; the Newton iteration,
assembly, contact and the sparse Cholesky run on the GPU (libifea_gpu.so). Errors raise the exception type the
reference would throw (see _lib.py).
"""
import ctypes as C
import math

import numpy as np

from ._lib import Params3D, StepInfo, lib, raise_for

_DT = {1: np.uint8, 4: np.int32, 8: np.float64}


class Forging3DSolver:
    def __init__(self, cfg, mesh, dies):
        L = lib()
        self._L = L
        p = Params3D(cfg.C, cfg.N, cfg.M, cfg.eps0, cfg.friction, cfg.ram, cfg.h, cfg.ds, cfg.tol, cfg.max_iter,
                     int(cfg.auto_step), cfg.max_cutbacks, cfg.remesh_quality, cfg.size, int(cfg.sym_x),
                     int(cfg.sym_y), cfg.sym_factor, cfg.penalty_factor, cfg.newton_blend, int(cfg.quadratic_ls),
                     int(cfg.extrapolate_start), int(cfg.adaptive_newton), int(cfg.sticky_secant), cfg.pcg_budget)
        h = C.c_void_p()
        raise_for(L.ifea3d_create(C.byref(p), C.byref(h)), "ifea3d_create rejected the parameters")
        self._h = h
        self.cfg = cfg
        x = np.ascontiguousarray(mesh.x, np.float64)
        t = np.ascontiguousarray(mesh.tets, np.int32)
        ox = np.ascontiguousarray(mesh.on_x0, np.uint8)
        oy = np.ascontiguousarray(mesh.on_y0, np.uint8)
        self._check(L.ifea3d_set_mesh(h, len(x), len(t), _dp(x), _ip(t), _u8(ox), _u8(oy)))
        for side, d in enumerate(dies):
            if hasattr(d, "triangles"):
                v = np.ascontiguousarray(d.vertices, np.float64)
                t = np.ascontiguousarray(d.triangles, np.int32)
                self._check(L.ifea3d_set_trimesh_die(h, side, len(v), _dp(v), len(t), _ip(t)))
            else:
                hh = np.ascontiguousarray(d.h, np.float64)
                self._check(L.ifea3d_set_die(h, side, d.nx, d.ny, d.x0, d.y0, d.dx, _dp(hh)))
        self._check(L.ifea3d_init(h, mesh.gap0, *mesh.bounds_for_velocity))
        self.nn, self.ne = len(x), len(t)
        self.last_info = None

    def _check(self, status):
        if status != 0:
            raise_for(status, self._L.ifea3d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.ifea3d_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------------- IForgingStepper
    @property
    def TotalStroke(self):
        return self.scalar("gap0")

    @property
    def NominalSteps(self):
        return int(math.ceil(self.scalar("gap0") / self.cfg.ds))

    @property
    def StepIndex(self):
        return int(self.scalar("step_index"))

    @property
    def IsFinished(self):
        return self.scalar("gap") <= 1e-9

    def step(self, cancel=None):
        """One increment (Forging3DSolver.Step); returns the step telemetry as a dict."""
        info = StepInfo()
        flag = C.byref(cancel) if cancel is not None else None
        self._check(self._L.ifea3d_step(self._h, C.byref(info), flag))
        self.last_info = {f: getattr(info, f) for f, _ in StepInfo._fields_}
        return self.last_info

    # ---------------------------------------------------------------- lower-level (teacher-forced parity)
    def prepare_step(self):
        self._check(self._L.ifea3d_prepare_step(self._h))

    def assemble(self, matrix, newton, v=None):
        e, p = C.c_double(), C.c_double()
        vp = None
        if v is not None:
            v = np.ascontiguousarray(v, np.float64)
            vp = _dp(v)
        self._check(self._L.ifea3d_assemble(self._h, int(matrix), int(newton), vp, C.byref(e), C.byref(p)))
        return e.value, p.value

    def apply_bc(self):
        md = C.c_double()
        self._check(self._L.ifea3d_apply_bc(self._h, C.byref(md)))
        return md.value

    def solve_velocity(self):
        it, conv = C.c_int32(), C.c_int32()
        self._check(self._L.ifea3d_solve_velocity(self._h, C.byref(it), C.byref(conv), None))
        return it.value, bool(conv.value)

    def final_evaluation(self):
        p, r = C.c_double(), C.c_double()
        self._check(self._L.ifea3d_final_evaluation(self._h, C.byref(p), C.byref(r)))
        return p.value, r.value

    def try_update(self, dt):
        ok = C.c_int32()
        self._check(self._L.ifea3d_try_update(self._h, dt, C.byref(ok)))
        return bool(ok.value)

    def set_cavity(self, points):
        """Sample points of the closed cavity (meshes.cavity_samples) for fill_percent()."""
        p = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
        self._check(self._L.ifea3d_set_cavity(self._h, len(p), _dp(p)))

    def fill_percent(self):
        """FillPercent of the snapshot (ThreeD/Forging3DSolver.cs:2174-2185): the share of the cavity samples inside
        the current mesh, counted on the GPU."""
        v = C.c_double()
        self._check(self._L.ifea3d_fill_percent(self._h, C.byref(v)))
        return v.value

    def set_stream(self, cuda_stream):
        """Run this context on an external CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self._L.ifea3d_set_stream(self._h, C.c_void_p(int(cuda_stream))))

    def set_warm(self, warm):
        self._check(self._L.ifea3d_set_warm(self._h, int(warm)))

    def pattern(self):
        nnz, ndof = C.c_int64(), C.c_int32()
        self._check(self._L.ifea3d_pattern_size(self._h, C.byref(nnz), C.byref(ndof)))
        cp = np.zeros(ndof.value + 1, np.int32)
        ri = np.zeros(nnz.value, np.int32)
        self._check(self._L.ifea3d_get_pattern(self._h, _ip(cp), _ip(ri)))
        return cp, ri

    def array(self, name):
        n, b = C.c_int64(), C.c_int32()
        self._check(self._L.ifea3d_array_size(self._h, name.encode(), C.byref(n), C.byref(b)))
        out = np.zeros(n.value, _DT[b.value])
        self._check(self._L.ifea3d_get_array(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), n.value))
        return out

    def set_array(self, name, values):
        n, b = C.c_int64(), C.c_int32()
        self._check(self._L.ifea3d_array_size(self._h, name.encode(), C.byref(n), C.byref(b)))
        a = np.ascontiguousarray(values, _DT[b.value]).ravel()
        self._check(self._L.ifea3d_set_array(self._h, name.encode(), a.ctypes.data_as(C.c_void_p), a.size))

    def scalar(self, name):
        v = C.c_double()
        self._check(self._L.ifea3d_get_scalar(self._h, name.encode(), C.byref(v)))
        return v.value

    def die_query(self, side, points, offset=0.0):
        """Clearance, projection, normal and surface height of die `side` (moved by offset along z) at points
        (n, 3), evaluated on the device: returns (clearance[n], projected[n,3], normal[n,3], surface_z[n])."""
        p = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
        n = len(p)
        c, q, nr, z = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
        self._check(self._L.ifea3d_die_query(self._h, int(side), n, _dp(p), float(offset), _dp(c), _dp(q), _dp(nr), _dp(z)))
        return c, q, nr, z

    def set_scalar(self, name, value):
        self._check(self._L.ifea3d_set_scalar(self._h, name.encode(), float(value)))


class GpuSpdSolver:
    """ISpdSolver on the GPU (Solver/Linear/ISpdSolver.cs:24-41): Analyze / Factorize / Solve with host arrays."""

    def __init__(self):
        L = lib()
        self._L = L
        h = C.c_void_p()
        raise_for(L.ifea_spd_create(C.byref(h)), "no CUDA device or library")
        self._h = h

    @property
    def Name(self):
        return self._L.ifea_spd_name(self._h).decode()

    @property
    def FactorNonZeros(self):
        return self._L.ifea_spd_factor_nonzeros(self._h)

    def _check(self, status):
        if status != 0:
            raise_for(status, self._L.ifea_spd_last_error(self._h).decode())

    def analyze(self, n, col_ptr, row_idx):
        self._cp = np.ascontiguousarray(col_ptr, np.int32)
        self._ri = np.ascontiguousarray(row_idx, np.int32)
        self._check(self._L.ifea_spd_analyze(self._h, n, _ip(self._cp), _ip(self._ri)))

    def factorize(self, values):
        v = np.ascontiguousarray(values, np.float64)
        self._check(self._L.ifea_spd_factorize(self._h, _dp(v)))

    def solve(self, b):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b)
        self._check(self._L.ifea_spd_solve(self._h, _dp(b), _dp(x)))
        return x

    def close(self):
        if getattr(self, "_h", None):
            self._L.ifea_spd_destroy(self._h)
            self._h = None

    __del__ = close


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _u8(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))
