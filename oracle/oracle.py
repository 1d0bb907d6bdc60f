"""ctypes wrapper of the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: the checker the CUDA path is compared against. Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this module.

The oracle restates ImpressionFEA.Core's forging path in C (see ``ifea_oracle.h``); this module only moves
arrays in and out. Parity pin: the reference's analytic known-answer tests (tests/test_oracle_kat.py).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from build_oracle import build_oracle  # noqa: F401  (only when run from this folder)
        _LIB = C.CDLL(path)
        _declare(_LIB)
    return _LIB


class O3DParams(C.Structure):
    _fields_ = [("C", C.c_double), ("N", C.c_double), ("M", C.c_double), ("eps0", C.c_double),
                ("friction", C.c_double), ("ram", C.c_double), ("h", C.c_double), ("ds", C.c_double),
                ("tol", C.c_double), ("max_iter", C.c_int), ("auto_step", C.c_int), ("max_cutbacks", C.c_int),
                ("remesh_quality", C.c_double), ("size", C.c_double), ("sym_x", C.c_int), ("sym_y", C.c_int),
                ("sym_factor", C.c_int), ("penalty_factor", C.c_double), ("newton_blend", C.c_double),
                ("quadratic_ls", C.c_int), ("extrapolate_start", C.c_int), ("adaptive_newton", C.c_int),
                ("sticky_secant", C.c_int), ("pcg_budget", C.c_int)]


class O2DParams(C.Structure):
    _fields_ = [("C", C.c_double), ("N", C.c_double), ("M", C.c_double), ("eps0", C.c_double),
                ("friction", C.c_double), ("ram", C.c_double), ("ds", C.c_double), ("tol", C.c_double),
                ("max_iter", C.c_int), ("axisymmetric", C.c_int), ("length", C.c_double), ("radius", C.c_double),
                ("height", C.c_double), ("nx", C.c_int), ("nz", C.c_int)]


REMESH_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)


def _declare(L):
    vp, dp, ip, i32p, u8p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int32), C.POINTER(C.c_uint8)
    i64p = C.POINTER(C.c_int64)
    sig = {
        "o3d_create": (vp, [C.POINTER(O3DParams)]), "o3d_destroy": (None, [vp]), "o3d_error": (C.c_char_p, [vp]),
        "o3d_set_mesh": (C.c_int, [vp, C.c_int, C.c_int, dp, i32p, u8p, u8p]),
        "o3d_set_die": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp]),
        "o3d_init": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
        "o3d_step": (C.c_int, [vp]), "o3d_prepare_step": (C.c_int, [vp]),
        "o3d_assemble": (C.c_double, [vp, C.c_int, C.c_int, dp, dp]),
        "o3d_apply_bc": (C.c_int, [vp, dp]), "o3d_solve_velocity": (C.c_int, [vp, ip]),
        "o3d_final_evaluation": (C.c_double, [vp, dp]), "o3d_try_update": (C.c_int, [vp, C.c_double, ip]),
        "o3d_set_warm": (None, [vp, C.c_int]), "o3d_array": (vp, [vp, C.c_char_p, i64p]),
        "o3d_scalar": (C.c_double, [vp, C.c_char_p]), "o3d_set_scalar": (C.c_int, [vp, C.c_char_p, C.c_double]),
        "o3d_die_project": (C.c_double, [vp, C.c_int, dp, C.c_double, dp, dp]),
        "o3d_die_clearance": (C.c_double, [vp, C.c_int, dp, C.c_double]),
        "o3d_set_trimesh_die": (C.c_int, [vp, C.c_int, C.c_int, dp, C.c_int, i32p]),
        "o3d_die_height": (C.c_double, [vp, C.c_int, C.c_double, C.c_double]),
        "o3d_tet_quality": (C.c_double, [dp, dp, dp, dp]),
        "o3d_set_remesher": (None, [vp, REMESH_FN, vp]),
        "o3d_replace_mesh": (C.c_int, [vp, C.c_int, C.c_int, dp, i32p, u8p, u8p, u8p, dp, dp, dp, dp, dp, dp]),
        "o_flow_stress": (C.c_double, [C.c_double] * 6),
        "o_principal_max3": (C.c_double, [C.c_double] * 6),
        "ospd_create": (vp, []), "ospd_destroy": (None, [vp]),
        "ospd_analyze": (C.c_int, [vp, C.c_int, i32p, i32p]), "ospd_factorize": (C.c_int, [vp, dp]),
        "ospd_solve": (C.c_int, [vp, dp, dp]), "ospd_factor_nonzeros": (C.c_int64, [vp]),
        "ospd_bad_pivot": (C.c_int, [vp]),
        "ospd_set_geometry": (None, [vp, C.c_int, dp]),
        "oband_create": (vp, [C.c_int, C.c_int]), "oband_destroy": (None, [vp]), "oband_bandwidth": (C.c_int, [vp]),
        "oband_add": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]), "oband_get": (C.c_double, [vp, C.c_int, C.c_int]),
        "oband_constrain": (None, [vp, C.c_int]), "oband_clear": (None, [vp]),
        "oband_factorize": (C.c_int, [vp, dp]), "oband_solve": (C.c_int, [vp, dp]),
        "oband_data": (dp, [vp, i64p]),
        "o2d_create": (vp, [C.POINTER(O2DParams), C.c_int, dp, C.c_int, dp]), "o2d_destroy": (None, [vp]),
        "o2d_error": (C.c_char_p, [vp]), "o2d_step": (C.c_int, [vp]), "o2d_prepare": (C.c_int, [vp]),
        "o2d_assemble": (C.c_double, [vp, C.c_int, C.c_int, dp, dp]),
        "o2d_solve_velocity": (C.c_int, [vp, C.c_int, ip]), "o2d_final_evaluation": (C.c_double, [vp, dp]),
        "o2d_array": (vp, [vp, C.c_char_p, i64p]), "o2d_scalar": (C.c_double, [vp, C.c_char_p]),
        "o2d_die_project": (C.c_double, [dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp]),
        "o2d_die_height": (C.c_double, [dp, C.c_int, C.c_double]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_DTYPES_3D = {"contact": np.uint8, "release": np.uint8, "fixed": np.uint8, "bsym": np.uint8, "is_surface": np.uint8,
              "n_fix": np.int32, "die_axis": np.int32, "g_start": np.int32, "g_node": np.int32, "col_ptr": np.int32,
              "row_idx": np.int32, "nbr_start": np.int32, "nbr": np.int32, "e_nbr": np.int32, "bface": np.int32,
              "bowner": np.int32, "tets": np.int32}
_DTYPES_2D = {"contact": np.uint8, "release": np.uint8, "rotated": np.uint8, "fixed": np.uint8, "is_axis": np.uint8,
              "conn": np.int32, "eq": np.int32, "loop": np.int32, "loop_owner": np.int32}


def _view(ptr, count, dtype):
    if not ptr or count == 0:
        return np.zeros(0, dtype)
    ct = np.ctypeslib.as_ctypes_type(np.dtype(dtype))
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(count,)).copy()


class Oracle3D:
    """Forging3DSolver restated on the CPU (ThreeD/Forging3DSolver.cs)."""

    def __init__(self, cfg, mesh, dies):
        L = lib()
        p = O3DParams(cfg.C, cfg.N, cfg.M, cfg.eps0, cfg.friction, cfg.ram, cfg.h, cfg.ds, cfg.tol, cfg.max_iter,
                      int(cfg.auto_step), cfg.max_cutbacks, cfg.remesh_quality, cfg.size, int(cfg.sym_x),
                      int(cfg.sym_y), cfg.sym_factor, cfg.penalty_factor, cfg.newton_blend, int(cfg.quadratic_ls),
                      int(cfg.extrapolate_start), int(cfg.adaptive_newton), int(cfg.sticky_secant), cfg.pcg_budget)
        self.L = L
        self.p = cfg
        self.h = L.o3d_create(C.byref(p))
        x = np.ascontiguousarray(mesh.x, np.float64)
        t = np.ascontiguousarray(mesh.tets, np.int32)
        ox = np.ascontiguousarray(mesh.on_x0, np.uint8)
        oy = np.ascontiguousarray(mesh.on_y0, np.uint8)
        self._check(L.o3d_set_mesh(self.h, len(x), len(t), _dp(x), t.ctypes.data_as(C.POINTER(C.c_int32)),
                                   ox.ctypes.data_as(C.POINTER(C.c_uint8)), oy.ctypes.data_as(C.POINTER(C.c_uint8))))
        for side, d in enumerate(dies):
            if hasattr(d, "triangles"):
                v = np.ascontiguousarray(d.vertices, np.float64)
                tr = np.ascontiguousarray(d.triangles, np.int32)
                self._check(L.o3d_set_trimesh_die(self.h, side, len(v), _dp(v), len(tr), tr.ctypes.data_as(C.POINTER(C.c_int32))))
            else:
                hh = np.ascontiguousarray(d.h, np.float64)
                self._check(L.o3d_set_die(self.h, side, d.nx, d.ny, d.x0, d.y0, d.dx, _dp(hh)))
        self._check(L.o3d_init(self.h, mesh.gap0, *mesh.bounds_for_velocity))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}: {self.L.o3d_error(self.h).decode()}")
        return rc

    def close(self):
        if self.h:
            self.L.o3d_destroy(self.h)
            self.h = None

    __del__ = close

    def step(self):
        return self._check(self.L.o3d_step(self.h))

    def try_step(self):
        rc = self.L.o3d_step(self.h)
        return rc, self.L.o3d_error(self.h).decode()

    def prepare_step(self):
        return self._check(self.L.o3d_prepare_step(self.h))

    def assemble(self, matrix, newton, v):
        v = np.ascontiguousarray(v, np.float64)
        pw = C.c_double()
        e = self.L.o3d_assemble(self.h, int(matrix), int(newton), _dp(v), C.byref(pw))
        return e, pw.value

    def apply_bc(self):
        md = C.c_double()
        self.L.o3d_apply_bc(self.h, C.byref(md))
        return md.value

    def solve_velocity(self):
        conv = C.c_int()
        it = self.L.o3d_solve_velocity(self.h, C.byref(conv))
        if it < 0:
            raise RuntimeError(self.L.o3d_error(self.h).decode())
        return it, bool(conv.value)

    def final_evaluation(self):
        r = C.c_double()
        p = self.L.o3d_final_evaluation(self.h, C.byref(r))
        return p, r.value

    def try_update(self, dt):
        ok = C.c_int()
        self.L.o3d_try_update(self.h, dt, C.byref(ok))
        return bool(ok.value)

    def set_warm(self, w):
        self.L.o3d_set_warm(self.h, int(w))

    def array(self, name):
        n = C.c_int64()
        ptr = self.L.o3d_array(self.h, name.encode(), C.byref(n))
        return _view(ptr, n.value, _DTYPES_3D.get(name, np.float64))

    def scalar(self, name):
        return self.L.o3d_scalar(self.h, name.encode())

    def set_scalar(self, name, v):
        return self.L.o3d_set_scalar(self.h, name.encode(), float(v))

    def enable_remesh(self, dies):
        """Remesh where the reference's Step remeshes, with the library's host remesher (the same host code the GPU
        stepper calls: RemeshCore, ThreeD/Forging3DSolver.cs:1958-2101): the oracle restates the per-iteration path
        only, and the remesh sits outside it on the host in both."""
        from impressionfea_b200 import _lib

        G = _lib.lib()
        vol_target = self.scalar("vol0") / self.p.sym_factor
        if any(hasattr(d, "triangles") for d in dies):
            raise NotImplementedError("the oracle remeshes with height-field dies only")
        self._die_keep = [np.ascontiguousarray(d.h, np.float64) for d in dies]
        grids = [_lib.DieGrid(d.nx, d.ny, d.x0, d.y0, d.dx, hh.ctypes.data_as(C.POINTER(C.c_double)))
                 for d, hh in zip(dies, self._die_keep)]

        def cb(_user, _s):
            f64 = lambda nm: np.ascontiguousarray(self.array(nm), np.float64)
            x, vg, eps, dmg, sig, rate, mean = (f64(n) for n in ("x", "vg", "eps", "dmg", "el_sig", "el_rate", "el_mean"))
            tets = np.ascontiguousarray(self.array("tets"), np.int32)
            hot = np.ascontiguousarray(self.array("hot"), np.float64)
            dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
            args = _lib.RemeshArgs(int(len(x) // 3), int(len(tets) // 4), dp(x), tets.ctypes.data_as(C.POINTER(C.c_int32)),
                                   dp(vg), dp(eps), dp(dmg), dp(sig), dp(rate), dp(mean), grids[0], grids[1],
                                   self.scalar("gap"), self.scalar("h"), vol_target, int(self.p.sym_x), int(self.p.sym_y),
                                   int(self.scalar("recovery_pass")), int(self.scalar("refinement_levels")),
                                   int(self.scalar("max_nodes")), self.scalar("sig_ref"), len(hot) // 4, dp(hot))
            r = C.c_void_p()
            st = G.ifea_remesh_workpiece(C.byref(args), C.byref(r))
            try:
                if st != 0:
                    return 0
                nn, ne = G.ifea_remesh_node_count(r), G.ifea_remesh_tet_count(r)
                out = {k: np.zeros(n, t) for k, n, t in (("x", 3 * nn, np.float64), ("tets", 4 * ne, np.int32),
                                                         ("onx", nn, np.uint8), ("ony", nn, np.uint8), ("contact", nn, np.uint8),
                                                         ("vg", 3 * nn, np.float64), ("eps", ne, np.float64), ("dmg", ne, np.float64),
                                                         ("sig", ne, np.float64), ("rate", ne, np.float64), ("mean", ne, np.float64))}
                ptr = lambda a: a.ctypes.data_as(C.POINTER(np.ctypeslib.as_ctypes_type(a.dtype)))
                G.ifea_remesh_get(r, *(ptr(out[k]) for k in ("x", "tets", "onx", "ony", "contact", "vg", "eps", "dmg", "sig", "rate", "mean")))
                rc = self.L.o3d_replace_mesh(self.h, nn, ne, ptr(out["x"]), ptr(out["tets"]), ptr(out["onx"]), ptr(out["ony"]),
                                             ptr(out["contact"]), ptr(out["vg"]), ptr(out["eps"]), ptr(out["dmg"]),
                                             ptr(out["sig"]), ptr(out["rate"]), ptr(out["mean"]))
                return 1 if rc == 0 else 0
            finally:
                G.ifea_remesh_destroy(r)

        self._remesh_cb = REMESH_FN(cb)
        self.L.o3d_set_remesher(self.h, self._remesh_cb, None)

    def die_project(self, side, p, offset):
        p = np.ascontiguousarray(p, np.float64)
        q = np.zeros(3)
        n = np.zeros(3)
        d = self.L.o3d_die_project(self.h, side, _dp(p), offset, _dp(q), _dp(n))
        return q, n, d

    def die_clearance(self, side, p, offset):
        p = np.ascontiguousarray(p, np.float64)
        return self.L.o3d_die_clearance(self.h, side, _dp(p), offset)

    def die_height(self, side, x, y):
        return self.L.o3d_die_height(self.h, side, float(x), float(y))


class OracleSpd:
    """Oracle ISpdSolver backend: supernodal multifrontal Cholesky (stand-in for MKL PARDISO / CSparse.NET)."""

    def __init__(self):
        self.L = lib()
        self.h = self.L.ospd_create()

    def set_geometry(self, xyz):
        """Node coordinates (3 per node) for the coordinate nested-dissection order of the next analysis."""
        self._xyz = np.ascontiguousarray(xyz, np.float64)
        self.L.ospd_set_geometry(self.h, len(self._xyz) // 3, _dp(self._xyz))

    def analyze(self, n, col_ptr, row_idx):
        self._cp = np.ascontiguousarray(col_ptr, np.int32)
        self._ri = np.ascontiguousarray(row_idx, np.int32)
        return self.L.ospd_analyze(self.h, n, self._cp.ctypes.data_as(C.POINTER(C.c_int32)),
                                   self._ri.ctypes.data_as(C.POINTER(C.c_int32)))

    def factorize(self, values):
        v = np.ascontiguousarray(values, np.float64)
        return self.L.ospd_factorize(self.h, _dp(v))

    def solve(self, b):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b)
        rc = self.L.ospd_solve(self.h, _dp(b), _dp(x))
        if rc != 0:
            raise RuntimeError("oracle solve failed")
        return x

    @property
    def factor_nonzeros(self):
        return self.L.ospd_factor_nonzeros(self.h)

    @property
    def bad_pivot(self):
        return self.L.ospd_bad_pivot(self.h)

    def close(self):
        if self.h:
            self.L.ospd_destroy(self.h)
            self.h = None

    __del__ = close


class OracleBand:
    """SymmetricBandMatrix restated (Solver/SymmetricBandMatrix.cs)."""

    def __init__(self, n, bw):
        self.L = lib()
        self.h = self.L.oband_create(n, bw)
        self.n = n

    @property
    def bandwidth(self):
        return self.L.oband_bandwidth(self.h)

    def add(self, i, j, v):
        if self.L.oband_add(self.h, i, j, v) != 0:
            raise ValueError(f"Entry ({i},{j}) lies outside the bandwidth {self.bandwidth}.")

    def get(self, i, j):
        return self.L.oband_get(self.h, i, j)

    def constrain(self, i):
        self.L.oband_constrain(self.h, i)

    def factorize(self):
        piv = C.c_double()
        row = self.L.oband_factorize(self.h, C.byref(piv))
        return row, piv.value

    def solve(self, rhs):
        rhs = np.array(rhs, np.float64)
        self.L.oband_solve(self.h, _dp(rhs))
        return rhs

    def data(self):
        n = C.c_int64()
        ptr = self.L.oband_data(self.h, C.byref(n))
        return _view(ptr, n.value, np.float64)

    def set_data(self, a):
        """Overwrite the stored band (row-wise lower band, n * (b + 1) values) in one copy."""
        n = C.c_int64()
        ptr = self.L.oband_data(self.h, C.byref(n))
        a = np.ascontiguousarray(a, np.float64)
        if a.size != n.value:
            raise ValueError(f"band of {a.size} values, the matrix stores {n.value}")
        C.memmove(ptr, a.ctypes.data, a.nbytes)

    def close(self):
        if self.h:
            self.L.oband_destroy(self.h)
            self.h = None

    __del__ = close


class Oracle2D:
    """ForgingSolver restated on the CPU (Solver/ForgingSolver.cs)."""

    def __init__(self, cfg):
        L = lib()
        self.L = L
        p = O2DParams(cfg.C, cfg.N, cfg.M, cfg.eps0, cfg.friction, cfg.ram, cfg.ds, cfg.tol, cfg.max_iter,
                      int(cfg.axisymmetric), cfg.length, cfg.radius, cfg.height, cfg.nx, cfg.nz)
        b = np.ascontiguousarray(cfg.bottom_profile, np.float64).ravel()
        t = np.ascontiguousarray(cfg.top_profile, np.float64).ravel()
        self.h = L.o2d_create(C.byref(p), len(b) // 2, _dp(b), len(t) // 2, _dp(t))
        err = L.o2d_error(self.h).decode()
        if err:
            raise RuntimeError(err)

    def step(self):
        rc = self.L.o2d_step(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle 2D error {rc}: {self.L.o2d_error(self.h).decode()}")

    def prepare(self):
        self.L.o2d_prepare(self.h)

    def assemble(self, matrix, newton, v):
        v = np.ascontiguousarray(v, np.float64)
        pw = C.c_double()
        e = self.L.o2d_assemble(self.h, int(matrix), int(newton), _dp(v), C.byref(pw))
        return e, pw.value

    def solve_velocity(self, picard_fallback=False):
        conv = C.c_int()
        it = self.L.o2d_solve_velocity(self.h, int(picard_fallback), C.byref(conv))
        if it < 0:
            raise RuntimeError(self.L.o2d_error(self.h).decode())
        return it, bool(conv.value)

    def final_evaluation(self):
        r = C.c_double()
        p = self.L.o2d_final_evaluation(self.h, C.byref(r))
        return p, r.value

    def array(self, name):
        n = C.c_int64()
        ptr = self.L.o2d_array(self.h, name.encode(), C.byref(n))
        return _view(ptr, n.value, _DTYPES_2D.get(name, np.float64))

    def scalar(self, name):
        return self.L.o2d_scalar(self.h, name.encode())

    def close(self):
        if self.h:
            self.L.o2d_destroy(self.h)
            self.h = None

    __del__ = close


def die2_project(points, side, p, offset):
    pts = np.ascontiguousarray(points, np.float64).ravel()
    q = [C.c_double() for _ in range(4)]
    d = lib().o2d_die_project(_dp(pts), len(pts) // 2, side, p[0], p[1], offset, *[C.byref(v) for v in q])
    return (q[0].value, q[1].value), (q[2].value, q[3].value), d


def die2_height(points, x):
    pts = np.ascontiguousarray(points, np.float64).ravel()
    return lib().o2d_die_height(_dp(pts), len(pts) // 2, x)


def flow_stress(C_, N, M, eps0, strain, rate):
    return lib().o_flow_stress(C_, N, M, eps0, strain, rate)


def principal_max3(*a):
    return lib().o_principal_max3(*a)


def tet_quality(a, b, c, d):
    arr = [np.ascontiguousarray(v, np.float64) for v in (a, b, c, d)]
    return lib().o3d_tet_quality(*[_dp(v) for v in arr])
