"""The remesher with host arrays: IsosurfaceStuffing.Stuff and TetRefiner.Refine (ThreeD/IsosurfaceStuffing.cs,
ThreeD/TetRefiner.cs) and the whole RemeshCore (ThreeD/Forging3DSolver.cs:1958-2145), run by the library's host
code (csrc/remesh.cu).

The stepper itself remeshes on its own when ``set_scalar("remesh", 1)``; these functions expose the pieces for
building billets, for a host that steps elsewhere, and for tests.
"""
import ctypes as C

import numpy as np

from ._lib import INSIDE_FN, SIZE_FN, DieGrid, RemeshArgs, lib, raise_for


def _take(L, h):
    nn, ne = L.ifea_tetmesh_node_count(h), L.ifea_tetmesh_tet_count(h)
    x = np.zeros((nn, 3))
    t = np.zeros((ne, 4), np.int32)
    raise_for(L.ifea_tetmesh_get(h, x.ctypes.data_as(C.POINTER(C.c_double)), t.ctypes.data_as(C.POINTER(C.c_int32))),
              "ifea_tetmesh_get failed")
    return x, t


def stuff(inside, lo, hi, h, sym_x=False, sym_y=False):
    """Tetrahedral mesh of {p : inside(x, y, z)} within the box [lo, hi] at lattice spacing h: (points, tets)."""
    L = lib()
    cb = INSIDE_FN(lambda x, y, z, _: 1 if inside(x, y, z) else 0)
    lo = np.ascontiguousarray(lo, np.float64)
    hi = np.ascontiguousarray(hi, np.float64)
    hm = C.c_void_p()
    raise_for(L.ifea_tetmesh_stuff(cb, None, lo.ctypes.data_as(C.POINTER(C.c_double)),
                                   hi.ctypes.data_as(C.POINTER(C.c_double)), float(h), int(sym_x), int(sym_y),
                                   C.byref(hm)), "isosurface stuffing failed")
    try:
        return _take(L, hm)
    finally:
        L.ifea_tetmesh_destroy(hm)


def stuff_and_refine(inside, lo, hi, h, size, max_nodes, sym_x=False, sym_y=False):
    """Stuffing at h, then longest-edge bisection to size(x, y, z): (points of the stuffed mesh, its tets,
    refined points, refined tets, edge splits)."""
    L = lib()
    cb = INSIDE_FN(lambda x, y, z, _: 1 if inside(x, y, z) else 0)
    sz = SIZE_FN(lambda x, y, z, _: float(size(x, y, z)))
    lo = np.ascontiguousarray(lo, np.float64)
    hi = np.ascontiguousarray(hi, np.float64)
    hm = C.c_void_p()
    raise_for(L.ifea_tetmesh_stuff(cb, None, lo.ctypes.data_as(C.POINTER(C.c_double)),
                                   hi.ctypes.data_as(C.POINTER(C.c_double)), float(h), int(sym_x), int(sym_y),
                                   C.byref(hm)), "isosurface stuffing failed")
    try:
        x0, t0 = _take(L, hm)
        splits = C.c_int32()
        raise_for(L.ifea_tetmesh_refine(hm, sz, None, int(max_nodes), C.byref(splits)), "refinement failed")
        x1, t1 = _take(L, hm)
        return x0, t0, x1, t1, splits.value
    finally:
        L.ifea_tetmesh_destroy(hm)


def remesh_workpiece(x, tets, vg, eps, dmg, sig, rate, mean, bottom, top, gap, h, vol_target, sym_x=True, sym_y=True,
                     recovery_pass=0, refinement_levels=0, max_nodes=1 << 30, sig_ref=0.0, hot=()):
    """RemeshCore on a deformed workpiece: x (nn, 3), tets (ne, 4), nodal velocity vg (nn, 3) and per-tet eps, dmg,
    sig, rate, mean; bottom/top height-field dies (meshes.HeightField, the top die at its closed place), die gap,
    element size h, the modelled part's initial volume; hot: (x, y, z, level) failure places for local refinement.
    Returns (accepted, why, result) with result a dict of the new x, tets, on_x0, on_y0, contact, vg and the
    remapped element fields (None when the new mesh is rejected)."""
    L = lib()
    P, I32, U8 = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_uint8)
    keep = []

    def dbl(a):
        a = np.ascontiguousarray(a, np.float64)
        keep.append(a)
        return a.ctypes.data_as(P)

    def grid(d):
        return DieGrid(int(d.nx), int(d.ny), float(d.x0), float(d.y0), float(d.dx), dbl(d.h))

    t = np.ascontiguousarray(tets, np.int32)
    hotp = np.ascontiguousarray(np.asarray(hot, np.float64).reshape(-1, 4))
    a = RemeshArgs(len(x), len(t), dbl(x), t.ctypes.data_as(I32), dbl(vg), dbl(eps), dbl(dmg), dbl(sig), dbl(rate),
                   dbl(mean), grid(bottom), grid(top), float(gap), float(h), float(vol_target), int(sym_x), int(sym_y),
                   int(recovery_pass), int(refinement_levels), int(max_nodes), float(sig_ref), len(hotp),
                   hotp.ctypes.data_as(P) if len(hotp) else None)
    out = C.c_void_p()
    st = L.ifea_remesh_workpiece(C.byref(a), C.byref(out))
    try:
        why = (L.ifea_remesh_why(out) or b"").decode() if out.value else ""
        if st == 3:  # IFEA_MESH_DISTORTED: the new mesh was rejected
            return False, why, None
        raise_for(st, "ifea_remesh_workpiece failed: " + why)
        nn, ne = L.ifea_remesh_node_count(out), L.ifea_remesh_tet_count(out)
        r = {"x": np.zeros((nn, 3)), "tets": np.zeros((ne, 4), np.int32), "on_x0": np.zeros(nn, np.uint8),
             "on_y0": np.zeros(nn, np.uint8), "contact": np.zeros(nn, np.uint8), "vg": np.zeros((nn, 3))}
        for k in ("eps", "dmg", "sig", "rate", "mean"):
            r[k] = np.zeros(ne)
        raise_for(L.ifea_remesh_get(out, r["x"].ctypes.data_as(P), r["tets"].ctypes.data_as(I32),
                                    r["on_x0"].ctypes.data_as(U8), r["on_y0"].ctypes.data_as(U8),
                                    r["contact"].ctypes.data_as(U8), r["vg"].ctypes.data_as(P),
                                    *[r[k].ctypes.data_as(P) for k in ("eps", "dmg", "sig", "rate", "mean")]),
                  "ifea_remesh_get failed")
        return True, why, r
    finally:
        if out.value:
            L.ifea_remesh_destroy(out)
