"""The remesher's building blocks with host arrays: IsosurfaceStuffing.Stuff and TetRefiner.Refine
(ThreeD/IsosurfaceStuffing.cs, ThreeD/TetRefiner.cs), run by the library's host code (csrc/remesh.cu).

The stepper itself remeshes on its own when ``set_scalar("remesh", 1)``; these functions expose the two pieces for
building billets and for tests.
"""
import ctypes as C

import numpy as np

from ._lib import INSIDE_FN, SIZE_FN, lib, raise_for


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
