"""The remesher's host building blocks (csrc/remesh.cu) against the reference's own tests of them:
StuffingTests.CylinderMeshIsManifoldAccurateAndWellShaped and LocalRefinementIsConformingAndKeepsVolume
(tests/ImpressionFEA.Core.Tests/StuffingTests.cs:8-89), restated with the same shapes, sizes and bounds.
These run on the host only (no GPU)."""
import numpy as np
import pytest

from impressionfea_b200.remesh import stuff, stuff_and_refine


def _volumes(x, t):
    a, b, c, d = (x[t[:, i]] for i in range(4))
    return np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a)) / 6


def _quality(x, t):
    a, b, c, d = (x[t[:, i]] for i in range(4))
    l2 = (((b - a) ** 2).sum(1) + ((c - a) ** 2).sum(1) + ((d - a) ** 2).sum(1) + ((c - b) ** 2).sum(1)
          + ((d - b) ** 2).sum(1) + ((d - c) ** 2).sum(1)) / 6
    return 6 * np.sqrt(2) * _volumes(x, t) / l2 ** 1.5


def _boundary_faces(t):
    f = np.concatenate([t[:, [0, 2, 1]], t[:, [0, 1, 3]], t[:, [0, 3, 2]], t[:, [1, 2, 3]]])
    key = np.sort(f, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    assert cnt.max() <= 2, "a face is shared by more than two tets"
    return f[cnt[inv.ravel()] == 1]


R, HGT = 20.0, 30.0


def _cyl(x, y, z):
    return x * x + y * y < R * R and 0 < z < HGT


@pytest.mark.parametrize("sym_x,sym_y", [(True, True), (False, True), (False, False)])
def test_cylinder_mesh_is_manifold_accurate_and_well_shaped(sym_x, sym_y):
    x, t = stuff(_cyl, (-R, -R, 0), (R, R, HGT), 3.0, sym_x, sym_y)
    exact = np.pi * R * R * HGT / ((2 if sym_x else 1) * (2 if sym_y else 1))
    vol = _volumes(x, t)
    assert (vol > 0).all()
    assert 0.97 <= vol.sum() / exact <= 1.01, vol.sum() / exact
    assert _quality(x, t).min() > 0.05
    for f in _boundary_faces(t):
        p = x[f]
        on_plane = (sym_x and (p[:, 0] == 0).all()) or (sym_y and (p[:, 1] == 0).all())
        if on_plane:
            continue
        for q in p:
            on_x, on_y = sym_x and q[0] == 0, sym_y and q[1] == 0
            dr = abs(np.hypot(q[0], q[1]) - R)
            dz = min(abs(q[2]), abs(q[2] - HGT))
            assert on_x or on_y or min(dr, dz) < 1e-3, f"surface node off the surface: {q}"


@pytest.mark.parametrize("sym", [False, True])
def test_local_refinement_is_conforming_and_keeps_volume(sym):
    h = 4.0
    x0, t0, x, t, splits = stuff_and_refine(_cyl, (-R, -R, 0), (R, R, HGT), h,
                                             lambda px, py, pz: h / 4 if pz < 8 else h, 400000, sym, sym)
    assert splits > 0
    v = _volumes(x, t)
    assert (v > 0).all(), "inverted tet after refinement"
    assert abs(_volumes(x0, t0).sum() - v.sum()) < 5e-7
    _boundary_faces(t)  # manifold: no face shared by more than two tets
    if sym:
        assert (x[:, 0] >= 0).all() and (x[:, 1] >= 0).all()
    assert _quality(x, t).min() > 0.05
    low = x[t].mean(axis=1)[:, 2] < 6
    e = np.stack([x[t[:, i]] - x[t[:, j]] for i in range(4) for j in range(i + 1, 4)], 1)
    longest = np.linalg.norm(e, axis=2).max(axis=1)
    assert longest[low].max() <= 1.05 * h / 4 + 1e-9
