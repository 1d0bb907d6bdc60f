"""The whole host remesh (RemeshCore, ThreeD/Forging3DSolver.cs:1958-2145, csrc/remesh.cu) on a squashed gear-blank
billet between its dies, on the host only (no GPU): the new mesh is accepted, manifold and positively oriented,
keeps the part's volume, is reproducible call to call, and every element field is carried over from the old tet
that the point locator (TetLocator, ThreeD/TetMesh.cs:116-263) must return for the new element's centroid: the
lowest-numbered old tet containing it (the first in its bucket cell, cells list tets in ascending order)."""
import numpy as np

from impressionfea_b200.meshes import gear_blank_case_3d
from impressionfea_b200.remesh import remesh_workpiece


def _volumes(x, t):
    a, b, c, d = (x[t[:, i]] for i in range(4))
    return np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a)) / 6


def _case():
    h = 2.0
    mesh, dies = gear_blank_case_3d(h, seed=5)
    x = np.array(mesh.x, np.float64)
    z0, height = x[:, 2].min(), np.ptp(x[:, 2])
    x[:, 2] = z0 + (x[:, 2] - z0) * 0.95  # 5 % upset, laterally free; the top die follows it down
    gap = mesh.gap0 - 0.05 * height
    t = np.asarray(mesh.tets, np.int32)
    ne = len(t)
    vol = _volumes(x, t).sum()
    vg = np.zeros_like(x)
    vg[:, 2] = -(x[:, 2] - z0) / height
    return h, dies, x, t, vg, vol, ne, gap


def _remesh(h, dies, x, t, vg, vol, ne, gap):
    f = np.arange(ne, dtype=np.float64)
    return remesh_workpiece(x, t, vg, f, f + 0.5, 100.0 + f, np.zeros(ne), np.zeros(ne), dies[0], dies[1], gap=gap,
                            h=h, vol_target=vol, sig_ref=100.0)


def test_remesh_is_accepted_manifold_volume_keeping_and_reproducible():
    case = _case()
    ok, why, r = _remesh(*case)
    assert ok, why
    x, t = r["x"], r["tets"]
    assert len(t) > 0 and t.min() >= 0 and t.max() < len(x)
    assert _volumes(x, t).min() > 0
    assert abs(_volumes(x, t).sum() / case[5] - 1) < 0.02
    f = np.concatenate([t[:, [0, 2, 1]], t[:, [0, 1, 3]], t[:, [0, 3, 2]], t[:, [1, 2, 3]]])
    _, cnt = np.unique(np.sort(f, axis=1), axis=0, return_counts=True)
    assert cnt.max() <= 2
    assert set(np.unique(r["contact"])) <= {0, 1, 2}
    assert np.isfinite(r["vg"]).all()
    ok2, _, r2 = _remesh(*case)
    assert ok2
    for k in r:
        np.testing.assert_array_equal(r[k], r2[k], err_msg=k)


def test_element_fields_come_from_the_lowest_containing_old_tet():
    h, dies, x, t, vg, vol, ne, gap = case = _case()
    ok, why, r = _remesh(*case)
    assert ok, why
    src = r["eps"].astype(np.int64)  # eps of old tet e was e
    np.testing.assert_array_equal(r["dmg"], src + 0.5)
    nx, nt = r["x"], r["tets"]
    cen = nx[nt].mean(axis=1)
    a, b, c, d = (x[t[:, i]] for i in range(4))
    v = _volumes(x, t)
    checked = 0
    for k in range(0, len(nt), max(1, len(nt) // 1500)):  # a sample of about 1,500 new elements
        p = cen[k]
        b0 = np.einsum("ij,ij->i", b - p, np.cross(c - p, d - p)) / 6 / v
        b1 = np.einsum("ij,ij->i", p - a, np.cross(c - a, d - a)) / 6 / v
        b2 = np.einsum("ij,ij->i", b - a, np.cross(p - a, d - a)) / 6 / v
        inside = np.nonzero((v > 0) & (b0 >= -1e-9) & (b1 >= -1e-9) & (b2 >= -1e-9) & (1 - b0 - b1 - b2 >= -1e-9))[0]
        if len(inside) == 0:
            continue  # outside the old mesh: the nearest centroid in the point's cell
        assert src[k] == inside[0], (k, src[k], inside[:5])
        checked += 1
    assert checked > 1000
