"""Snapshot telemetry on the GPU: FillPercent (ThreeD/Forging3DSolver.cs:2174-2185), the share of the closed
cavity's sample points (BuildCavitySamples, :2157-2172) that lie inside the current mesh, counted by the device
point locator. Checked against a brute-force count of the same points in the same tets with the same barycentric
test (TetLocator.Find, ThreeD/TetMesh.cs:198-221): an integer count, so bit-exact."""
import numpy as np
import pytest

from impressionfea_b200.forging3d import Forging3DSolver
from impressionfea_b200.meshes import cavity_samples, gear_blank_outline
from impressionfea_b200.workloads import closed_die_gear_blank

pytestmark = pytest.mark.gpu


def _vol(a, b, c, d):
    # TetMesh.Volume in its own evaluation order: (b - a) . ((c - a) x (d - a)) / 6
    u, v, w = b - a, c - a, d - a
    cx = v[..., 1] * w[..., 2] - v[..., 2] * w[..., 1]
    cy = v[..., 2] * w[..., 0] - v[..., 0] * w[..., 2]
    cz = v[..., 0] * w[..., 1] - v[..., 1] * w[..., 0]
    return (u[..., 0] * cx + u[..., 1] * cy + u[..., 2] * cz) / 6.0


def _inside_count(x, tets, pts):
    inside = np.zeros(len(pts), bool)
    for s in range(0, len(tets), 400):
        t = tets[s:s + 400]
        a, b, c, d = (x[t[:, i]] for i in range(4))
        lo = np.minimum(np.minimum(a, b), np.minimum(c, d))
        hi = np.maximum(np.maximum(a, b), np.maximum(c, d))
        cand = np.all((pts[:, None, :] >= lo[None] - 1e-9) & (pts[:, None, :] <= hi[None] + 1e-9), axis=2)
        pi, ti = np.nonzero(cand & ~inside[:, None])
        if len(pi) == 0:
            continue
        p = pts[pi]
        A, B, C, D = a[ti], b[ti], c[ti], d[ti]
        v = _vol(A, B, C, D)
        b0, b1, b2 = _vol(p, B, C, D) / v, _vol(A, p, C, D) / v, _vol(A, B, p, D) / v
        b3 = 1 - b0 - b1 - b2
        ok = (v > 0) & (b0 >= -1e-9) & (b1 >= -1e-9) & (b2 >= -1e-9) & (b3 >= -1e-9)
        inside[pi[ok]] = True
    return int(inside.sum())


def test_fill_percent_counts_the_cavity_samples_inside_the_mesh():
    cfg, mesh, dies = closed_die_gear_blank(target_tets=5000)
    pts = cavity_samples(dies, gear_blank_outline, 52.0, 52.0)
    s = Forging3DSolver(cfg, mesh, dies)
    s.set_cavity(pts)
    for _ in range(4):
        s.step()
        x = s.array("x").reshape(-1, 3)
        want = 100.0 * _inside_count(x, mesh.tets, pts) / len(pts)
        assert s.fill_percent() == want
    assert 0 < want < 100
    s.close()
