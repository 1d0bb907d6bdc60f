"""The triangulated die (TriMeshDie over TriMeshSolid, ThreeD/TriMeshSolid.cs:248-297) in the oracle, against an
independent brute-force restatement: the signed clearance is the distance to the nearest triangle within the
6 mm reach, negative inside the solid; the projection is the nearest point with its triangle's normal; the surface
height is the highest (bottom die) or lowest (top die) crossing of the vertical line. Exact geometry, so the
comparisons are to 1e-12."""
import numpy as np
import pytest

from impressionfea_b200.config import Forging3DConfig
from impressionfea_b200.meshes import TriMeshDie, upset_case_3d
from oracle import Oracle3D


def _closest_on_triangle(p, a, b, c):
    # Ericson, Real-Time Collision Detection, 5.1.5 (Voronoi regions of the triangle)
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0 and d2 <= 0:
        return a
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0 and d4 <= d3:
        return b
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        return a + d1 / (d1 - d3) * ab
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0 and d5 <= d6:
        return c
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        return a + d2 / (d2 - d6) * ac
    va = d3 * d6 - d5 * d4
    if va <= 0 and d4 - d3 >= 0 and d5 - d6 >= 0:
        return b + (d4 - d3) / ((d4 - d3) + (d5 - d6)) * (c - b)
    den = 1.0 / (va + vb + vc)
    return a + ab * (vb * den) + ac * (vc * den)


def _brute(die, p):
    best, q = np.inf, None
    for t in die.triangles:
        a, b, c = die.vertices[t]
        x = _closest_on_triangle(p, a, b, c)
        d = np.linalg.norm(x - p)
        if d < best:
            best, q, n = d, x, np.cross(b - a, c - a)
    return best, q, n / np.linalg.norm(n)


def _case(dies):
    mesh, _ = upset_case_3d(8.0, 16.0, 2.0, 11.0, seed=1)
    cfg = Forging3DConfig(C=150, N=0.1, M=0.12, eps0=0.01, friction=0.3, ram=10, h=2.0, ds=0.2, size=16.0, tol=1e-4)
    return Oracle3D(cfg, mesh, dies)


def test_box_die_clearance_projection_and_height():
    bottom = TriMeshDie.box((-30, -30, -10), (30, 30, 0))
    top = TriMeshDie.box((-30, -30, 11), (30, 30, 25))
    o = _case((bottom, top))
    rng = np.random.default_rng(3)
    for p in rng.uniform((-25, -25, -4), (25, 25, 4), (60, 3)):
        d, q, n = _brute(bottom, p)
        c = o.die_clearance(0, p, 0.0)
        inside = p[2] < 0
        want = min(d, 6.0) * (-1 if inside else 1)
        assert abs(c - want) < 1e-12, (p, c, want)
        qo, no, _ = o.die_project(0, p, 0.0)
        if d < 24:
            assert np.allclose(qo, q, atol=1e-12) and np.allclose(no, n, atol=1e-12)
        assert o.die_height(0, p[0], p[1]) == pytest.approx(0.0, abs=1e-12)
    # the top die moved by an offset along z: clearance of a point 1 mm below its face
    assert o.die_clearance(1, np.array([1.0, 2.0, 8.0]), -2.0) == pytest.approx(1.0, abs=1e-12)
    assert o.die_height(1, 3.0, -4.0) == pytest.approx(11.0, abs=1e-12)
    o.close()


def test_shaped_punch_matches_brute_force():
    surf = lambda x, y: 12.0 + 0.05 * (x * x + y * y) ** 0.5 * 2 + 0.3 * np.sin(0.4 * x)
    top = TriMeshDie.grid_block(surf, -20, 20, -20, 20, 24, 30.0, top=True)
    bottom = TriMeshDie.box((-30, -30, -10), (30, 30, 0))
    o = _case((bottom, top))
    rng = np.random.default_rng(4)
    for p in rng.uniform((-15, -15, 7), (15, 15, 16), (80, 3)):
        d, q, n = _brute(top, p)
        c = o.die_clearance(1, p, 0.0)
        zs = o.die_height(1, p[0], p[1])
        inside = p[2] > zs
        want = min(d, 6.0) * (-1 if inside else 1)
        assert abs(c - want) < 1e-12, (p, c, want)
        qo, no, _ = o.die_project(1, p, 0.0)
        assert np.allclose(qo, q, atol=1e-12) and np.allclose(no, n, atol=1e-12)
    o.close()
