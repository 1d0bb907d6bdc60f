"""Pins the CPU oracle to the reference's own known-answer tests.

The reference cannot run here (C# .NET 10) and stores no golden field vectors; its analytic KATs are the pin:
tests/ImpressionFEA.Core.Tests/SolverVerificationTests.cs:44-113, Solver3DTests.cs:30-49, NumericsTests.cs:8-62.
"""
import math

import numpy as np
import pytest

from impressionfea_b200.config import Forging2DConfig, Forging3DConfig
from impressionfea_b200.meshes import upset_case_3d
from oracle import Oracle2D, Oracle3D, OracleBand, OracleSpd, die2_height, die2_project


def _upset2d(axi, m, shut=30.0):
    # SolverVerificationTests.cs:14-40 (flat dies shut at 30, R=20, H=40, L=50, h=2, ds=0.5, v=40)
    return Forging2DConfig(C=100, N=0, M=0.1, eps0=1, friction=m, ram=40, ds=0.5, tol=1e-5, max_iter=60,
                           axisymmetric=axi, length=50, radius=20, height=40, nx=10, nz=20,
                           bottom_profile=np.array([[0, 0], [200, 0]]), top_profile=np.array([[0, shut], [200, shut]]))


def test_frictionless_axisymmetric_upset_matches_homogeneous_solution():
    # SolverVerificationTests.cs:44-53
    o = Oracle2D(_upset2d(True, 0))
    o.step()
    expected = 100 * 1.0 ** 0.1 * math.pi * 20 * 20
    assert 0.995 <= o.scalar("load") / expected <= 1.005


def test_frictionless_plane_strain_upset_matches_homogeneous_solution():
    # SolverVerificationTests.cs:55-64
    o = Oracle2D(_upset2d(False, 0))
    o.step()
    rate_bar = 2 / math.sqrt(3) * 40.0 / 40.0
    expected = 2 / math.sqrt(3) * 100 * rate_bar ** 0.1 * (2 * 20) * 50
    assert 0.995 <= o.scalar("load") / expected <= 1.005


def test_friction_raises_load_within_upper_bound():
    # SolverVerificationTests.cs:66-78
    o = Oracle2D(_upset2d(True, 0.5))
    o.step()
    frictionless = 100 * math.pi * 400
    avitzur = frictionless * (1 + 0.5 * 40 / (3 * math.sqrt(3) * 40))
    assert o.scalar("load") > 1.01 * frictionless
    assert o.scalar("load") < 1.02 * avitzur


def test_full_upset_conserves_volume_and_reaches_shut_height():
    # SolverVerificationTests.cs:103-113
    o = Oracle2D(_upset2d(True, 0.3))
    while o.scalar("gap") > 1e-9:
        o.step()
    assert abs(o.scalar("gap0") - o.scalar("gap") - 10.0) < 1e-6
    assert abs(100 * (o.scalar("volume") - o.scalar("vol0")) / o.scalar("vol0")) < 0.5
    assert abs(o.array("x").reshape(-1, 2)[:, 1].max() - 30.0) < 1e-3


def test_damage_is_non_negative_and_peaks_at_the_bulge():
    # SolverVerificationTests.cs:80-101
    o = Oracle2D(_upset2d(True, 0.5))
    while o.scalar("gap") > 1e-9:
        o.step()
    d = o.array("dmg")
    x = o.array("x").reshape(-1, 2)
    c = o.array("conn").reshape(-1, 4)
    worst = int(np.argmax(d))
    cx = x[c[worst], 0].mean()
    assert d.min() >= 0
    assert 0.02 <= d[worst] <= 2.0
    assert cx > 0.75 * x[:, 0].max()


def test_3d_frictionless_upset_matches_homogeneous_solution():
    # Solver3DTests.cs:30-49 (quarter model, h=3, R=20, H=40, shut 20, v=40)
    mesh, dies = upset_case_3d(20, 40, 3.0, 20.0)
    cfg = Forging3DConfig(C=100, N=0, M=0.1, eps0=1, friction=0, ram=40, h=3, ds=0.5, size=40)
    o = Oracle3D(cfg, mesh, dies)
    x = o.array("x").reshape(-1, 3)
    t = mesh.tets
    vol = np.einsum("ij,ij->i", x[t[:, 1]] - x[t[:, 0]], np.cross(x[t[:, 2]] - x[t[:, 0]], x[t[:, 3]] - x[t[:, 0]])).sum() / 6
    o.step()
    expected = 100 * (40.0 / 40.0) ** 0.1 * (4 * vol / 40)
    assert 0.99 <= o.scalar("load") / expected <= 1.01


def test_band_cholesky_matches_dense_solution():
    # NumericsTests.cs:8-38 (n=40, bw=5; values from a seeded generator, 10 decimals)
    n, bw = 40, 5
    rng = np.random.default_rng(7)
    dense = np.zeros((n, n))
    band = OracleBand(n, bw)
    for i in range(n):
        for j in range(max(0, i - bw), i):
            v = rng.random() - 0.5
            dense[i, j] = dense[j, i] = v
            band.add(i, j, v)
        dense[i, i] = 4 + rng.random()
        band.add(i, i, dense[i, i])
    x = np.sin(np.arange(n))
    b = dense @ x
    row, _ = band.factorize()
    assert row == -1
    np.testing.assert_allclose(band.solve(b), x, atol=1e-10, rtol=0)


def test_non_positive_definite_matrix_is_reported():
    # NumericsTests.cs:40-48
    m = OracleBand(3, 1)
    m.add(0, 0, 1)
    m.add(1, 1, -1)
    m.add(2, 2, 1)
    row, pivot = m.factorize()
    assert row == 1 and pivot < 0


def test_die_projection_and_clearance():
    # NumericsTests.cs:50-62
    pts = np.array([[0, -10], [10, -10], [11, 0], [30, 0]], float)
    assert abs(die2_height(pts, 5) + 10) < 1e-12
    assert abs(die2_height(pts, 10.5) + 5) < 1e-12
    q, nrm, d = die2_project(pts, 0, (20, -0.2), 0)
    assert abs(q[1]) < 1e-12 and abs(d - 0.2) < 1e-12 and abs(nrm[1] - 1) < 1e-12


def test_oracle_sparse_cholesky_matches_dense():
    rng = np.random.default_rng(3)
    n = 60
    A = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.1)
    A = A + A.T + n * np.eye(n)
    cp = [0]
    ri = []
    for j in range(n):
        rows = np.nonzero(A[:, j])[0]
        ri.extend(rows)
        cp.append(len(ri))
    vals = np.concatenate([A[np.nonzero(A[:, j])[0], j] for j in range(n)])
    f = OracleSpd()
    f.analyze(n, np.array(cp), np.array(ri))
    assert f.factorize(vals) == 0
    b = rng.standard_normal(n)
    np.testing.assert_allclose(f.solve(b), np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)
