"""Triangulated dies on the GPU (common.cuh tm_*, TriMeshDie over TriMeshSolid, ThreeD/TriMeshSolid.cs:248-297):
the device's clearance, projection and surface height against the oracle's restatement at random points (the same
arithmetic in the same order: equal to the last bit), and increments of an upsetting case between a box and a
shaped punch against the oracle (iteration counts and contact flags equal, loads and velocities to 1e-6)."""
import numpy as np
import pytest

from impressionfea_b200.config import Forging3DConfig
from impressionfea_b200.forging3d import Forging3DSolver
from impressionfea_b200.meshes import HeightField, TriMeshDie, upset_case_3d
from oracle import Oracle3D

pytestmark = pytest.mark.gpu


def _punch():
    surf = lambda x, y: 11.0 + 0.08 * np.hypot(x, y) + 0.3 * np.sin(0.4 * x)
    return TriMeshDie.grid_block(surf, -24, 24, -24, 24, 32, 30.0, top=True)


def _case(dies):
    mesh, _ = upset_case_3d(8.0, 16.0, 1.6, 11.0, seed=7)
    cfg = Forging3DConfig(C=150, N=0.1, M=0.12, eps0=0.01, friction=0.3, ram=10, h=1.6, ds=0.25, size=16.0, tol=1e-4)
    return cfg, mesh, dies


@pytest.mark.parametrize("which", ["box", "punch", "height_field"])
def test_die_queries_match_the_oracle_bit_for_bit(which):
    box = TriMeshDie.box((-30, -30, -10), (30, 30, 0))
    if which == "height_field":
        dies = (HeightField.flat(0.0, 40.0), HeightField.sample(lambda x, y: 11.0 + 0.02 * x * x, -30, 30, -30, 30, 1.0))
    else:
        dies = (box, _punch() if which == "punch" else TriMeshDie.box((-30, -30, 11), (30, 30, 25)))
    cfg, mesh, dies = _case(dies)
    g, o = Forging3DSolver(cfg, mesh, dies), Oracle3D(cfg, mesh, dies)
    rng = np.random.default_rng(11)
    pts = rng.uniform((-20, -20, -3), (20, 20, 14), (400, 3))
    for side, offset in ((0, 0.0), (1, 0.0), (1, -1.5)):
        c, q, n, z = g.die_query(side, pts, offset)
        for k in range(len(pts)):
            assert c[k] == o.die_clearance(side, pts[k], offset), (which, side, k)
            qo, no, _ = o.die_project(side, pts[k], offset)
            assert np.array_equal(q[k], qo) and np.array_equal(n[k], no), (which, side, k)
            zo = o.die_height(side, pts[k, 0], pts[k, 1])
            assert (np.isnan(z[k]) and np.isnan(zo)) or z[k] == zo, (which, side, k)
    g.close()
    o.close()


def test_upsetting_under_a_shaped_punch_tracks_the_oracle():
    cfg, mesh, dies = _case((TriMeshDie.box((-30, -30, -10), (30, 30, 0)), _punch()))
    g, o = Forging3DSolver(cfg, mesh, dies), Oracle3D(cfg, mesh, dies)
    for k in range(4):
        a = g.step()
        o.step()
        assert a["iterations"] == o.scalar("iterations"), f"increment {k + 1}"
        assert abs(a["load"] / o.scalar("load") - 1) < 1e-6, f"increment {k + 1}"
        np.testing.assert_array_equal(g.array("contact"), o.array("contact"), err_msg=f"increment {k + 1}")
        vg, vo = g.array("vg"), o.array("vg")
        assert np.linalg.norm(vg - vo) / np.linalg.norm(vo) < 1e-6, f"increment {k + 1}"
    assert (g.array("contact") == 2).any(), "the punch must be in contact"
    g.close()
    o.close()
