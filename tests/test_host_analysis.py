"""Host-side analysis on the CPU: the library's topology builds (mesh3d.cpp, mesh2d.cpp) and multifrontal symbolic
analysis (multifrontal.cpp), compiled with g++ into a small driver (host_analysis_driver.cpp).

- The topology arrays are bit-exact with the oracle's restatement of TetMesh and BuildPattern/BuildAnp
  (ThreeD/TetMesh.cs:18-64, Forging3DSolver.cs:469-515, :774-795, :1248-1261), and the 2D quad mesh's
  connectivity, reverse Cuthill-McKee numbering and boundary loop with the oracle's QuadMesh
  (Mesh/QuadMesh.cs:51-221).
- The symbolic analysis of a 3 x 3 node-block pattern runs on the node graph and expands to equations; in the
  identity order it must reproduce the equation-by-equation analysis (block 1) byte for byte, with a
  self-consistent front layout (every lower-triangle entry scattered exactly once, child rows found in the
  parent front).
"""
import os
import subprocess

import numpy as np
import pytest

from impressionfea_b200.config import Forging2DConfig, Forging3DConfig
from impressionfea_b200.meshes import gear_blank_case_3d, upset_case_3d
from oracle import Oracle2D, Oracle3D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "impressionfea_b200", "csrc")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("host") / "host_analysis_driver")
    cmd = ["g++", "-O2", "-std=c++17", "-I", CSRC, "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "host_analysis_driver.cpp"), os.path.join(CSRC, "mesh3d.cpp"),
           os.path.join(CSRC, "mesh2d.cpp"), os.path.join(CSRC, "multifrontal.cpp"), "-L", os.path.join(CUDA, "lib64"), "-lcusolver",
           "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-pthread", "-o", exe]
    subprocess.check_call(cmd)
    return exe


def _read(path):
    out = {}
    dt = {1: np.uint8, 4: np.int32, 8: np.int64}
    with open(path, "rb") as f:
        while True:
            name = f.read(24)
            if len(name) < 24:
                return out
            eb = int(np.frombuffer(f.read(4), np.int32)[0])
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            out[name.rstrip(b"\0").decode()] = np.frombuffer(f.read(eb * n), dt[eb]).copy()


def _run(driver, tmp_path, mesh, block, order=None):
    mp, op = tmp_path / "mesh.bin", tmp_path / f"out{block}{order or ''}.bin"
    with open(mp, "wb") as f:
        np.array([len(mesh.x), len(mesh.tets)], np.int32).tofile(f)
        np.ascontiguousarray(mesh.x, np.float64).tofile(f)
        np.ascontiguousarray(mesh.tets, np.int32).tofile(f)
        np.ascontiguousarray(mesh.on_x0, np.uint8).tofile(f)
        np.ascontiguousarray(mesh.on_y0, np.uint8).tofile(f)
    subprocess.check_call([driver, str(mp), str(op), str(block)] + ([order] if order else []))
    return _read(op)


def _cases():
    up_mesh, up_dies = upset_case_3d(10.0, 20.0, 2.0, 12.0, seed=1)
    gb_mesh, gb_dies = gear_blank_case_3d(3.0, seed=2)
    # 12.6k nodes: above the size from which the topology and analysis passes run on host threads
    gf_mesh, gf_dies = gear_blank_case_3d(1.2, seed=3)
    return {"upset": (up_mesh, up_dies, 2.0, 20.0), "gear_blank": (gb_mesh, gb_dies, 3.0, 50.0),
            "gear_blank_threaded": (gf_mesh, gf_dies, 1.2, 50.0)}


CASES = _cases()

SYMBOLIC = ("sym_scalars", "perm", "pinv", "c0", "ncol", "m", "parent", "level", "front_off", "idx_start", "idx",
            "relmap_start", "relmap", "uvec_start", "a_dst", "a_src", "a_level_start", "level_start", "level_list",
            "level_pool_start", "ext_start", "ext_child")


@pytest.mark.parametrize("case", sorted(CASES))
def test_topology_is_bit_exact_with_the_oracle(driver, tmp_path, case):
    mesh, dies, h, size = CASES[case]
    got = _run(driver, tmp_path, mesh, 3)
    cfg = Forging3DConfig(C=150, N=0.1, M=0.12, eps0=0.01, friction=0.3, ram=10, h=h, ds=0.2 * h, size=size,
                          tol=1e-6)
    ora = Oracle3D(cfg, mesh, dies)
    ora.prepare_step()  # builds the ANP patches (BuildAnp)
    try:
        for name in ("col_ptr", "row_idx", "nbr_start", "nbr", "e_nbr", "g_start", "g_node", "bface", "bowner",
                     "bsym", "is_surface"):
            np.testing.assert_array_equal(got[name], np.asarray(ora.array(name)).astype(got[name].dtype),
                                          err_msg=name)
    finally:
        ora.close()


@pytest.mark.parametrize("case", sorted(CASES))
def test_nodal_symbolic_analysis_matches_equation_level(driver, tmp_path, case):
    mesh = CASES[case][0]
    nodal = _run(driver, tmp_path, mesh, 3)
    eqn = _run(driver, tmp_path, mesh, 1)
    for name in SYMBOLIC:
        np.testing.assert_array_equal(nodal[name], eqn[name], err_msg=name)


@pytest.mark.parametrize("case", sorted(CASES))
def test_analysis_from_the_topology_node_lists_matches_the_pattern_scan(driver, tmp_path, case):
    # the stepper hands its topology's node lists to the analysis instead of the scan of the 3 x 3 block pattern
    scan = _run(driver, tmp_path, CASES[case][0], 3, "xyz")
    lists = _run(driver, tmp_path, CASES[case][0], 3, "lists")
    for name in SYMBOLIC:
        np.testing.assert_array_equal(lists[name], scan[name], err_msg=name)


@pytest.mark.parametrize("order", [None, "xyz"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_front_layout_is_self_consistent(driver, tmp_path, case, order):
    r = _run(driver, tmp_path, CASES[case][0], 3, order)
    n, nsuper = int(r["sym_scalars"][0]), int(r["sym_scalars"][1])
    perm, pinv, cp, ri = r["perm"], r["pinv"], r["col_ptr"], r["row_idx"]
    assert np.array_equal(np.sort(perm), np.arange(n)) and np.array_equal(pinv[perm], np.arange(n))
    c0, ncol, m, idx, ids = r["c0"], r["ncol"], r["m"], r["idx"], r["idx_start"]
    assert c0[0] == 0 and np.array_equal(c0[1:], (c0 + ncol)[:-1]) and c0[-1] + ncol[-1] == n
    for s in range(nsuper):
        rows = idx[ids[s]:ids[s + 1]]
        assert len(rows) == m[s] and np.all(np.diff(rows) > 0)
        assert np.array_equal(rows[:ncol[s]], np.arange(c0[s], c0[s] + ncol[s]))
        p = r["parent"][s]
        if p >= 0:  # every update row of s sits in the parent's front at the recorded position
            prow = idx[ids[p]:ids[p + 1]]
            rel = r["relmap"][r["relmap_start"][s]:r["relmap_start"][s + 1]]
            assert np.array_equal(prow[rel], rows[ncol[s]:])
    # every entry on or below the diagonal of P A P' is scattered exactly once
    col = np.repeat(np.arange(n), np.diff(cp))
    lower = np.nonzero(pinv[ri] >= pinv[col])[0]
    assert np.array_equal(np.sort(r["a_src"]), lower)
    assert len(np.unique(r["a_dst"])) == len(r["a_dst"])


@pytest.mark.parametrize("nx,nz", [(20, 60), (7, 5), (12, 31)])
def test_quad_numbering_and_boundary_loop_are_bit_exact_with_the_oracle(driver, tmp_path, nx, nz):
    op = tmp_path / "quad.bin"
    subprocess.check_call([driver, "quad", str(nx), str(nz), str(op)])
    got = _read(op)
    ora = Oracle2D(Forging2DConfig(nx=nx, nz=nz))
    try:
        for name in ("conn", "eq", "loop", "loop_owner"):
            np.testing.assert_array_equal(got[name], np.asarray(ora.array(name)).astype(np.int32), err_msg=name)
        assert got["quad_scalars"][3] == ora.scalar("half_band")
    finally:
        ora.close()
    # element matrix entries land in at most one band cell each; every residual entry lands in exactly one DOF
    ne, src = nx * nz, got["cell_src"]
    assert len(np.unique(src)) == len(src) and src.min() >= 0 and src.max() < ne * 64
    assert np.array_equal(np.sort(got["dof_src"]), np.arange(ne * 8))


@pytest.mark.parametrize("case", sorted(CASES))
def test_coordinate_dissection_separates_its_halves(driver, tmp_path, case):
    """Coordinate nested dissection: the order is a permutation of whole node blocks and every supernode's parent is
    eliminated after it (the front layout itself is checked by test_front_layout_is_self_consistent)."""
    r = _run(driver, tmp_path, CASES[case][0], 3, "xyz")
    perm, n = r["perm"], int(r["sym_scalars"][0])
    assert np.array_equal(np.sort(perm), np.arange(n))
    assert np.array_equal(perm.reshape(-1, 3) % 3, np.tile(np.arange(3), (n // 3, 1)))
    assert np.all(perm.reshape(-1, 3)[:, 1] == perm.reshape(-1, 3)[:, 0] + 1)
    parent = r["parent"]
    assert np.all((parent == -1) | (parent > np.arange(len(parent))))
