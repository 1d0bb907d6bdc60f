"""Parity of the 3D CUDA path (libifea_gpu.so through the C ABI) with the CPU oracle.

Integer work (pattern, slot maps, contact flags) must be bit-exact. Floating-point work is compared at FP64
tolerances: per-element and per-node arithmetic is written in the reference's order without FMA contraction,
so it agrees to a few ulps (pow() differs between CUDA and glibc); reductions, the factorisation and the PCG
differ in summation order, which the Newton iteration damps to far below the 1e-6 relative bar.
"""
import numpy as np
import pytest

from impressionfea_b200.config import Forging3DConfig
from impressionfea_b200.forging3d import Forging3DSolver, GpuSpdSolver
from impressionfea_b200 import _lib
from impressionfea_b200.meshes import upset_case_3d
from oracle import Oracle3D

pytestmark = pytest.mark.gpu

RTOL_ELEM = 1e-12      # per-element / per-node FP64 arithmetic (a few ulps of pow())
RTOL_ENERGY = 1e-10    # global sums: 1/2 v.K_vol.v cancels the penalty terms, so its summation order shows
RTOL_STATE = 1e-6      # velocity, strain and load over Newton iterations and increments
RTOL_X = 1e-7          # coordinates after increments (moved by dt * velocity)
# effective strain after increments: the time integral of the strain rate, a derivative of the velocity, so on
# this coarse 1.6k-tet mesh it carries about 1.5 times the velocity's relative difference (the published meshes
# hold it to 1e-6: tests/test_gpu_baseline_meshes.py)
RTOL_STRAIN = 3e-6


def _case(friction=0.3, R=10.0, H=20.0, h=2.0, shut=12.0, seed=1):
    mesh, dies = upset_case_3d(R, H, h, shut, seed=seed)
    cfg = Forging3DConfig(C=150, N=0.1, M=0.12, eps0=0.01, friction=friction, ram=10, h=h, ds=0.4 * h * 0.5,
                          size=H, tol=1e-6)
    return cfg, mesh, dies


@pytest.fixture(scope="module")
def pair():
    cfg, mesh, dies = _case()
    return Forging3DSolver(cfg, mesh, dies), Oracle3D(cfg, mesh, dies), cfg, mesh


def _close(a, b, rtol, what):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err <= rtol, f"{what}: max abs diff / max |ref| = {err:.3e} > {rtol:.1e}"

def _close_l2(a, b, rtol, what):
    """Relative L2 error of a field. The converged fields of both paths differ by the PCG stopping point (relative
    residual 1e-7, as in the reference) amplified by the penalty's conditioning, which shows most in single
    elements: the field-level bar is taken in the L2 norm."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    err = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    assert err <= rtol, f"{what}: relative L2 error {err:.3e} > {rtol:.1e}"



def test_pattern_and_slot_maps_are_bit_exact(pair):
    gpu, ora, _, _ = pair
    cp, ri = gpu.pattern()
    np.testing.assert_array_equal(cp, ora.array("col_ptr"))
    np.testing.assert_array_equal(ri, ora.array("row_idx"))
    np.testing.assert_array_equal(gpu.array("nbr_start"), ora.array("nbr_start"))
    np.testing.assert_array_equal(gpu.array("nbr"), ora.array("nbr"))
    np.testing.assert_array_equal(gpu.array("e_nbr"), ora.array("e_nbr"))
    np.testing.assert_array_equal(gpu.array("bface"), ora.array("bface"))
    np.testing.assert_array_equal(gpu.array("is_surface"), ora.array("is_surface"))


def test_initial_contact_and_placement(pair):
    gpu, ora, _, _ = pair
    np.testing.assert_array_equal(gpu.array("contact"), ora.array("contact"))
    np.testing.assert_array_equal(gpu.array("x"), ora.array("x"))
    _close(gpu.array("vg"), ora.array("vg"), 0, "initial velocity")
    _close(gpu.array("h_local"), ora.array("h_local"), 0, "local lengths")
    assert abs(gpu.scalar("vol0") / ora.scalar("vol0") - 1) < 1e-13


def test_prepare_step_matches(pair):
    gpu, ora, _, _ = pair
    gpu.prepare_step()
    ora.prepare_step()
    np.testing.assert_array_equal(gpu.array("fixed"), ora.array("fixed"))
    np.testing.assert_array_equal(gpu.array("n_fix"), ora.array("n_fix"))
    np.testing.assert_array_equal(gpu.array("die_axis"), ora.array("die_axis"))
    np.testing.assert_array_equal(gpu.array("ax"), ora.array("ax"))
    np.testing.assert_array_equal(gpu.array("grad"), ora.array("grad"))
    np.testing.assert_array_equal(gpu.array("vol"), ora.array("vol"))
    np.testing.assert_array_equal(gpu.array("v_node"), ora.array("v_node"))
    np.testing.assert_array_equal(gpu.array("g_coef"), ora.array("g_coef"))
    np.testing.assert_array_equal(gpu.array("kvol"), ora.array("kvol"))
    _close(gpu.array("a_fric"), ora.array("a_fric"), 0, "friction areas")
    _close(gpu.array("k_fric"), ora.array("k_fric"), 0, "friction k")
    _close(gpu.array("v"), ora.array("v"), 0, "velocity guess")


@pytest.mark.parametrize("newton", [0, 1])
def test_assemble_matrix_residual_energy(pair, newton):
    gpu, ora, _, _ = pair
    v = ora.array("v") * (1 + 0.01 * np.sin(np.arange(len(ora.array("v")))))  # a non-trivial velocity field
    eg, pg = gpu.assemble(1, newton, v)
    eo, po = ora.assemble(1, newton, v)
    assert abs(eg / eo - 1) < RTOL_ENERGY and abs(pg / po - 1) < RTOL_ENERGY
    _close(gpu.array("val"), ora.array("val"), RTOL_ELEM, "assembled values")
    _close(gpu.array("r"), ora.array("r"), 1e-11, "residual")
    _close(gpu.array("el_sig"), ora.array("el_sig"), RTOL_ELEM, "element flow stress")
    _close(gpu.array("el_rate"), ora.array("el_rate"), RTOL_ELEM, "element strain rate")
    # boundary conditions and regularisation (SolveVelocity :892-913)
    mg = gpu.apply_bc()
    mo = ora.apply_bc()
    assert abs(mg / mo - 1) < 1e-12
    _close(gpu.array("val"), ora.array("val"), RTOL_ELEM, "values after BC")
    _close(gpu.array("r"), ora.array("r"), 1e-11, "residual after BC")


def test_residual_only_assembly(pair):
    gpu, ora, _, _ = pair
    v = ora.array("v")
    eg, pg = gpu.assemble(0, 0, v)
    eo, po = ora.assemble(0, 0, v)
    assert abs(eg / eo - 1) < RTOL_ENERGY and abs(pg / po - 1) < RTOL_ENERGY
    _close(gpu.array("r"), ora.array("r"), RTOL_ENERGY, "residual")


@pytest.mark.parametrize("wide_rows", [None, 48])
def test_increments_track_the_oracle(wide_rows):
    # wide_rows=48 sends most fronts of this small case through the multi-CTA solve path and the pivot-block
    # inverses, which the default threshold keeps for the taller fronts of larger meshes
    cfg, mesh, dies = _case(seed=2)
    gpu = Forging3DSolver(cfg, mesh, dies)
    if wide_rows is not None:
        gpu.set_scalar("wide_front_rows", wide_rows)
    ora = Oracle3D(cfg, mesh, dies)
    for k in range(4):
        info = gpu.step()
        ora.step()
        assert info["iterations"] == ora.scalar("iterations"), f"step {k + 1}: Newton iterations differ"
        assert abs(info["load"] / ora.scalar("load") - 1) < RTOL_STATE, f"step {k + 1}: load"
        np.testing.assert_array_equal(gpu.array("contact"), ora.array("contact"))
        _close_l2(gpu.array("vg"), ora.array("vg"), RTOL_STATE, f"step {k + 1}: velocity")
        # x moves by dt * vg: it inherits the velocity's 1e-6 relative tolerance scaled by the stroke increment
        # over the billet size (0.2 / 20 here), so 1e-7 of the largest coordinate
        _close(gpu.array("x"), ora.array("x"), RTOL_X, f"step {k + 1}: coordinates")
        _close_l2(gpu.array("eps"), ora.array("eps"), RTOL_STRAIN, f"step {k + 1}: effective strain")
        assert abs(gpu.scalar("gap") - ora.scalar("gap")) < 1e-12
    if wide_rows is not None:
        assert gpu.scalar("big_fronts") > 0


def test_frictionless_upset_load_matches_homogeneous_solution():
    # Solver3DTests.cs:30-49 on the GPU path
    mesh, dies = upset_case_3d(20, 40, 3.0, 20.0)
    cfg = Forging3DConfig(C=100, N=0, M=0.1, eps0=1, friction=0, ram=40, h=3, ds=0.5, size=40)
    with Forging3DSolver(cfg, mesh, dies) as s:
        x = s.array("x").reshape(-1, 3)
        t = mesh.tets
        vol = np.einsum("ij,ij->i", x[t[:, 1]] - x[t[:, 0]], np.cross(x[t[:, 2]] - x[t[:, 0]], x[t[:, 3]] - x[t[:, 0]])).sum() / 6
        info = s.step()
        assert 0.99 <= info["load"] / (100 * 4 * vol / 40) <= 1.01


def test_spd_backend_solves_and_reports_non_spd():
    # CudssSolver.TryCreate's self-test (Solver/Linear/CudssSolver.cs:83-93) and a random SPD system
    s = GpuSpdSolver()
    s.analyze(2, [0, 2, 4], [0, 1, 0, 1])
    s.factorize([4, 1, 1, 3])
    x = s.solve([1, 2])
    assert abs(4 * x[0] + x[1] - 1) < 1e-9 and abs(x[0] + 3 * x[1] - 2) < 1e-9
    rng = np.random.default_rng(5)
    n = 300
    A = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.05)
    A = A + A.T + n * np.eye(n)
    cp, ri, vals = [0], [], []
    for j in range(n):
        rows = np.nonzero(A[:, j])[0]
        ri.extend(rows)
        vals.extend(A[rows, j])
        cp.append(len(ri))
    s.analyze(n, np.array(cp), np.array(ri))
    s.factorize(np.array(vals))
    b = rng.standard_normal(n)
    np.testing.assert_allclose(s.solve(b), np.linalg.solve(A, b), rtol=1e-9, atol=1e-12)
    bad = np.array(vals)
    bad[cp[7]:cp[8]][np.array(ri[cp[7]:cp[8]]) == 7] = -1.0
    with pytest.raises(_lib.MatrixNotPositiveDefiniteError):
        s.factorize(bad)
        s.solve(b)
