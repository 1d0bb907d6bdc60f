"""Parity of the 2D CUDA path (Q4 kernel, band assembly, GPU band Cholesky) with the CPU oracle."""
import math

import numpy as np
import pytest

from impressionfea_b200 import _lib
from impressionfea_b200.config import Forging2DConfig
from impressionfea_b200.forging2d import ForgingSolver2D, band_factor_solve
from oracle import Oracle2D, OracleBand

pytestmark = pytest.mark.gpu


def _upset(axi, m, shut=30.0):
    return Forging2DConfig(C=100, N=0, M=0.1, eps0=1, friction=m, ram=40, ds=0.5, tol=1e-5, max_iter=60,
                           axisymmetric=axi, length=50, radius=20, height=40, nx=10, nz=20,
                           bottom_profile=np.array([[0, 0], [200, 0]]), top_profile=np.array([[0, shut], [200, shut]]))


def _close(a, b, rtol, what):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    assert err <= rtol, f"{what}: {err:.3e} > {rtol:.1e}"


def test_equation_numbering_and_boundary_loop_bit_exact():
    cfg = Forging2DConfig()
    g, o = ForgingSolver2D(cfg), Oracle2D(cfg)
    np.testing.assert_array_equal(g.array("eq"), o.array("eq"))
    np.testing.assert_array_equal(g.array("loop"), o.array("loop"))
    np.testing.assert_array_equal(g.array("loop_owner"), o.array("loop_owner"))
    assert g.scalar("half_band") == o.scalar("half_band")
    np.testing.assert_array_equal(g.array("contact"), o.array("contact"))


@pytest.mark.parametrize("newton", [0, 1])
def test_assembly_matches(newton):
    cfg = _upset(True, 0.3)
    g, o = ForgingSolver2D(cfg), Oracle2D(cfg)
    g.prepare()
    o.prepare()
    np.testing.assert_array_equal(g.array("fixed"), o.array("fixed"))
    np.testing.assert_array_equal(g.array("rotated"), o.array("rotated"))
    _close(g.array("a_fric"), o.array("a_fric"), 0, "friction areas")
    v = o.array("v") * (1 + 0.01 * np.cos(np.arange(len(o.array("v")))))
    eg, pg = g.assemble(1, newton, v)
    eo, po = o.assemble(1, newton, v)
    assert abs(eg / eo - 1) < 1e-12 and abs(pg / po - 1) < 1e-12
    _close(g.array("band"), o.array("band"), 1e-12, "band values")
    _close(g.array("r"), o.array("r"), 1e-11, "residual")
    _close(g.array("el_sig"), o.array("el_sig"), 1e-12, "element flow stress")


def test_gpu_band_cholesky_is_bit_identical_to_the_reference_loop():
    cfg = Forging2DConfig()
    o = Oracle2D(cfg)
    o.prepare()
    o.assemble(1, 1, o.array("v"))
    band = o.array("band")
    hb = int(o.scalar("half_band"))
    n = len(o.array("v"))
    ob = OracleBand(n, hb)
    for i in range(n):
        for j in range(max(0, i - hb), i + 1):
            v = band[i * (hb + 1) + (j - i + hb)]
            if v != 0:
                ob.add(i, j, v)
    for d in np.nonzero(o.array("fixed"))[0]:
        ob.constrain(int(d))
    a0 = ob.data().copy()
    rhs = np.sin(np.arange(n))
    row, _ = ob.factorize()
    assert row == -1
    x_ref = ob.solve(rhs)
    L, x = band_factor_solve(a0, hb, rhs)
    np.testing.assert_array_equal(L, ob.data())
    np.testing.assert_array_equal(x, x_ref)


def _spd_band(n, b, seed):
    rng = np.random.default_rng(seed)
    w = b + 1
    a = np.zeros(n * w)
    for i in range(n):
        lo = max(0, i - b)
        a[i * w + (lo - i + b):i * w + b] = rng.random(i - lo) - 0.5
        a[i * w + b] = 2.0 * b + 1.0 + rng.random()
    return a, rng.standard_normal(n)


# (n, half-bandwidth): bands narrower than a panel (1, 5), one column either side of the 32-column panel, a
# circular window reloaded many times (2000 x 85: the 2D decks' shape; 3000 x 60), the whole band resident
# (90 x 64, 70 x 69, 150 x 110), 16- and 8-column panels (1200 x 140, 1200 x 145) and a band too wide for the
# shared-memory window, factorised in place (1500 x 160)
@pytest.mark.parametrize("n,b", [(100, 1), (200, 5), (150, 31), (150, 33), (2000, 85), (3000, 60), (90, 64),
                                 (70, 69), (150, 110), (1200, 140), (1200, 145), (1500, 160)])
def test_blocked_band_cholesky_is_bit_identical_to_the_reference_loop(n, b):
    a, rhs = _spd_band(n, b, n + b)
    ob = OracleBand(n, b)
    ob.set_data(a)
    row, _ = ob.factorize()
    assert row == -1
    x_ref = ob.solve(rhs)
    L, x = band_factor_solve(a, b, rhs)
    np.testing.assert_array_equal(L, ob.data())
    np.testing.assert_array_equal(x, x_ref)


def test_blocked_band_reports_the_first_failing_row_inside_a_panel():
    n, b = 400, 40
    a, rhs = _spd_band(n, b, 5)
    a[77 * (b + 1) + b] = -3.0  # row 77: the third panel's 14th column
    with pytest.raises(_lib.MatrixNotPositiveDefiniteError, match="equation 77 "):
        band_factor_solve(a, b, rhs)


def test_gpu_band_reports_non_positive_pivot():
    # NumericsTests.cs:40-48
    a = np.zeros(3 * 2)
    a[0 * 2 + 1], a[1 * 2 + 1], a[2 * 2 + 1] = 1, -1, 1
    with pytest.raises(_lib.MatrixNotPositiveDefiniteError):
        band_factor_solve(a, 1, np.ones(3))


def test_frictionless_axisymmetric_upset_load():
    # SolverVerificationTests.cs:44-53 on the GPU path
    g = ForgingSolver2D(_upset(True, 0))
    info = g.step()
    assert 0.995 <= info["load"] / (100 * math.pi * 400) <= 1.005


def test_config1_increments_track_the_oracle():
    cfg = Forging2DConfig()
    g, o = ForgingSolver2D(cfg), Oracle2D(cfg)
    for k in range(5):
        info = g.step()
        o.step()
        assert info["iterations"] == o.scalar("iterations"), f"step {k + 1}"
        assert abs(info["load"] / o.scalar("load") - 1) < 1e-6, f"step {k + 1}: load"
        np.testing.assert_array_equal(g.array("contact"), o.array("contact"))
        _close(g.array("x"), o.array("x"), 1e-9, f"step {k + 1}: coordinates")
        _close(g.array("eps"), o.array("eps"), 1e-6, f"step {k + 1}: strain")
