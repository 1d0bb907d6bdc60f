"""Independent cases stepped together (csrc/batch.cpp) and the launch-parameter tuner.

Stepping cases side by side from a pool of host threads changes nothing in any case's arithmetic: each context has
its own streams and its reductions run in a fixed order, so the batched cases reproduce the same cases stepped one
after another bit for bit. The tuner only changes launch shapes (which trailing updates use the tensor cores, which
fronts the multi-CTA solves take), so a tuned case stays within rounding of an untuned one.
"""
import numpy as np
import pytest

from impressionfea_b200.batch import ForgingBatch, autotune
from impressionfea_b200.config import Forging2DConfig, Forging3DConfig
from impressionfea_b200.forging2d import ForgingSolver2D
from impressionfea_b200.forging3d import Forging3DSolver
from impressionfea_b200.meshes import upset_case_3d

pytestmark = pytest.mark.gpu


def _cases():
    out = []
    for k, (R, H, h, f) in enumerate([(10.0, 20.0, 2.5, 0.3), (8.0, 18.0, 2.0, 0.5)]):
        mesh, dies = upset_case_3d(R, H, h, 0.7 * H, seed=k)
        cfg = Forging3DConfig(C=120 + 20 * k, N=0.1, M=0.1, eps0=0.01, friction=f, ram=20, h=h, ds=0.3, size=H, tol=1e-4)
        out.append(("3d", cfg, mesh, dies))
    out.append(("2d", Forging2DConfig(nx=10, nz=30)))
    out.append(("2d", Forging2DConfig(nx=12, nz=24, friction=0.5)))
    return out


def _make(cases):
    s3 = [Forging3DSolver(c[1], c[2], c[3]) for c in cases if c[0] == "3d"]
    s2 = [ForgingSolver2D(c[1]) for c in cases if c[0] == "2d"]
    return s3, s2


def test_batched_cases_reproduce_the_cases_stepped_one_by_one():
    cases = _cases()
    a3, a2 = _make(cases)
    ref = [[s.step() for _ in range(3)] for s in a3 + a2]
    b3, b2 = _make(cases)
    batch = ForgingBatch(b3, b2)
    got, status = batch.step(3)
    assert (status == 0).all()
    for c, (r, g) in enumerate(zip(ref, got)):
        for k in range(3):
            assert r[k]["iterations"] == g[k]["iterations"], f"case {c} increment {k + 1}"
            assert r[k]["load"] == g[k]["load"], f"case {c} increment {k + 1}"
    for s, t in zip(a3 + a2, b3 + b2):
        np.testing.assert_array_equal(s.array("x"), t.array("x"))
        np.testing.assert_array_equal(s.array("contact"), t.array("contact"))
    batch.close()


def test_autotune_picks_a_candidate_and_keeps_the_results():
    mesh, dies = upset_case_3d(12.0, 24.0, 1.6, 16.0, seed=3)
    cfg = Forging3DConfig(C=150, N=0.1, M=0.12, eps0=0.01, friction=0.4, ram=50, h=1.6, ds=0.3, size=24.0, tol=1e-4)
    plain, tuned = Forging3DSolver(cfg, mesh, dies), Forging3DSolver(cfg, mesh, dies)
    for s in (plain, tuned):
        s.set_scalar("factor_fp32", 1)
    choice = autotune(tuned, use_cache=False)
    assert choice["tc_rows"] in (512, 1024, 2048, 1e9) and choice["wide_front_rows"] in (96, 192, 384)
    assert choice["best_ms"] > 0
    again = autotune(Forging3DSolver(cfg, mesh, dies), use_cache=True)  # same size class: from the cache
    assert again["best_ms"] == -1 and again["tc_rows"] == choice["tc_rows"]
    for k in range(3):
        a, b = plain.step(), tuned.step()
        assert abs(a["load"] / b["load"] - 1) < 1e-6, f"increment {k + 1}"
