"""The CPU FP64 restatement of the warm-start network (oracle/mlp_ref.py), pinned before it checks the GPU:
its analytic gradient against central finite differences, and its bfloat16 rounding against known values."""
import numpy as np

import mlp_ref


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.001953125, 1.005859375, -3.14159265, 0.0, 65504.0])
    # bfloat16 spacing at 1 is 2^-7: 1 + 2^-8 ties to even (1.0), 1 + 2^-9 rounds down, 1 + 3 * 2^-9 rounds up
    np.testing.assert_array_equal(mlp_ref.to_bf16(x), [1.0, 1.0, 1.0, 1.0078125, -3.140625, 0.0, 65536.0])


def test_analytic_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.uniform(-0.3, 0.3, mlp_ref.NPAR)
    x = rng.standard_normal((24, mlp_ref.NIN))
    t = rng.standard_normal((24, mlp_ref.NOUT))
    _, g = mlp_ref.loss_and_gradients(p, x, t)
    for i in rng.choice(mlp_ref.NPAR, 60, replace=False):
        e = np.zeros(mlp_ref.NPAR)
        e[i] = 1e-6
        fd = (mlp_ref.loss_and_gradients(p + e, x, t)[0] - mlp_ref.loss_and_gradients(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), f"parameter {i}: {g[i]} vs {fd}"


def test_adam_step_matches_its_definition():
    w, g = np.array([0.5, -0.25], np.float32), np.array([0.1, -2.0], np.float32)
    w1, m1, v1 = mlp_ref.adam_step(w, g, np.zeros(2), np.zeros(2), 1, 1e-3)
    # the first bias-corrected step moves every weight by lr against the sign of its gradient
    np.testing.assert_allclose(w1, w - 1e-3 * np.sign(g), rtol=1e-5)
