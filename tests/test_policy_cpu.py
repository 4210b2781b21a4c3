"""CPU checks of the learned-policy network oracle: its analytic gradient
against central finite differences, and the BF16 rounding it shares with the
GPU kernels."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, (64, mlp.F))
    y = rng.uniform(0, 3, 64)
    p = mlp.glorot_params(2).astype(np.float64)
    loss, g = mlp.loss_grad64(x, y, p)
    idx = np.concatenate([rng.choice(mlp.PARAMS, 40, replace=False),
                          [mlp.OFF_B3, mlp.OFF_W3, mlp.OFF_B1, mlp.OFF_W1]])
    fd = mlp.finite_difference(x, y, p, idx)
    assert loss > 0
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-6)


def test_bf16_rounding_ties_to_even():
    # bfloat16 spacing at 1.0 is 2^-7
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5],
                 np.float32)
    r = mlp.bf16_round(a)
    # ties: 1+2^-8 -> 1.0 (even), 1+3*2^-8 -> 1+2^-6 (even); others to nearest
    np.testing.assert_array_equal(r, np.array([1.0, 1.0, 1.0 + 2 ** -6, 1.0, 1.0 + 2 ** -7, -2.5],
                                              np.float32))
