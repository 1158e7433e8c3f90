"""The learned scheduler's network restated on the CPU (oracle/mlp_oracle.py):
its backward pass against central finite differences, and its BF16 rounding
against known values.  The GPU training kernels are checked against it in
tests/test_gpu_learned.py."""
import numpy as np

import mlp_oracle as m


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.140625, 1e-3],
                 dtype=np.float32)
    got = m.bf16_round(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties go to the even mantissa (1.0);
    # 1 + 3*2^-8 is halfway between 1 + 2^-7 and 1 + 2^-6: ties go to 1 + 2^-6
    exp = np.array([1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5, 3.140625, 0.00099945068359375], dtype=np.float32)
    assert np.array_equal(got, exp)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, m.N_PARAMS)
    X = rng.normal(size=(64, 16))
    y = rng.integers(0, 3, 64)
    cw = (1.0, 2.0, 0.5)
    loss, g = m.loss_and_grad(p, X, y, cw, quantize=False)
    assert loss > 0
    eps = 1e-6
    idx = np.concatenate([rng.choice(1024, 20, replace=False), 1024 + np.arange(0, 64, 7),
                          1088 + rng.choice(4096, 20, replace=False), 5184 + np.arange(0, 64, 9),
                          5248 + np.arange(0, 192, 17), 5440 + np.arange(3)])
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = m.loss_and_grad(q, X, y, cw, quantize=False)
        q[i] -= 2 * eps
        lm, _ = m.loss_and_grad(q, X, y, cw, quantize=False)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-7 * max(1.0, abs(g[i])), i
