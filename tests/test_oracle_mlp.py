"""CPU checks of the MLP oracle (the checker of the learned-correction kernels):
its hand-written backpropagation agrees with central finite differences."""
import numpy as np

from oracle import mlp_oracle as M


def test_layout_size():
    assert M.NP == 4 * 64 + 64 + 64 * 64 + 64 + 64 + 1 == 4545


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(size=M.NP) * 0.2
    F = rng.normal(size=(40, 4))
    T = rng.normal(size=40)
    _, g = M.loss_and_grad(p, F, T)
    eps = 1e-6
    for i in list(range(0, M.NP, 97)) + [M.NP - 1]:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (M.loss_and_grad(pp, F, T)[0] - M.loss_and_grad(pm, F, T)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(g[i]), (i, fd, g[i])


def test_bf16_round():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159], dtype=np.float32)
    r = M.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie rounds to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - (-3.140625)) < 1e-6
