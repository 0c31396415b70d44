"""CPU check of the network oracle: its backward pass against finite differences
(with the BF16 roundings switched off, where the loss is smooth)."""
import numpy as np

from oracle import mlp_oracle as MO


def test_oracle_backward_matches_finite_differences():
    widths = (5, 7, 6, 2)
    rng = np.random.default_rng(4)
    npar = sum(widths[l] * widths[l + 1] + widths[l + 1] for l in range(len(widths) - 1))
    p = rng.normal(size=npar) * 0.5
    X = rng.normal(size=(9, 5))
    T = rng.normal(size=(9, 2))
    mask = np.array([1.0, 0.5])
    mean, std = X.mean(0), X.std(0)
    g, loss = MO.grad(p, widths, mean, std, X, T, mask, round_bf16=False)
    h = 1e-6
    fd = np.zeros_like(p)
    for k in range(npar):
        q = p.copy(); q[k] += h
        lp = MO.grad(q, widths, mean, std, X, T, mask, round_bf16=False)[1]
        q[k] -= 2 * h
        lm = MO.grad(q, widths, mean, std, X, T, mask, round_bf16=False)[1]
        fd[k] = (lp - lm) / (2 * h)
    assert np.max(np.abs(fd - g)) < 1e-6 * max(1.0, np.max(np.abs(g)))


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], dtype=np.float32)
    r = MO.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
