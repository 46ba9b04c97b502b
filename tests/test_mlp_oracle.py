"""The CPU oracle of the learned warm start's network (oracle/mlp.py): its
analytic gradient against central finite differences of its own loss, in
plain FP64 (no BF16 rounding), and its BF16 rounding helper."""
import numpy as np

from oracle import mlp as om


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.1415926], dtype=np.float64)
    r = om.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # a tie rounds to the even mantissa
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) == 0.0


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    d, o, n = 5, 3, 7
    x = rng.normal(size=(n, d))
    y = rng.normal(size=(n, o))
    count = om.H * d + om.H + om.H * om.H + om.H + o * om.H + o
    p = rng.normal(scale=0.1, size=count)
    ins = (np.zeros(d), np.ones(d))
    outs = (np.zeros(o), np.ones(o))
    _, g = om.loss_grad(p, x, y, ins, outs, rounding=False)
    idx = rng.choice(count, size=40, replace=False)
    for i in idx:
        e = np.zeros(count)
        e[i] = 1e-6
        lp, _ = om.loss_grad(p + e, x, y, ins, outs, rounding=False)
        lm, _ = om.loss_grad(p - e, x, y, ins, outs, rounding=False)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
