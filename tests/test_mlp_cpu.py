"""The CPU reference of the picker MLP: its analytic gradients agree with
finite differences (float64, no bf16 rounding)."""
import numpy as np

from oracle import mlp_ref


def _layout(din, h, dout):
    dims = [din, h, h, h, dout]
    off, out = 0, []
    for l in range(4):
        w = off
        off = (off + dims[l] * dims[l + 1] + 15) // 16 * 16
        b = off
        off = (off + dims[l + 1] + 15) // 16 * 16
        out.append((w, b, dims[l + 1], dims[l]))
    return out, off


def test_analytic_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    layout, n = _layout(16, 16, 16)
    p = rng.standard_normal(n) * 0.3
    x = rng.standard_normal((16, 16))
    t = rng.standard_normal((16, 16))
    mask = (rng.random((16, 16)) < 0.7).astype(np.float64)
    loss, g = mlp_ref.loss_and_grads(p, layout, x, t, mask, rounding=False)
    for idx in rng.choice(n, 40, replace=False):
        e = np.zeros(n)
        e[idx] = 1e-6
        lp, _ = mlp_ref.loss_and_grads(p + e, layout, x, t, mask, rounding=False)
        lm, _ = mlp_ref.loss_and_grads(p - e, layout, x, t, mask, rounding=False)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[idx]) <= 1e-5 * max(1.0, abs(fd)), (idx, fd, g[idx])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.140625], np.float32)
    r = mlp_ref.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == -2.5 and r[4] == 3.140625
