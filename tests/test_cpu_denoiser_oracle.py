"""The numpy oracle of the learned denoiser: its backward (exact float64 mode)
against central finite differences of its forward, and the BF16 rounding."""
import numpy as np

from oracle import denoiser as dn


def random_params(rng, scale=0.2):
    p = rng.normal(0.0, scale, dn.PARAMS).astype(np.float32)
    for l in range(3):
        base = l * dn.LAYER
        w = p[base:base + dn.TAPS * dn.C * dn.C].reshape(dn.TAPS, dn.C, dn.C)
        if l == 0:
            w[:, 4:, :] = 0.0
        if l == 2:
            w[:, :, 4:] = 0.0
            p[base + dn.TAPS * dn.C * dn.C + 4:base + dn.LAYER] = 0.0
    return p


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    shape = (3, 4, 5)
    periodic = (1, 0, 1)
    x = rng.normal(0, 1, shape + (4,))
    target = rng.normal(0, 1, shape + (4,))
    p = random_params(rng).astype(np.float64)
    _, g = dn.loss_grad(p, x, target, periodic, bf16_mode=False)
    for trial in range(6):
        v = rng.normal(0, 1, dn.PARAMS)
        v[g == 0] = 0.0
        eps = 1e-6
        lp, _ = dn.loss_grad(p + eps * v, x, target, periodic, bf16_mode=False)
        lm, _ = dn.loss_grad(p - eps * v, x, target, periodic, bf16_mode=False)
        fd = (lp - lm) / (2 * eps)
        an = float(g @ v)
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (trial, fd, an)


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0], dtype=np.float32)
    r = dn.bf16(a)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert r[3] == -2.5 and r[4] == 0.0
