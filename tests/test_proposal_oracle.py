"""CPU pins of the learned-proposal oracle (oracle/proposal_oracle.py): its
analytic gradient against central finite differences in exact (FP64, no BF16
rounding) arithmetic, and its BF16 rounding against known values."""

from __future__ import annotations

import numpy as np


def test_bf16_rounding_is_nearest_even():
    from oracle import proposal_oracle as po

    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0], np.float32)
    # 1 + 2^-8 lies halfway between 1 and 1 + 2^-7: ties to even -> 1
    np.testing.assert_array_equal(po.bf16(x), np.array([1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5, 0.0], np.float32))


def test_analytic_gradient_matches_finite_differences(monkeypatch):
    from oracle import proposal_oracle as po

    def unpack64(params):
        p = np.asarray(params, np.float64).ravel()
        o, out = 0, []
        for n, sh in [(768, (12, 64)), (64, (64,)), (4096, (64, 64)), (64, (64,)), (4096, (64, 64)), (64, (64,)),
                      (64, (64,)), (1, (1,))]:
            out.append(p[o:o + n].reshape(sh))
            o += n
        return out

    def forward64(params, features, *, keep=False):
        W1, b1, W2, b2, W3, b3, w4, b4 = unpack64(params)
        x = np.asarray(features, np.float64)
        z1 = x @ W1 + b1
        h1 = po.silu(z1)
        z2 = h1 @ W2 + b2
        h2 = po.silu(z2)
        z3 = h2 @ W3 + b3
        h3 = po.silu(z3)
        logits = h3 @ w4 + b4[0]
        return (logits, (x, z1, h1, z2, h2, z3, h3)) if keep else logits

    monkeypatch.setattr(po, "bf16", lambda a: np.asarray(a, np.float64))
    monkeypatch.setattr(po, "unpack", unpack64)
    monkeypatch.setattr(po, "forward", forward64)
    rng = np.random.default_rng(0)
    p = rng.normal(size=po.PARAMS) * 0.2
    x = rng.normal(size=(50, 12))
    off = np.array([0, 20, 50])
    t = rng.random(50)
    w = np.array([0.7, 1.3])
    _, g = po.loss_and_grad(p, x, off, t, w)
    worst = 0.0
    for idx in range(0, po.PARAMS, 97):
        e = np.zeros_like(p)
        e[idx] = 1e-6
        fd = (po.loss_and_grad(p + e, x, off, t, w)[0] - po.loss_and_grad(p - e, x, off, t, w)[0]) / 2e-6
        worst = max(worst, abs(fd - g[idx]) / (abs(fd) + 1e-6))
    assert worst < 1e-4
