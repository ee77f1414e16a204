"""GPU parity of the learned-proposal network (include/hase_b200_proposal.h)
against the CPU restatement oracle/proposal_oracle.py.

Tolerance: the device and the oracle round the same operands to BF16 and
accumulate in FP32 in a different order (~1e-7 relative); an activation that
sits on a BF16 rounding boundary can round to the neighbouring value on one
side (one BF16 ulp, 2^-8 relative), so single logits may move by a few 1e-3
of the logit scale while the bulk agrees to ~1e-5.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net(seed=3):
    from haseongpu_b200 import build
    from haseongpu_b200.proposal import ProposalNet

    build.build_library()
    return ProposalNet(device=0, seed=seed)


@pytest.mark.parametrize("rows", [1, 127, 128, 1000, 40_000])
def test_forward_matches_oracle(rows):
    from oracle import proposal_oracle as po

    rng = np.random.default_rng(rows)
    feats = rng.normal(size=(rows, po.FEATURES)).astype(np.float32)
    with _net() as net:
        params = net.params
        params[-1] = 0.25  # non-zero output bias
        params[po.FEATURES * po.HIDDEN:po.FEATURES * po.HIDDEN + po.HIDDEN] = rng.normal(scale=0.1, size=po.HIDDEN)
        net.params = params
        dev = net.forward(feats)
    ref = po.forward(params, feats)
    scale = max(1.0, float(np.abs(ref).max()))
    err = np.abs(dev - ref) / scale
    assert np.all(np.isfinite(dev))
    assert np.median(err) < 1e-4, np.sort(err)[-5:]
    assert err.max() < 2e-2, np.sort(err)[-5:]


def test_forward_initial_params_are_deterministic():
    with _net(seed=11) as a, _net(seed=11) as b, _net(seed=12) as c:
        assert np.array_equal(a.params, b.params)
        assert not np.array_equal(a.params, c.params)


def _groups(rng, sizes):
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    return off


def test_loss_and_gradient_match_oracle():
    """Device loss / gradient (tensor-core forward and backward products, FP32
    reductions) against the FP64 oracle on the same BF16-rounded operands."""
    from oracle import proposal_oracle as po

    rng = np.random.default_rng(5)
    sizes = [300, 1, 129, 1024, 77, 2500, 640]
    off = _groups(rng, sizes)
    rows = int(off[-1])
    feats = rng.normal(size=(rows, po.FEATURES)).astype(np.float32)
    targets = (rng.random(rows) ** 4).astype(np.float32)
    gw = rng.uniform(0.5, 2.0, len(sizes)).astype(np.float32)
    with _net(seed=9) as net:
        params = net.params * 1.5
        params[po.FEATURES * po.HIDDEN:po.FEATURES * po.HIDDEN + po.HIDDEN] = rng.normal(scale=0.2, size=po.HIDDEN)
        net.params = params
        loss, grad = net.loss_grad(off, feats, targets, gw)
    ref_loss, ref_grad = po.loss_and_grad(params, feats, off, targets, gw)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    cos = float(np.dot(grad, ref_grad) / (np.linalg.norm(grad) * np.linalg.norm(ref_grad)))
    assert cos > 0.9999, cos
    scale = np.abs(ref_grad).max()
    err = np.abs(grad - ref_grad)
    assert np.all(err <= 2e-3 * scale + 2e-2 * np.abs(ref_grad)), float((err / scale).max())
    assert abs(grad[-1]) < 1e-4 * scale  # the softmax does not depend on the output bias (FP32 sum of +-q, t)


def test_training_learns_a_known_proposal():
    """Targets drawn from a known softmax over 12-d features; training on the
    device drives the cross entropy to its entropy floor."""
    rng = np.random.default_rng(6)
    G, P = 64, 400
    off = np.arange(G + 1, dtype=np.uint32) * P
    feats = rng.normal(size=(G * P, 12)).astype(np.float32)
    true_logit = 1.5 * feats[:, 0] - 0.8 * feats[:, 3] ** 2 + np.sin(2 * feats[:, 5]) + 0.5 * feats[:, 7] * feats[:, 8]
    t = np.exp(true_logit - true_logit.max())
    t = t.reshape(G, P)
    t /= t.sum(1, keepdims=True)
    entropy = float(-(t * np.log(t)).sum(1).mean())
    with _net(seed=1) as net:
        loss0, _ = net.loss_grad(off, feats, t.ravel())
        hist = net.train(off, feats, t.ravel(), steps=600, groups_per_step=16, learning_rate=3e-3)
        loss1, _ = net.loss_grad(off, feats, t.ravel())
    assert np.all(np.isfinite(hist))
    assert loss0 - entropy > 0.3
    assert loss1 - entropy < 0.1 * (loss0 - entropy), (loss0, loss1, entropy)
