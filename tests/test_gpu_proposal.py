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
