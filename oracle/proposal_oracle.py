"""CPU restatement of the learned-proposal network (TEST INFRASTRUCTURE ONLY:
the product library never imports this file; tests use it as the checker).

The network and its numerics follow include/hase_b200_proposal.h:

- 12 features -> 64 -> 64 -> 64 (SiLU) -> 1 logit;
- W1..W3 and w4 rounded to BF16 (round to nearest even);
- layer inputs (features and hidden activations) rounded to BF16 before
  each tensor-core layer, products accumulated in FP32;
- biases and the output layer in FP32 (the last hidden layer feeds the
  output layer unrounded).

Loss of one sample point (group of rows): cross entropy between the softmax
of its logits and the normalised target weights t (>= 0), scaled by the
group weight,  L_g = -w_g * sum_i (t_i / sum t) * log softmax(l)_i.
``loss_and_grad`` returns the loss and dL/dparams in the master-vector order
W1[12][64] b1 W2[64][64] b2 W3[64][64] b3 w4 b4.  It is computed in FP64 on
the same BF16-rounded operands as the device (straight-through for the
roundings): the backward products dz3 W3^T and dz2 W2^T take dz rounded to
BF16 (they run on the tensor cores), the weight and bias gradients take the
unrounded dz (FP32 reductions on the device).
"""

from __future__ import annotations

import numpy as np

FEATURES = 12
HIDDEN = 64
PARAMS = FEATURES * HIDDEN + HIDDEN + 2 * (HIDDEN * HIDDEN + HIDDEN) + HIDDEN + 1


def bf16(x):
    """Round float32 values to the nearest BF16 value (ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32).copy()
    special = ~np.isfinite(a)
    out[special] = a[special]
    return out


def unpack(params):
    p = np.asarray(params, np.float32).ravel()
    assert p.size == PARAMS
    o = 0

    def take(n, shape):
        nonlocal o
        v = p[o:o + n].reshape(shape)
        o += n
        return v

    W1 = take(FEATURES * HIDDEN, (FEATURES, HIDDEN))
    b1 = take(HIDDEN, (HIDDEN,))
    W2 = take(HIDDEN * HIDDEN, (HIDDEN, HIDDEN))
    b2 = take(HIDDEN, (HIDDEN,))
    W3 = take(HIDDEN * HIDDEN, (HIDDEN, HIDDEN))
    b3 = take(HIDDEN, (HIDDEN,))
    w4 = take(HIDDEN, (HIDDEN,))
    b4 = take(1, (1,))
    return W1, b1, W2, b2, W3, b3, w4, b4


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(params, features, *, keep=False):
    """Logits [rows] (float32 arithmetic with the device's BF16 roundings)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params)
    x = bf16(np.asarray(features, np.float32).reshape(-1, FEATURES))
    z1 = x @ bf16(W1) + b1
    h1 = bf16(silu(z1))
    z2 = h1 @ bf16(W2) + b2
    h2 = bf16(silu(z2))
    z3 = h2 @ bf16(W3) + b3
    h3 = silu(z3)
    logits = h3 @ bf16(w4) + b4[0]
    if keep:
        return logits.astype(np.float32), (x, z1, h1, z2, h2, z3, h3)
    return logits.astype(np.float32)


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_and_grad(params, features, offsets, targets, group_weights=None):
    """Mean over groups of the weighted cross entropy and its gradient (FP64).

    offsets [G+1] delimit the rows of each group (sample point); targets [rows]
    are non-negative scores per row (normalised within the group)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = [np.asarray(a, np.float64) for a in unpack(params)]
    logits, (x, z1, h1, z2, h2, z3, h3) = forward(params, features, keep=True)
    x, z1, h1, z2, h2, z3, h3 = [np.asarray(a, np.float64) for a in (x, z1, h1, z2, h2, z3, h3)]
    l = np.asarray(logits, np.float64)
    t = np.asarray(targets, np.float64)
    off = np.asarray(offsets, np.int64)
    G = off.size - 1
    gw = np.ones(G) if group_weights is None else np.asarray(group_weights, np.float64)
    dl = np.zeros_like(l)
    loss = 0.0
    for g in range(G):
        a, b = off[g], off[g + 1]
        tg = t[a:b]
        ts = tg.sum()
        if ts <= 0 or b <= a:
            continue
        lg = l[a:b]
        m = lg.max()
        lse = m + np.log(np.exp(lg - m).sum())
        q = np.exp(lg - lse)
        tn = tg / ts
        loss += gw[g] * -(tn * (lg - lse)).sum()
        dl[a:b] = gw[g] * (q - tn)
    loss /= G
    dl /= G
    W2r, W3r, w4r, W1r = (np.asarray(bf16(np.asarray(w, np.float32)), np.float64) for w in (W2, W3, w4, W1))
    g_w4 = h3.T @ dl
    g_b4 = dl.sum()
    def r(a):
        return np.asarray(bf16(np.asarray(a, np.float32)), np.float64)

    # the weight gradients take dz as the BF16 operand of the tensor-core
    # product h^T dz (hase_proposal.cu, mlpBackwardKernel); the bias sums keep it in FP32
    dz3 = np.outer(dl, w4r) * _dsilu(z3)
    g_W3 = h2.T @ r(dz3)
    g_b3 = dz3.sum(0)
    dz2 = (r(dz3) @ W3r.T) * _dsilu(z2)
    g_W2 = h1.T @ r(dz2)
    g_b2 = dz2.sum(0)
    dz1 = (r(dz2) @ W2r.T) * r(_dsilu(z1))  # silu'(z1) kept as bf16 rows on the device
    g_W1 = x.T @ r(dz1)
    g_b1 = dz1.sum(0)
    grad = np.concatenate([g_W1.ravel(), g_b1, g_W2.ravel(), g_b2, g_W3.ravel(), g_b3, g_w4, [g_b4]])
    return float(loss), grad
