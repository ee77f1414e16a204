"""Host front end of the learned importance proposal (include/hase_b200_proposal.h)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class ProposalNet:
    """The proposal MLP on one device (FP32 master parameters on the host)."""

    FEATURES = N.PROPOSAL_FEATURES
    PARAMS = N.PROPOSAL_PARAMS

    def __init__(self, device: int = 0, seed: int = 0):
        handle = C.c_void_p()
        N.check(N.lib().hase_proposal_create(int(device), int(seed) & 0xFFFFFFFF, C.byref(handle)))
        self.handle = handle
        self.device = int(device)

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.PARAMS, np.float32)
        N.check(N.lib().hase_proposal_get_params(self.handle, N.ptr(out, N._f32p)))
        return out

    @params.setter
    def params(self, value):
        p = np.ascontiguousarray(np.asarray(value, np.float32).ravel())
        if p.size != self.PARAMS:
            raise ValueError(f"expected {self.PARAMS} parameters, got {p.size}")
        N.check(N.lib().hase_proposal_set_params(self.handle, N.ptr(p, N._f32p)))

    def forward(self, features) -> np.ndarray:
        f = np.ascontiguousarray(np.asarray(features, np.float32).reshape(-1, self.FEATURES))
        out = np.empty(f.shape[0], np.float32)
        N.check(N.lib().hase_proposal_forward(self.handle, f.shape[0], N.ptr(f, N._f32p), N.ptr(out, N._f32p)))
        return out

    @staticmethod
    def _batch(offsets, features, targets, group_weights, keep):
        off = keep(np.ascontiguousarray(np.asarray(offsets, np.uint32).ravel()))
        f = keep(np.ascontiguousarray(np.asarray(features, np.float32).reshape(-1, N.PROPOSAL_FEATURES)))
        t = keep(np.ascontiguousarray(np.asarray(targets, np.float32).ravel()))
        if f.shape[0] != int(off[-1]) or t.size != int(off[-1]):
            raise ValueError("features and targets must have offsets[-1] rows")
        w = None if group_weights is None else keep(np.ascontiguousarray(np.asarray(group_weights, np.float32)))
        return N.ProposalBatch(off.size - 1, N.ptr(off, N._u32p), N.ptr(f, N._f32p), N.ptr(t, N._f32p),
                               N.ptr(w, N._f32p))

    def loss_grad(self, offsets, features, targets, group_weights=None):
        """Mean cross-entropy loss of the groups and its gradient (device)."""
        held = []
        b = self._batch(offsets, features, targets, group_weights, lambda a: held.append(a) or a)
        loss = np.zeros(1, np.float32)
        grad = np.empty(self.PARAMS, np.float32)
        N.check(N.lib().hase_proposal_loss_grad(self.handle, C.byref(b), N.ptr(loss, N._f32p), N.ptr(grad, N._f32p)))
        return float(loss[0]), grad

    def train(self, offsets, features, targets, *, steps, groups_per_step, learning_rate=1e-3, group_weights=None,
              beta1=0.0, beta2=0.0, epsilon=0.0):
        """Adam on the device; returns the loss of every step."""
        held = []
        b = self._batch(offsets, features, targets, group_weights, lambda a: held.append(a) or a)
        d = N.ProposalTrainDesc(int(steps), int(groups_per_step), float(learning_rate), float(beta1), float(beta2),
                                float(epsilon))
        hist = np.empty(int(steps), np.float32)
        N.check(N.lib().hase_proposal_train(self.handle, C.byref(b), C.byref(d), N.ptr(hist, N._f32p)))
        return hist

    def close(self):
        if getattr(self, "handle", None):
            N.lib().hase_proposal_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
