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
