"""Learned coarse correction (an addition on top of the reference's plain
Schwarz-CG; see include/hoefem.h, hoefem_learned_*)."""
import ctypes as C

import numpy as np

from ._capi import check, host_f64, host_i64, lib, ptr
from .model import _same_space

F, H, NM = 64, 256, 32


class LearnedCoarseCorrection:
    """MLP 64 -> 256 -> 256 -> 32 over a coarse space of `num_subdomains`
    coarse subdomains x 32 local modes.  Parameter layout (flat float32):
    W1 (64 x 256), b1, W2 (256 x 256), b2, W3 (256 x 32), b3."""

    def __init__(self, model, dirichlet_nodes=(), num_subdomains=256, seed=0):
        self.model = model
        bc = host_i64(dirichlet_nodes)
        h = C.c_void_p()
        check(lib().hoefem_learned_create(model._h, bc.ctypes.data if bc.size else None, bc.size, num_subdomains,
                                          seed, C.byref(h)))
        self._h = h
        self._lib = lib()  # kept for __del__ at interpreter exit
        self.num_subdomains = num_subdomains
        n = C.c_int64()
        check(lib().hoefem_learned_num_params(h, C.byref(n)))
        self.num_params = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_lib", None) is not None:
            self._lib.hoefem_learned_destroy(h)
            self._h = None

    def num_pairs(self):
        n = C.c_int64()
        check(lib().hoefem_learned_num_pairs(self._h, C.byref(n)))
        return n.value

    def add_pair(self, r, e):
        check(lib().hoefem_learned_add_pair(self._h, ptr(r)[0], ptr(e)[0], _same_space(r, e)))

    def train(self, steps, batch=256, lr=1e-3, seed=0):
        hist = np.zeros(max(int(steps), 1), dtype=np.float32)
        check(lib().hoefem_learned_train(self._h, int(steps), int(batch), float(lr), int(seed), hist.ctypes.data))
        return hist[: int(steps)]

    def forward_backward(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = C.c_float()
        g = np.zeros(self.num_params, dtype=np.float32)
        out = np.zeros((X.shape[0], NM), dtype=np.float32)
        check(lib().hoefem_learned_forward_backward(self._h, X.ctypes.data, T.ctypes.data, X.shape[0], C.byref(loss),
                                                    g.ctypes.data, out.ctypes.data))
        return loss.value, g, out

    def infer(self, X, bf16=True):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros((X.shape[0], NM), dtype=np.float32)
        check(lib().hoefem_learned_infer(self._h, X.ctypes.data, X.shape[0], 1 if bf16 else 0, out.ctypes.data))
        return out

    def get_weights(self):
        w = np.zeros(self.num_params, dtype=np.float32)
        check(lib().hoefem_learned_get_weights(self._h, w.ctypes.data))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.num_params
        check(lib().hoefem_learned_set_weights(self._h, w.ctypes.data))

    def predict(self, r, x0=None):
        if x0 is None:
            x0 = np.zeros_like(r) if isinstance(r, np.ndarray) else r.new_zeros(r.shape)
        check(lib().hoefem_learned_predict(self._h, ptr(r)[0], ptr(x0)[0], _same_space(r, x0)))
        return x0
