"""Learned initial guess for con2prim (rhllc::GetPhysValueStab seeded by a network).

    net = LearnedGuess(device=0, seed=1)
    net.train(U, p, epochs=8)                  # U [n,5], p [n]: CUDA float64 tensors
    stats, n_back = net.con2prim(U2, W2)       # batch con2prim seeded by the network

The network (3 -> 64 -> 64 -> 1, ReLU) predicts log(p / tau), tau = E - D, from
(log(Q/tau), log(|S|/tau), log(tau/D)), Q = E - sqrt(|S|^2 + D^2).  Training and inference run in this library's own
CUDA kernels (include/rrhd.h, "learned con2prim guess").
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class LearnedGuess:
    N_PARAMS = 4481

    def __init__(self, device: int = 0, seed: int = 1):
        h = C.c_void_p()
        L.check(L.lib.rrhd_mlp_create(device, seed, C.byref(h)), "rrhd_mlp_create")
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            L.lib.rrhd_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        th = np.zeros(self.N_PARAMS, np.float32)
        nm = np.zeros(8, np.float32)
        L.check(L.lib.rrhd_mlp_get(self._h, L.ptr(th), L.ptr(nm)), "rrhd_mlp_get")
        return th, nm

    def set_params(self, theta=None, norm=None):
        th = None if theta is None else np.ascontiguousarray(theta, np.float32)
        nm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        L.check(L.lib.rrhd_mlp_set(self._h, L.ptr(th), L.ptr(nm)), "rrhd_mlp_set")

    def save(self, path: str):
        th, nm = self.params()
        np.savez(path, theta=th, norm=nm)

    def load(self, path: str):
        z = np.load(path)
        self.set_params(z["theta"], z["norm"])

    def train(self, U, p, epochs: int = 8, batch: int = 4096, lr: float = 2e-3, seed: int = 3,
              set_norm: bool = True, stream=None):
        hist = np.zeros(epochs, np.float32)
        L.check(L.lib.rrhd_mlp_train(self._h, L.ptr(U), L.ptr(p), U.shape[0], epochs, batch, lr, seed,
                                     1 if set_norm else 0, L.ptr(hist), stream), "rrhd_mlp_train")
        return hist

    def gradient(self, U, p):
        g = np.zeros(self.N_PARAMS, np.float32)
        loss = C.c_float()
        L.check(L.lib.rrhd_mlp_gradient(self._h, L.ptr(U), L.ptr(p), U.shape[0], L.ptr(g), C.byref(loss)),
                "rrhd_mlp_gradient")
        return g, loss.value

    def con2prim(self, U, W, status=None, eos: int = 1, gamma: float = 4.0 / 3.0, fallback: bool = True,
                 k_stall: int = 8, guess=None, stream=None):
        st = L.C2pStats()
        nb = C.c_int64()
        L.check(L.lib.rrhd_con2prim_batch_mlp(self._h, eos, gamma, L.ptr(U), L.ptr(W), L.ptr(status), U.shape[0],
                                              1 if fallback else 0, k_stall, C.byref(st), C.byref(nb), L.ptr(guess),
                                              stream), "rrhd_con2prim_batch_mlp")
        return st, nb.value
