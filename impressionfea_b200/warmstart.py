"""The learned warm start: a per-node MLP that predicts each node's velocity change over the coming increment.

It replaces the initial guess of LoadVelocityGuess (ThreeD/Forging3DSolver.cs:854-869). The network
(16 -> 128 -> 128 -> 128 -> 3, GELU, BF16 weights and activations, FP32 accumulation) runs and trains on the
B200 tensor cores through the C ABI (``ifea_mlp_*`` in include/ifea_gpu.h). A solver records training samples from
its own converged increments (``attach(solver, record=True)``); after ``train()`` the network gives a solver its
starting velocity (``attach(solver, predict=True)``), which the solver keeps only where the functional is lower
than at the reference's start.
"""
import ctypes as C

import numpy as np

from ._lib import lib, raise_for

NIN, HID, NOUT = 16, 128, 3


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class WarmStartNetwork:
    def __init__(self, seed=0):
        L = lib()
        self._L = L
        h = C.c_void_p()
        raise_for(L.ifea_mlp_create(C.c_uint64(seed), C.byref(h)), "no CUDA device or library")
        self._h = h
        self.npar = int(L.ifea_mlp_param_count())
        self.last_train_ms = 0.0

    def _check(self, st):
        if st != 0:
            raise_for(st, self._L.ifea_mlp_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.ifea_mlp_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return self._h

    def params(self):
        p = np.zeros(self.npar, np.float32)
        self._check(self._L.ifea_mlp_get_params(self._h, _fp(p), self.npar))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._L.ifea_mlp_set_params(self._h, _fp(p), p.size))

    def normalisation(self):
        n = np.zeros(2 * NIN + 2 * NOUT, np.float32)
        self._check(self._L.ifea_mlp_get_normalisation(self._h, _fp(n)))
        return n

    def set_normalisation(self, n):
        n = np.ascontiguousarray(n, np.float32)
        self._check(self._L.ifea_mlp_set_normalisation(self._h, _fp(n)))

    def identity_normalisation(self):
        self.set_normalisation(np.concatenate([np.zeros(NIN), np.ones(NIN), np.zeros(NOUT), np.ones(NOUT)]))

    def add_samples(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        self._check(self._L.ifea_mlp_add_samples(self._h, _fp(x), _fp(t), len(x)))

    @property
    def samples(self):
        return int(self._L.ifea_mlp_samples(self._h))

    def clear_samples(self):
        self._check(self._L.ifea_mlp_clear_samples(self._h))

    def fit_normalisation(self):
        self._check(self._L.ifea_mlp_fit_normalisation(self._h))

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((len(x), NOUT), np.float32)
        self._check(self._L.ifea_mlp_forward(self._h, _fp(x), len(x), _fp(y)))
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.npar, np.float32)
        loss = C.c_float()
        self._check(self._L.ifea_mlp_gradients(self._h, _fp(x), _fp(t), len(x), _fp(g), C.byref(loss)))
        return loss.value, g

    def train(self, steps, batch=8192, lr=1e-3, seed=0):
        loss, ms = C.c_float(), C.c_double()
        self._check(self._L.ifea_mlp_train(self._h, int(steps), int(batch), C.c_float(lr), C.c_uint64(seed),
                                           C.byref(loss), C.byref(ms)))
        self.last_train_ms = ms.value
        return loss.value

    def attach(self, solver, record=False, predict=False):
        """Make a Forging3DSolver record training samples into this network and/or start from its predictions."""
        mode = (1 if record else 0) | (2 if predict else 0)
        solver._check(self._L.ifea3d_set_warm_start(solver._h, self._h if mode else None, mode))
        solver._warm_start_net = self if mode else None  # keeps the network alive while the solver uses it
