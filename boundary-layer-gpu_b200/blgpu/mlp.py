"""The learned wall-stress network over the C ABI (blgpu_mlp_*).

Net(4 -> 64 -> 64 -> 64 -> 2, GELU) on the tensor cores with BF16 operands
and FP32 accumulation; trained on the device by its own forward/backward
kernels and Adam.  Inputs per wall point: u and w at the sampling row,
ln(h |u| / nu) / 10 and 100 h dP/dx; outputs 1000 tau_x and 1000 tau_z.
"""
import ctypes

import numpy as np

from . import _lib

_fp = ctypes.POINTER(ctypes.c_float)


def _f(a):
    return a.ctypes.data_as(_fp)


class WallNet:
    def __init__(self, device=0, seed=1):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check_mlp(self.lib.blgpu_mlp_create(int(device), ctypes.c_ulonglong(seed), ctypes.byref(h)))
        self.h = h
        self.nparams = int(self.lib.blgpu_mlp_nparams())
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.blgpu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        _lib.check_mlp(rc, self.h)

    @property
    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        self._ck(self.lib.blgpu_mlp_get_params(self.h, _f(p), self.nparams))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._ck(self.lib.blgpu_mlp_set_params(self.h, _f(p), p.size))

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], 2), dtype=np.float32)
        self._ck(self.lib.blgpu_mlp_forward(self.h, _f(X), X.shape[0], _f(Y)))
        return Y

    def gradient(self, X, T):
        """(loss, gradient) over host samples X[rows][4], T[rows][2]."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        self._ck(self.lib.blgpu_mlp_gradient(self.h, _f(X), _f(T), X.shape[0], _f(g), ctypes.byref(loss)))
        return float(loss.value), g

    def add_data(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        self._ck(self.lib.blgpu_mlp_add_data(self.h, _f(X), _f(T), X.shape[0]))

    def sample(self, solver, jh):
        """Append the wall samples of a Solver's current state (row jh)."""
        rc = self.lib.blgpu_mlp_sample(self.h, solver.ctx, int(jh))
        if rc:
            _lib.check(rc, solver.ctx)

    def clear_data(self):
        self._ck(self.lib.blgpu_mlp_clear_data(self.h))

    @property
    def num_samples(self):
        return int(self.lib.blgpu_mlp_num_samples(self.h))

    def data(self):
        n = self.num_samples
        X = np.zeros((n, 4), dtype=np.float32)
        T = np.zeros((n, 2), dtype=np.float32)
        self._ck(self.lib.blgpu_mlp_get_data(self.h, _f(X), _f(T), n))
        return X, T

    def train(self, steps, batch=8192, lr=1e-3):
        """Adam steps on the device training set; returns the last batch loss."""
        loss = ctypes.c_float()
        self._ck(self.lib.blgpu_mlp_train(self.h, int(steps), int(batch), ctypes.c_float(lr), ctypes.byref(loss)))
        return float(loss.value)

    def steps(self):
        n = ctypes.c_longlong()
        self._ck(self.lib.blgpu_mlp_steps(self.h, ctypes.byref(n)))
        return int(n.value)

    def loss_history(self, n):
        h = np.zeros(n, dtype=np.float32)
        self._ck(self.lib.blgpu_mlp_loss_history(self.h, _f(h), int(n)))
        return h

    def eval(self):
        """Loss over the whole training set."""
        loss = ctypes.c_float()
        self._ck(self.lib.blgpu_mlp_eval(self.h, ctypes.byref(loss)))
        return float(loss.value)
