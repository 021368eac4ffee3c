"""Ensembles of independent boxes advanced together (C ABI blgpu_ensemble_*).

Each box is an ordinary Solver; the Ensemble advances all of them with one
CUDA-graph launch per step whose branches run concurrently on the GPU.
"""
import ctypes

from . import _lib
from ._lib import check_ensemble


class Ensemble:
    def __init__(self, solvers):
        self.lib = _lib.load()
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s.ctx for s in self.solvers])
        h = ctypes.c_void_p()
        check_ensemble(self.lib.blgpu_ensemble_create(arr, len(self.solvers), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.blgpu_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        check_ensemble(rc, self.h)

    @property
    def cells(self):
        return sum(s.nx * s.ny * s.nz for s in self.solvers)

    def advance(self, nsteps):
        self._ck(self.lib.blgpu_ensemble_advance(self.h, int(nsteps)))

    def advance_sequential(self, nsteps):
        self._ck(self.lib.blgpu_ensemble_advance_sequential(self.h, int(nsteps)))

    def time(self, nsteps, sequential=False):
        """Device milliseconds of nsteps steps (graph capture excluded)."""
        ms = ctypes.c_double()
        self._ck(self.lib.blgpu_ensemble_time(self.h, int(nsteps), 1 if sequential else 0, ctypes.byref(ms)))
        return ms.value

    def sync(self):
        self._ck(self.lib.blgpu_ensemble_sync(self.h))

    def launches(self):
        return int(self.lib.blgpu_ensemble_launches(self.h))

    def autotune(self, steps=3):
        n = ctypes.c_int()
        self._ck(self.lib.blgpu_ensemble_autotune(self.h, int(steps), ctypes.byref(n)))
        return n.value
