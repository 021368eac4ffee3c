"""The allocation-free check_divergence entry point, through the C ABI.

blgpu_check_divergence_noalloc serves hosts that own all device memory and
cannot call cudaMalloc (for example an OpenACC program handing over its
data-region arrays by device address).  It must give the same maximum
divergence as the context-based blgpu_max_divergence on the same state, on
two calls in a row (the second call reuses the shared scratch left by the
first).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from blgpu import _lib, cases

pytestmark = pytest.mark.gpu


def _state(seed, amp):
    c = cases.laminar_case(nx=61, ny=23, nz=19, lx=20.0, ly=5.0, lz=3.0)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + amp * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + amp * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + amp * rng.standard_normal(c.W.shape))
    return c


def _existing(c):
    s = cases.solver_for(c)
    v = s.check_divergence()
    s.close()
    return v


def test_noalloc_divergence_matches_context_entry_point(gpu):
    import torch
    lib = _lib.load()
    dev = torch.device("cuda:0")
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    for seed, amp in ((11, 1e-2), (12, 3e-1)):
        c = _state(seed, amp)
        ref = _existing(c)
        t = [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev) for a in (c.U, c.V, c.W)]
        g = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (c.x, c.y, c.z)]
        torch.cuda.synchronize()
        rc = lib.blgpu_check_divergence_noalloc(*[ctypes.c_void_p(a.data_ptr()) for a in t + g],
                                                c.nx, c.ny, c.nz, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, lib.blgpu_last_error(None)
        torch.cuda.synchronize()
        got = float(out.item())
        assert got > 0
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)


def test_noalloc_rejects_oversized_grid(gpu):
    lib = _lib.load()
    dummy = ctypes.c_void_p(16)
    rc = lib.blgpu_check_divergence_noalloc(dummy, dummy, dummy, dummy, dummy, dummy, 64, 300, 300, dummy, None)
    assert rc == -1
    assert b"65536" in lib.blgpu_last_error(None)


def test_noalloc_divergence_keeps_nan(gpu):
    """A NaN in the velocity field gives a NaN maximum, as the context's check does."""
    import torch
    lib = _lib.load()
    dev = torch.device("cuda:0")
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    c = _state(13, 1e-2)
    U = np.array(c.U, order="F")
    U[20, 7, 5] = np.nan
    t = [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev) for a in (U, c.V, c.W)]
    g = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (c.x, c.y, c.z)]
    torch.cuda.synchronize()
    rc = lib.blgpu_check_divergence_noalloc(*[ctypes.c_void_p(a.data_ptr()) for a in t + g],
                                            c.nx, c.ny, c.nz, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0, lib.blgpu_last_error(None)
    torch.cuda.synchronize()
    assert np.isnan(float(out.item()))
