"""Streamed state transfers (blgpu_upload_state_async / _download_state_async):
a sequence of states passed through the solver with the copies overlapping
the steps gives the same bits as the synchronous upload / advance / download
of each state."""
import numpy as np
import pytest
import torch

from blgpu import cases, FP64, MIXED

pytestmark = pytest.mark.gpu


def pinned(shape):
    n = int(np.prod(shape))
    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape, order="F")


@pytest.mark.parametrize("precision", [MIXED, FP64])
def test_streamed_states_match_synchronous(gpu, precision):
    c = cases.turbulent_case(nx=66, ny=33, nz=24, lx=8.0, ly=2.0, lz=3.0, seed=5, cfl=-0.01)
    rng = np.random.default_rng(11)
    states = []
    for q in range(3):
        states.append(tuple(np.asfortranarray(a + 1e-2 * rng.standard_normal(a.shape)) for a in (c.U, c.V, c.W)))
    ref = []
    s = cases.solver_for(c, precision=precision)
    for U, V, W in states:
        s.upload_state(U, V, W, 0.0)
        s.advance(2)
        ref.append(s.download_state()[:3])
    s.close()
    s = cases.solver_for(c, precision=precision)
    ins, outs = [], []
    for U, V, W in states:
        i3 = tuple(pinned(a.shape) for a in (U, V, W))
        for d, a in zip(i3, (U, V, W)):
            d[...] = a
        o3 = tuple(pinned(a.shape) for a in (U, V, W))
        ins.append(i3)
        outs.append(o3)
        s.upload_state_async(*i3, 0.0)
        s.advance(2)
        s.download_state_async(*o3)
    s.sync()
    s.close()
    for r, o in zip(ref, outs):
        for a, b in zip(r, o):
            assert np.array_equal(a, b)
