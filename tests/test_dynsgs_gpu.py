"""Dynamic Smagorinsky eddy viscosity on the device (LES = 2: coefficient
averaged in z, subgrid.f90:261-414; LES = 3: pointwise, subgrid.f90:420-583)
against the oracle: one evaluation on noisy fields, LES steps, and the mixed
form against FP64."""
import numpy as np
import pytest

import oracle
from blgpu import cases, FP64, MIXED

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def noisy(nx, ny, nz, seed, amp, **kw):
    c = cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=20.0, ly=5.0, lz=3.0, **kw)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + amp * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + amp * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + amp * rng.standard_normal(c.W.shape))
    return c


@pytest.mark.parametrize("model", [2, 3])
@pytest.mark.parametrize("grid", [(26, 14, 11), (61, 17, 16), (300, 9, 40)])
def test_dynamic_nu_t_matches_oracle(gpu, model, grid):
    """300 x 9 x 40: several 128-point x blocks of the filter kernel (the
    halo at ib-1 and ib+128 and the guard at the last block) and three
    16-plane k blocks, against the oracle."""
    c = noisy(*grid, seed=31, amp=0.05)
    s = cases.solver_for(c, les_model=model)
    o = oracle.oracle_for(c)
    nut = s.compute_eddy_viscosity()
    ref = o.dynamic_smagorinsky(model)
    assert ref.max() > 0 and (ref > 0).mean() > 0.1
    # FP64 in the oracle's evaluation order; sqrt against pow(x, 0.5) and the
    # Mij Lij / Mij Mij quotient leave a few ulps
    assert np.abs(nut - ref).max() <= 1e-12 * np.abs(ref).max()
    s.close()


@pytest.mark.parametrize("model", [2, 3])
def test_dynamic_les_steps_match_oracle(gpu, model):
    c = noisy(40, 13, 18, seed=32, amp=2e-3, cfl=-2e-3)
    s = cases.solver_for(c, les_model=model)
    o = oracle.oracle_for(c)
    o.set_les(model)
    for _ in range(3):
        s.time_step()
        o.step()
    U, V, W, _, _ = s.download_state()
    Ur, Vr, Wr, _, _ = o.state()
    assert rel(U, Ur) < 1e-10 and rel(V, Vr) < 1e-10 and rel(W, Wr) < 1e-10
    assert rel(s.nu_t(), o.nu_t()) < 1e-9
    s.close()


@pytest.mark.parametrize("model", [2, 3])
def test_dynamic_les_mixed_close_to_fp64(gpu, model):
    c = cases.turbulent_case(nx=66, ny=33, nz=24, lx=8.0, ly=2.0, lz=3.0, seed=7, cfl=-0.01)
    a = cases.solver_for(c, precision=MIXED, les_model=model)
    b = cases.solver_for(c, precision=FP64, les_model=model)
    a.advance(5)
    b.advance(5)
    for x, y in zip(a.download_state()[:3], b.download_state()[:3]):
        assert np.all(np.isfinite(x)) and rel(x, y) < 1e-5
    assert rel(a.nu_t(), b.nu_t()) < 1e-3
    a.close()
    b.close()
