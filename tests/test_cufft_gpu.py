"""The cuFFT comparison path of the Poisson solve (poisson = POISSON_CUFFT:
solve_poisson_gpu, projection.f90:93-204, with the plans of
cufft_init_plans, cufft_solver.f90:26-62) against the oracle and against the
hand-written transforms on the same states."""
import numpy as np
import pytest

import oracle
from blgpu import cases, FP64, MIXED, POISSON_CUFFT, POISSON_NATIVE

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def noisy(nx, ny, nz, seed=0, amp=1e-2, **kw):
    c = cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=20.0, ly=5.0, lz=3.0, **kw)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + amp * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + amp * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + amp * rng.standard_normal(c.W.shape))
    return c


@pytest.mark.parametrize("grid", [(26, 14, 11), (60, 17, 15), (37, 9, 24), (131, 33, 24)])
def test_cufft_projection_fp64(gpu, grid):
    """Boundary pass, projection, boundary pass (the substep's order): rhs_p
    and the projected fields within 1e-12 of the oracle and of the native
    kernels, and the field divergence free to 1e-12."""
    c = noisy(*grid, seed=4)
    out = {}
    for name, po in (("cufft", POISSON_CUFFT), ("native", POISSON_NATIVE)):
        s = cases.solver_for(c, poisson=po)
        s.set_dt(0.01)
        s.apply_boundary_conditions(2)
        s.compute_projection_step(2)
        out[name] = (s.rhs_p()[:, :, :-1],) + tuple(s.download_state()[:3])
        s.apply_boundary_conditions(2)
        assert s.check_divergence() < 1e-12
        s.close()
    o = oracle.oracle_for(c)
    o.set_dt(0.01)
    o.apply_bc(2)
    o.projection(2)
    ref = (o.rhs_p()[:, :, :-1],) + tuple(o.state()[:3])
    for a, b, r in zip(out["cufft"], out["native"], ref):
        assert rel(a, r) < 1e-12, rel(a, r)
        assert rel(a, b) < 1e-12, rel(a, b)


def test_cufft_steps_fp64(gpu):
    """10 RK3 steps of config 1 (128 x 64 x 32 laminar) on the cuFFT path:
    the FP64 parity bar against the oracle."""
    c = cases.laminar_case()
    s = cases.solver_for(c, poisson=POISSON_CUFFT)
    o = oracle.oracle_for(c, threads=4)
    s.advance(10)
    o.advance(10)
    U, V, W, P, t = s.download_state()
    Ur, Vr, Wr, Pr, tr = o.state()
    # W stays at round-off size in this z-independent flow: compared absolutely
    assert rel(U, Ur) < 1e-10 and rel(V, Vr) < 1e-10 and np.abs(W - Wr).max() < 1e-12
    assert rel(P, Pr) < 1e-8
    assert s.check_divergence() <= 1e-12
    s.close()


def test_cufft_mixed_turbulent(gpu):
    """Mixed form with C2C plans on a turbulent box with Lund inflow: within
    the mixed form's tolerance of the FP64 oracle after 5 steps, and of the
    native mixed path."""
    # fixed dt: on this coarse y grid the CFL dt of compute_dt (the viscous
    # limit, time_integration.f90:546-575) would be far above the convective one
    c = cases.turbulent_case(nx=130, ny=33, nz=34, lx=16.0, ly=2.0, lz=3.0, seed=11, cfl=-0.01)
    res = {}
    for po in (POISSON_CUFFT, POISSON_NATIVE):
        s = cases.solver_for(c, precision=MIXED, poisson=po)
        s.advance(5)
        res[po] = s.download_state()[:3]
        assert s.check_divergence() < 1e-3
        s.close()
    o = oracle.oracle_for(c, threads=4)
    o.advance(5)
    ref = o.state()[:3]
    errs = [(rel(a, r), rel(a, b)) for a, b, r in zip(res[POISSON_CUFFT], res[POISSON_NATIVE], ref)]
    print("mixed cuFFT path: (vs oracle, vs native) per component", errs)
    for name, (eo, en) in zip("uvw", errs):
        assert eo < (1e-4 if name == "v" else 1e-5), (name, eo)
        assert en < (1e-4 if name == "v" else 1e-5), (name, en)
