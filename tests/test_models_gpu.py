"""Device models and diagnostics against the oracle: Smagorinsky eddy
viscosity (subgrid.f90:609-730), LES steps, z-averaged statistics and Cf
(statistics.f90:26-201), the equilibrium law of the wall solved by Newton
(wallmodel.f90:1951-1985, Newton_solver.f90), and the laminar skin friction
of config 1 against the Blasius value 0.664/sqrt(Re_x)."""
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


@pytest.mark.parametrize("grid", [(26, 14, 11), (60, 17, 15)])
def test_smagorinsky_matches_oracle(gpu, grid):
    c = noisy(*grid, seed=21, amp=0.05)
    s = cases.solver_for(c, les_model=1)
    o = oracle.oracle_for(c)
    nut = s.compute_eddy_viscosity()
    ref = o.smagorinsky()
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    assert np.abs(nut[inner] - ref[inner]).max() <= 1e-14 * np.abs(ref).max()
    assert (nut[inner] >= 0).all() and ref.max() > 0
    s.close()


def test_les_steps_match_oracle(gpu):
    c = noisy(40, 13, 18, seed=22, amp=2e-3, cfl=-2e-3)
    s = cases.solver_for(c, les_model=1)
    o = oracle.oracle_for(c)
    o.set_les(1)
    for _ in range(4):
        s.time_step()
        o.step()
    U, V, W, _, _ = s.download_state()
    Ur, Vr, Wr, _, _ = o.state()
    assert rel(U, Ur) < 1e-10 and rel(V, Vr) < 1e-10 and rel(W, Wr) < 1e-10
    s.close()


def test_statistics_match_oracle(gpu):
    c = noisy(60, 17, 15, seed=23, amp=1e-3, cfl=-2e-3)
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    for _ in range(2):
        s.time_step()
        o.step()
    a, b = s.compute_statistics(), o.statistics()
    for k in ("Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "UVmean", "Pmean", "P2mean", "Cf",
              "dUdy_wall"):
        assert rel(a[k], b[k]) < 1e-10, k
    for k in ("theta_inlet", "delta99_inlet", "Retheta_inlet"):
        assert a[k] == pytest.approx(b[k], rel=1e-10)
    s.close()


def test_law_of_the_wall_matches_oracle(gpu):
    c = cases.turbulent_case(nx=64, ny=49, nz=18, lx=10.0, ly=3.0, lz=2.0)
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    guess = (0.5 * 0.027 * (c.x / c.nu) ** (-1.0 / 7.0)) ** 0.5  # utau_ref, initialization.f90:740
    u1, it1 = s.law_of_the_wall(guess)
    u2, it2 = o.law_of_the_wall(guess)
    assert it1 == it2 and it1 < 30
    assert np.abs(u1 - u2).max() <= 1e-12 * np.abs(u2).max()
    # the solution satisfies the log law at y = yg(3)
    yg = cases.centres_ghost(c.y)
    Um = c.U[1:-1, 2, 1:-1].mean(axis=1)
    f = u1[1:-1] / 0.38 * np.log(yg[2] * u1[1:-1] / c.nu) + 5.2 * u1[1:-1] - Um
    assert np.abs(f).max() < 1e-8
    s.close()


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_laminar_cfg1_skin_friction_blasius(gpu, precision):
    """Config 1: 200 RK3 steps at CFL 0.5; Cf(x) within 2% of 0.664/sqrt(Re_x)
    away from the inlet (3 points) and the outlet (5 points), as the
    reference's laminar_test/postprocess.py:164-170 compares it."""
    c = cases.laminar_case()
    s = cases.solver_for(c, precision=precision)
    s.advance(200)
    st = s.compute_statistics()
    rex = c.x / c.nu
    cf_bl = 0.664 / np.sqrt(rex)
    sl = slice(3, c.nx - 5)
    err = np.abs(st["Cf"][sl] - cf_bl[sl]) / cf_bl[sl]
    assert err.max() < 0.02, err.max()
    assert s.check_divergence() < (1e-12 if precision == FP64 else 1e-4)
    s.close()
