"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bars: the FP64 RHS is bit-identical to the oracle's restatement of
equations.f90; boundary conditions and projection agree to rounding; full
steps agree to relative L2 <= 1e-10 after 10 steps with max divergence
<= 1e-12 (the FP64 target); the mixed form stays within 1e-5.
"""
import numpy as np
import pytest

import oracle
from blgpu import cases, Solver, FP64, MIXED

pytestmark = pytest.mark.gpu

REL10 = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def noisy_laminar(nx, ny, nz, seed=0, amp=1e-2, **kw):
    c = cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=kw.pop("lx", 20.0), ly=kw.pop("ly", 5.0),
                           lz=kw.pop("lz", 3.0), **kw)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + amp * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + amp * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + amp * rng.standard_normal(c.W.shape))
    return c


GRIDS = [(26, 14, 11), (60, 17, 15), (128, 64, 32), (37, 9, 24)]


@pytest.mark.parametrize("grid", GRIDS)
def test_rhs_bit_identical(gpu, grid):
    c = noisy_laminar(*grid, seed=1)
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    got = s.compute_rhs(c.U, c.V, c.W)
    ref = o.rhs(c.U, c.V, c.W)
    for g, r in zip(got, ref):
        assert g.shape == r.shape
        assert np.array_equal(g, r), np.abs(g - r).max()
    s.close()


@pytest.mark.parametrize("seed", [3, 4])
def test_rhs_bit_identical_turbulent(gpu, seed):
    """The FP64 RHS on a stretched turbulent box: wall-refined y spacings,
    10 % noise, 15 M quotients, each formed from the reciprocal tables by
    Markstein's correction, must equal the oracle's IEEE divisions bit for
    bit, in every FP64 kernel: the two-point window (the default), the
    one-point kernel of global loads (rhs_pts 1) and the TMA-fed one (4)."""
    c = cases.turbulent_case(nx=200, ny=65, nz=48, lx=20.0, ly=2.0, lz=3.0, seed=seed, cfl=-0.01)
    ref = oracle.oracle_for(c).rhs(c.U, c.V, c.W)
    for pts in (0, 1, 4):
        s = cases.solver_for(c)
        s.set_tiles(rhs_pts=pts)
        got = s.compute_rhs(c.U, c.V, c.W)
        s.close()
        for g, r in zip(got, ref):
            assert g.shape == r.shape
            assert np.array_equal(g, r), np.abs(g - r).max()


@pytest.mark.parametrize("grid", GRIDS[:3])
@pytest.mark.parametrize("rk_step", [1, 2, 3])
def test_boundary_conditions(gpu, grid, rk_step):
    c = noisy_laminar(*grid, seed=2)
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    for x in (s, o):
        x.set_dt(0.01)
    s.apply_boundary_conditions(rk_step)
    o.apply_bc(rk_step)
    U, V, W, _, _ = s.download_state()
    Ur, Vr, Wr, _, _ = o.state()
    assert np.array_equal(V, Vr) and np.array_equal(W, Wr)
    # U differs only by the summation order of the mass-flux reduction
    assert np.abs(U - Ur).max() <= 1e-14 * np.abs(Ur).max()
    s.close()


# N = nx-2 = 129 = 3*43 and 254 = 2*127: x transforms with a prime stage
# above the register butterflies (direct summation over (butterfly, output))
@pytest.mark.parametrize("grid", GRIDS + [(131, 9, 12), (256, 9, 12)])
def test_projection(gpu, grid):
    c = noisy_laminar(*grid, seed=3)
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    for x in (s, o):
        x.set_dt(0.02)
    s.apply_boundary_conditions(1)
    o.apply_bc(1)
    s.compute_projection_step(1)
    o.projection(1)
    U, V, W, P, _ = s.download_state()
    Ur, Vr, Wr, Pr, _ = o.state()
    assert rel(U, Ur) < 1e-13 and rel(V, Vr) < 1e-12 and rel(W, Wr) < 1e-12
    assert rel(P, Pr) < 1e-11
    rp, rpr = s.rhs_p()[:, :, :-1], o.rhs_p()[:, :, :-1]
    assert rel(rp, rpr) < 1e-11
    s.apply_boundary_conditions(1)
    o.apply_bc(1)
    assert s.check_divergence() < 1e-12
    assert abs(s.check_divergence() - o.max_divergence()) < 1e-12
    s.close()


@pytest.mark.parametrize("rk", [3, 2, 1])
def test_steps_small(gpu, rk):
    """5 steps at a fixed dt (CFL < 0) on a grid with nzp = 13 (prime) and
    N = 58 = 2*29 (radix-29 stage)."""
    c = noisy_laminar(60, 17, 15, seed=4, amp=1e-3, rk_scheme=rk, cfl=-2e-3)
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    for _ in range(5):
        s.time_step()
        o.step()
    U, V, W, P, t = s.download_state()
    Ur, Vr, Wr, Pr, tr = o.state()
    assert t == pytest.approx(tr, rel=1e-15)
    assert rel(U, Ur) < REL10 and rel(V, Vr) < REL10 and rel(W, Wr) < REL10
    assert s.check_divergence() <= 1e-12
    s.close()


@pytest.mark.parametrize("grid", GRIDS)
def test_compute_dt_exact(gpu, grid):
    """compute_dt (time_integration.f90:528-591): the device max-reduction
    gives the oracle's dt to the last bit, with the convective bound active."""
    c = noisy_laminar(*grid, seed=8, amp=0.3)
    c.U = np.asfortranarray(c.U + 2.0)
    c.V = np.asfortranarray(c.V + 1.0)
    c.W = np.asfortranarray(c.W + 1.0)
    c.cfl = 0.37
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    assert s.compute_dt() == o.compute_dt()
    s.close()


@pytest.mark.parametrize("comp", [0, 1, 2])
@pytest.mark.parametrize("grid", GRIDS)
def test_compute_dt_exact_each_component(gpu, grid, comp):
    """dt set by the convective bound of one velocity component: the other
    two are zero at one interior point (their bounds infinite) and the
    chosen one is shifted by 50, so that its bound is below the viscous
    one; the oracle's dt to the last bit in each case."""
    c = noisy_laminar(*grid, seed=9 + comp, amp=0.3)
    F = [c.U, c.V, c.W]
    for q in range(3):
        F[q] = np.array(F[q], order="F")
        if q == comp:
            F[q] += 50.0
        else:
            F[q][3, 3, 3] = 0.0
    c.U, c.V, c.W = F
    c.cfl = 0.37
    s = cases.solver_for(c)
    o = oracle.oracle_for(c)
    dt = o.compute_dt()
    assert 0 < dt < 0.37 * 3.0 / 50.0
    assert s.compute_dt() == dt
    s.close()


@pytest.mark.parametrize("grid", GRIDS)
def test_compute_dt_mixed(gpu, grid):
    """The mixed form's compute_dt (four points per thread, 16-byte loads)
    against the oracle on the FP32-rounded fields; the w bound is taken as
    1 / min(|w| / C) there, so agreement is to rounding, not bitwise."""
    c = noisy_laminar(*grid, seed=9, amp=0.3)
    c.U = np.asfortranarray((c.U + 2.0).astype(np.float32).astype(np.float64))
    c.V = np.asfortranarray((c.V + 1.0).astype(np.float32).astype(np.float64))
    c.W = np.asfortranarray((c.W + 1.0).astype(np.float32).astype(np.float64))
    c.cfl = 0.37
    s = cases.solver_for(c, precision=MIXED)
    o = oracle.oracle_for(c)
    assert s.compute_dt() == pytest.approx(o.compute_dt(), rel=1e-14)
    s.close()


def test_laminar_cfg1_10_steps(gpu):
    """Config 1 (128x64x32 laminar Blasius, RK3, CFL 0.5): 10 steps."""
    c = cases.laminar_case()
    s = cases.solver_for(c)
    o = oracle.oracle_for(c, threads=4)
    s.advance(10)
    o.advance(10)
    U, V, W, P, t = s.download_state()
    Ur, Vr, Wr, Pr, tr = o.state()
    assert rel(U, Ur) < REL10 and rel(V, Vr) < REL10
    assert np.abs(W - Wr).max() < 1e-12
    assert rel(P, Pr) < 1e-8
    assert s.check_divergence() <= 1e-12
    assert t == pytest.approx(tr, rel=1e-14)
    s.close()


def test_advance_graph_equals_eager(gpu):
    c = noisy_laminar(37, 9, 24, seed=5, amp=1e-3)
    a = cases.solver_for(c)
    b = cases.solver_for(c)
    a.advance(4)
    for _ in range(4):
        b.compute_dt()
        b.time_step()
    for x, y in zip(a.download_state()[:4], b.download_state()[:4]):
        assert np.array_equal(x, y)


def test_inflow_modes(gpu):
    """temporal inflow modes (boundary_conditions.f90:137-180)"""
    c = noisy_laminar(40, 13, 18, seed=6, amp=1e-4)
    rng = np.random.default_rng(9)
    n, m = 3, 2
    zmode = np.array([0.0, 1.0, 2.0]) * 2 * np.pi / 3.0
    tmode = np.array([1.0, 2.0]) * 0.1
    qu = 1e-3 * (rng.standard_normal((c.ny + 1, n, m)) + 1j * rng.standard_normal((c.ny + 1, n, m)))
    qv = 1e-3 * (rng.standard_normal((c.ny, n, m)) + 1j * rng.standard_normal((c.ny, n, m)))
    qw = 1e-3 * (rng.standard_normal((c.ny + 1, n, m)) + 1j * rng.standard_normal((c.ny + 1, n, m)))
    s = cases.solver_for(c)
    s.set_inflow_modes(zmode, tmode, qu, qv, qw)
    o = oracle.oracle_for(c)
    o.set_modes(zmode, tmode, qu, qv, qw)
    for _ in range(3):
        s.compute_dt()
        o.compute_dt()
        s.time_step()
        o.step()
    U, V, W, _, _ = s.download_state()
    Ur, Vr, Wr, _, _ = o.state()
    assert rel(U, Ur) < REL10 and rel(V, Vr) < REL10 and rel(W, Wr) < REL10
    s.close()


def test_mixed_precision_error(gpu):
    """FP32 fields/RHS/transforms with FP64 Thomas, zero mode and mass flux."""
    c = cases.laminar_case()
    s = cases.solver_for(c, precision=MIXED)
    o = oracle.oracle_for(c, threads=4)
    s.advance(10)
    o.advance(10)
    U, V, W, P, t = s.download_state()
    Ur, Vr, Wr, Pr, tr = o.state()
    eu, ev = rel(U, Ur), rel(V, Vr)
    assert eu < 1e-5 and ev < 1e-4, (eu, ev)
    assert s.check_divergence() < 1e-4
    s.close()


def test_errors_are_reported(gpu):
    s = Solver(32, 16, 16, 1e-3, -1e-3)
    with pytest.raises(Exception, match="grid"):
        s.time_step()
    s.close()


@pytest.mark.parametrize("precision", [FP64, MIXED])
@pytest.mark.parametrize("grid", [(60, 17, 15), (131, 33, 24), (37, 9, 24)])
def test_tiled_y_solve_matches_ring(gpu, precision, grid):
    """The TMA-tiled y-solve (one pass, both sweeps in shared memory) and the
    register-ring kernel evaluate the same recurrences in the same order."""
    c = noisy_laminar(*grid, seed=7, cfl=-2e-3)
    out = []
    for thomas in (1, 2):
        s = cases.solver_for(c, precision=precision)
        s.set_tiles(thomas=thomas)
        assert s.tiles()["thomas"] == thomas
        s.advance(3)
        out.append(s.download_state()[:4])
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


# NM = ny-1 of 16, 32, 8, 64 (the ensemble boxes), 256 (the headline box)
# and 100 (a last segment with fewer rows)
@pytest.mark.parametrize("precision", [FP64, MIXED])
@pytest.mark.parametrize("grid", [(60, 17, 15), (131, 33, 24), (37, 9, 24), (66, 65, 20), (50, 257, 12),
                                  (34, 101, 14)])
def test_tile_scan_y_solve_matches_ring(gpu, precision, grid):
    """The tiled y-solve with each mode's rows split over the tile's spare
    lanes (shuffle scans of the two linear recurrences) against the register
    ring: the same sums reassociated, so FP64 agrees to rounding and the
    mixed form to its FP32 storage of the intermediate rows."""
    c = noisy_laminar(*grid, seed=11, cfl=-2e-3)
    out = []
    for thomas in (1, 3):
        s = cases.solver_for(c, precision=precision)
        s.set_tiles(thomas=thomas)
        assert s.tiles()["thomas"] == thomas
        s.apply_boundary_conditions(1)
        s.compute_projection_step(1)
        out.append((s.download_state()[:3], s.rhs_p()))
        s.close()
    tol_p, tol_u = (1e-12, 1e-14) if precision == FP64 else (2e-5, 1e-6)
    assert rel(out[1][1], out[0][1]) < tol_p, rel(out[1][1], out[0][1])
    for a, b in zip(out[1][0], out[0][0]):
        assert rel(a, b) < tol_u, rel(a, b)


def test_tile_scan_y_solve_oracle_steps(gpu):
    """Five FP64 RK3 steps with the tile-scan y-solve against the oracle."""
    c = noisy_laminar(60, 17, 15, seed=12, amp=1e-3, cfl=-2e-3)
    s = cases.solver_for(c)
    s.set_tiles(thomas=3)
    o = oracle.oracle_for(c)
    for _ in range(5):
        s.time_step()
        o.step()
    for a, b in zip(s.download_state()[:3], o.state()[:3]):
        assert rel(a, b) < REL10
    assert s.check_divergence() < 1e-12
    s.close()
