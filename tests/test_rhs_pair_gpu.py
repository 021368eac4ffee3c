"""The mixed form's DNS RHS with two x-points per thread (shared face fluxes,
k-1 face terms carried between planes, one-plane-ahead fetches), in scalar
FP32 (rhs_pts 2), in packed FP32x2 instructions (rhs_pts 3) and packed with
TMA-staged planes (rhs_pts 4), against the
one-point register-window kernel and the FP64 oracle, for odd and even nx
(an even nx leaves the last pair half inside the range)."""
import numpy as np
import pytest

import oracle
from blgpu import cases, FP64, MIXED

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def noisy(nx, ny, nz, seed, amp=5e-2):
    c = cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=20.0, ly=5.0, lz=3.0)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + amp * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + amp * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + amp * rng.standard_normal(c.W.shape))
    return c


@pytest.mark.parametrize("grid", [(26, 14, 11), (27, 14, 11), (37, 9, 24), (60, 17, 15), (131, 33, 70)])
def test_pair_rhs_matches_single_and_fp64(gpu, grid):
    c = noisy(*grid, seed=sum(grid))
    ref = oracle.oracle_for(c).rhs(c.U, c.V, c.W)
    got = {}
    for pts in (1, 2, 3, 4):
        s = cases.solver_for(c, precision=MIXED)
        s.set_tiles(rhs_pts=pts)
        assert s.tiles()["rhs_pts"] == pts
        got[pts] = s.compute_rhs(c.U, c.V, c.W)
        s.close()
    for q in range(3):
        assert got[1][q].shape == ref[q].shape
        assert rel(got[1][q], ref[q]) < 3e-5
        for pts in (2, 3, 4):
            assert got[pts][q].shape == ref[q].shape
            assert rel(got[pts][q], ref[q]) < 3e-5
            assert rel(got[pts][q], got[1][q]) < 3e-5
            # the zero columns (u at i = nx-1, v and w at i = nx) stay exactly zero
            assert np.all(got[pts][q][-1] == 0.0)


@pytest.mark.parametrize("nx", [66, 67])
def test_pair_steps_match_single(gpu, nx):
    c = cases.turbulent_case(nx=nx, ny=33, nz=40, lx=8.0, ly=2.0, lz=3.0, seed=nx, cfl=-0.01)
    runs = {}
    for pts in (1, 2, 3, 4):
        s = cases.solver_for(c, precision=MIXED)
        s.set_tiles(rhs_pts=pts)
        s.advance(5)
        runs[pts] = s.download_state()[:3]
        s.close()
    b = cases.solver_for(c, precision=FP64)
    b.advance(5)
    ref = b.download_state()[:3]
    b.close()
    for pts in (2, 3, 4):
        for x1, x2, r in zip(runs[1], runs[pts], ref):
            assert np.all(np.isfinite(x2))
            assert rel(x2, x1) < 1e-6
            assert rel(x2, r) < 1e-5


@pytest.mark.parametrize("pts", [2, 3, 4])
def test_pair_rhs_chunk_length_does_not_change_results(gpu, pts):
    """The carried k-1 face terms round as the ones formed at a chunk's first
    plane, so the k-planes per CTA leave the steps bit-identical."""
    c = cases.turbulent_case(nx=67, ny=33, nz=40, lx=8.0, ly=2.0, lz=3.0, seed=5, cfl=-0.01)
    runs = []
    for kc in (8, 5, 37):
        s = cases.solver_for(c, precision=MIXED)
        s.set_tiles(rhs_pts=pts, rhs_kc=kc)
        s.advance(3)
        runs.append(s.download_state()[:3])
        s.close()
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert np.array_equal(a, b)


def test_packed_forms_agree_bitwise(gpu):
    """The TMA-staged kernel evaluates the packed kernel's expressions on the
    same values, only read from shared memory: the steps agree bit for bit
    (odd nx: a CTA whose last pair is half outside; ny - 1 = 40 rows: a
    partial row block; the last chunk of k-planes short)."""
    c = cases.turbulent_case(nx=131, ny=41, nz=29, lx=8.0, ly=2.0, lz=3.0, seed=9, cfl=-0.01)
    runs = []
    for pts in (3, 4):
        s = cases.solver_for(c, precision=MIXED)
        s.set_tiles(rhs_pts=pts, rhs_kc=8)
        s.advance(3)
        runs.append(s.download_state()[:3])
        s.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
