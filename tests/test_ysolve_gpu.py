"""The y-solve with the pivots formed in the kernel (tiles = thomas 3)
against the pivot-table forms: the same recurrences with the same roundings
(ysolve.cuh), so the states after a few steps are bit-identical, in FP64 and
in the mixed form (whose box-scale modes go through the FP64 plane)."""
import numpy as np
import pytest

from blgpu import cases, FP64, MIXED

pytestmark = pytest.mark.gpu


def noisy(nx, ny, nz, seed, amp=1e-2, **kw):
    c = cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=20.0, ly=5.0, lz=3.0, **kw)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + amp * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + amp * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + amp * rng.standard_normal(c.W.shape))
    return c


@pytest.mark.parametrize("precision", [FP64, MIXED])
@pytest.mark.parametrize("grid", [(60, 17, 15), (131, 33, 24), (37, 9, 24), (200, 40, 20)])
def test_recomputed_pivots_match_table(gpu, precision, grid):
    c = noisy(*grid, seed=8, cfl=-2e-3)
    out = []
    for thomas in (1, 2, 3):
        s = cases.solver_for(c, precision=precision)
        s.set_tiles(thomas=thomas)
        assert s.tiles()["thomas"] == thomas
        s.advance(3)
        out.append(s.download_state()[:4])
        s.close()
    for ref in out[1:]:
        for a, b in zip(out[0], ref):
            assert np.array_equal(a, b)


def test_recomputed_pivots_full_shape(gpu):
    """814 x 65 x 193 (x and z of the headline box): the tiles and the ring agree bitwise."""
    c = cases.turbulent_case(nx=814, ny=65, nz=193, ly=1.0, cfl=-5e-3)
    out = []
    for thomas in (1, 3):
        s = cases.solver_for(c, precision=MIXED)
        s.set_tiles(thomas=thomas)
        s.advance(2)
        out.append(s.download_state()[:3])
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
