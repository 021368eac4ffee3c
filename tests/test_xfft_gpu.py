"""The x transforms (divergence + DCT-II, inverse DCT): the two-pass
register FFT (N = nx-2 = A B, compile-time indices) against the Stockham
shared-memory FFT and the FP64 path, at the built lengths (812 = 29 x 28,
510 = 17 x 30, 190 = 19 x 10, 126 = 14 x 9 in the mixed form; 812 in FP64),
for one projection and for a few steps."""
import numpy as np
import pytest

from blgpu import BlgpuError, cases, FP64, MIXED

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def noisy(nx, ny, nz, seed):
    c = cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=40.0, ly=5.0, lz=4.0)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + 0.05 * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + 0.05 * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + 0.05 * rng.standard_normal(c.W.shape))
    c.cfl = -0.01
    return c


# (814, 10, 13): an odd number of lines (9 x 11), so the last warp holds one real line
@pytest.mark.parametrize("nx,ny,nz", [(814, 9, 12), (814, 17, 33), (512, 13, 20), (814, 10, 13), (192, 9, 12),
                                      (128, 11, 14)])
def test_two_pass_x_transform_matches_stockham_and_fp64(gpu, nx, ny, nz):
    c = noisy(nx, ny, nz, nx + ny)
    out = {}
    for name, prec, xfft in (("two", MIXED, 2), ("stock", MIXED, 1), ("fp64", FP64, 0)):
        s = cases.solver_for(c, precision=prec)
        if prec == MIXED:
            assert s.tiles()["xfft"] == 0
            s.set_tiles(xfft=xfft)
        s.apply_boundary_conditions(1)
        s.compute_projection_step(1)
        s.apply_boundary_conditions(1)
        out[name] = (s.download_state()[:3], s.rhs_p(), s.check_divergence())
        s.close()
    (U2, V2, W2), p2, d2 = out["two"]
    (Us, Vs, Ws), ps, ds = out["stock"]
    (U6, V6, W6), p6, d6 = out["fp64"]
    # FP32 pressure against FP64: 5e-6 to 3e-5 relative for the two-pass
    # transform, 3e-5 to 5e-5 for the Stockham one at N = 812
    assert rel(p2, p6) < 1e-4 and rel(ps, p6) < 1e-4, (rel(p2, p6), rel(ps, p6))
    assert rel(p2, ps) < 1e-4
    for a, b in ((U2, U6), (V2, V6), (W2, W6)):
        assert rel(a, b) < 1e-5
    assert d2 < 1e-3 and d2 <= 10 * ds + 1e-6


@pytest.mark.parametrize("nw", [1, 3, 5, 8])
def test_two_pass_lines_per_cta(gpu, nw):
    """Every lines-per-CTA choice of both kernels gives the same bits."""
    c = noisy(814, 9, 12, 5)
    runs = []
    for t in (dict(xfft=2), dict(xfft=2, dct_nw=nw, idct_nw=nw)):
        s = cases.solver_for(c, precision=MIXED)
        s.set_tiles(**t)
        s.apply_boundary_conditions(1)
        s.compute_projection_step(1)
        runs.append((s.download_state()[:3], s.rhs_p()))
        s.close()
    for a, b in zip(runs[0][0] + (runs[0][1],), runs[1][0] + (runs[1][1],)):
        assert np.array_equal(a, b)


def test_two_pass_steps_close_to_fp64(gpu):
    c = cases.turbulent_case(nx=814, ny=17, nz=24, lx=40.0, ly=2.0, lz=3.0, seed=3, cfl=-0.01)
    a = cases.solver_for(c, precision=MIXED)
    b = cases.solver_for(c, precision=FP64)
    a.advance(5)
    b.advance(5)
    for x, y in zip(a.download_state()[:3], b.download_state()[:3]):
        assert np.all(np.isfinite(x))
        assert rel(x, y) < 1e-5


def test_two_pass_refused_where_not_built(gpu):
    c = noisy(66, 9, 12, 1)
    s = cases.solver_for(c, precision=MIXED)
    with pytest.raises(BlgpuError, match="xfft 2"):
        s.set_tiles(xfft=2)
    s.set_tiles(xfft=1)
    s.close()
    # FP64: the two-pass transform is built for N = 812 only
    f = cases.solver_for(noisy(128, 9, 12, 2), precision=FP64)
    with pytest.raises(BlgpuError, match="xfft 2"):
        f.set_tiles(xfft=2)
    f.close()
    f = cases.solver_for(noisy(814, 9, 12, 2), precision=FP64)
    f.set_tiles(xfft=2)
    assert f.tiles()["xfft"] == 2
    f.close()


@pytest.mark.parametrize("nx,ny,nz", [(814, 9, 12), (814, 10, 13)])
def test_fp64_two_pass_matches_stockham(gpu, nx, ny, nz):
    """The FP64 instance of the two-pass transform (the FP64 default at
    N = 812) against the FP64 Stockham transform: one projection agrees to
    FP64 rounding, and every lines-per-CTA choice gives the same bits."""
    c = noisy(nx, ny, nz, nx + 2 * ny)
    out = {}
    for name, t in (("two", dict(xfft=2)), ("stock", dict(xfft=1)), ("two3", dict(xfft=2, dct_nw=3, idct_nw=6))):
        s = cases.solver_for(c, precision=FP64)
        s.set_tiles(**t)
        s.apply_boundary_conditions(1)
        s.compute_projection_step(1)
        out[name] = (s.download_state()[:3], s.rhs_p())
        s.close()
    (a, pa), (b, pb), (d, pd) = out["two"], out["stock"], out["two3"]
    assert rel(pa, pb) < 1e-12
    for x, y in zip(a, b):
        assert rel(x, y) < 1e-13
    for x, y in zip(a + (pa,), d + (pd,)):
        assert np.array_equal(x, y)
