"""The mixed form's z transforms on the tensor cores (TF32 products with a
three-term split; mma.sync and tcgen05 with tensor-memory accumulators):
against the FP32 direct sums and against the FP64 path, for odd and even z
lengths of every served order (M/2+1 rounded up to 16: 32, 48, 64, 80, 96)."""
import numpy as np
import pytest

from blgpu import cases, FP64, MIXED

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def noisy(nz, seed):
    c = cases.laminar_case(nx=34, ny=17, nz=nz, lx=10.0, ly=5.0, lz=4.0)
    rng = np.random.default_rng(seed)
    c.U = np.asfortranarray(c.U + 0.05 * rng.standard_normal(c.U.shape))
    c.V = np.asfortranarray(c.V + 0.05 * rng.standard_normal(c.V.shape))
    c.W = np.asfortranarray(c.W + 0.05 * rng.standard_normal(c.W.shape))
    c.cfl = -0.01
    return c


@pytest.mark.parametrize("form", [2, 3])
@pytest.mark.parametrize("nz", [64, 65, 96, 97, 127, 159, 193, 194])
def test_tensor_core_z_transform_matches_direct_and_fp64(gpu, nz, form):
    c = noisy(nz, nz)
    out = {}
    for name, prec, zdft in (("tc", MIXED, form), ("direct", MIXED, 1), ("fp64", FP64, 0)):
        s = cases.solver_for(c, precision=prec)
        if prec == MIXED:
            s.set_tiles(zdft=zdft)
        # boundary pass before (compatible Neumann problem) and after (ghost
        # cells the divergence check reads), as in a substep
        s.apply_boundary_conditions(1)
        s.compute_projection_step(1)
        s.apply_boundary_conditions(1)
        out[name] = (s.download_state()[:3], s.rhs_p(), s.check_divergence())
        s.close()
    (Ut, Vt, Wt), pt, dt = out["tc"]
    (Ud, Vd, Wd), pd, dd = out["direct"]
    (U6, V6, W6), p6, d6 = out["fp64"]
    # FP32 pressure against FP64 on a noisy field (both z-transform forms
    # alike), then the two forms against each other
    assert rel(pt, p6) < 3e-5 and rel(pd, p6) < 3e-5, (rel(pt, p6), rel(pd, p6))
    assert rel(pt, pd) < 1e-5
    for a, b in ((Ut, U6), (Vt, V6), (Wt, W6)):
        assert rel(a, b) < 1e-5
    assert dt < 1e-3 and dt <= 10 * dd + 1e-6


@pytest.mark.parametrize("form", [0, 2, 3])
def test_tensor_core_path_steps_close_to_fp64(gpu, form):
    c = cases.turbulent_case(nx=66, ny=33, nz=193, lx=8.0, ly=2.0, lz=8.0, seed=9, cfl=-0.01)
    a = cases.solver_for(c, precision=MIXED)
    assert a.tiles()["zdft"] == 0
    a.set_tiles(zdft=form)
    b = cases.solver_for(c, precision=FP64)
    a.advance(10)
    b.advance(10)
    A, B = a.download_state()[:3], b.download_state()[:3]
    for x, y in zip(A, B):
        assert rel(x, y) < 1e-5
