"""CPU tests of the parity oracle (no GPU): its transforms, its ZGTSV
restatement and its Poisson variants are pinned against numpy/scipy and
against each other; the step is checked for discrete divergence."""
import numpy as np
import pytest
from scipy.fft import dct
from scipy.linalg.lapack import zgtsv

import oracle
from blgpu import cases


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12, 30, 62, 94, 97, 126, 190, 191, 254, 510, 812, 1022, 3248])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    scale = np.abs(ref).max()
    assert np.abs(oracle.fft(x) - ref).max() <= 1e-14 * scale
    assert np.abs(oracle.fft(x, inverse=True) - np.fft.ifft(x) * n).max() <= 1e-14 * scale


@pytest.mark.parametrize("n", [4, 7, 126, 191, 812])
def test_dct_matches_scipy(n):
    f = np.random.default_rng(n).standard_normal(n)
    c = oracle.dct2(f)
    assert np.abs(c - dct(f, 2) / 2).max() <= 1e-13 * np.abs(f).sum()


@pytest.mark.parametrize("pivot", [False, True])
def test_zgtsv_matches_lapack(pivot):
    rng = np.random.default_rng(7)
    n = 64
    dl = rng.random(n - 1) * (5.0 if pivot else 1.0) + 0j
    d = -3.0 - rng.random(n) + 0j
    du = rng.random(n - 1) + 0j
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x, info = oracle.zgtsv(dl, d, du, b)
    ref = zgtsv(dl, d, du, b)
    assert info == 0 and ref[4] == 0
    assert np.abs(x - ref[3]).max() <= 1e-14 * np.abs(ref[3]).max()


def test_zgtsv_singular_reports_info():
    x, info = oracle.zgtsv(np.zeros(3), np.array([1.0, 0.0, 1.0, 1.0]), np.zeros(3), np.ones(4))
    assert info == 2


def _small_case(nx=24, ny=12, nz=10):
    return cases.laminar_case(nx=nx, ny=ny, nz=nz, lx=12.0, ly=4.0, lz=3.0)


def test_poisson_variants_agree():
    """4N embedding + ZGTSV (projection.f90:210-288) and 2N twiddle +
    precomputed Thomas (projection.f90:93-204) give the same projection."""
    c = _small_case(nx=26, ny=14, nz=11)  # odd nz: prime nzp = 9? (9 = 3^2) and N = 24
    rng = np.random.default_rng(3)
    c.V = c.V + 1e-3 * rng.standard_normal(c.V.shape)
    c.W = c.W + 1e-3 * rng.standard_normal(c.W.shape)
    o0 = oracle.oracle_for(c, variant=0)
    o1 = oracle.oracle_for(c, variant=1)
    for o in (o0, o1):
        o.set_dt(0.05)
        o.apply_bc(1)
        o.projection(1)
        o.apply_bc(1)
    U0, V0, W0, P0, _ = o0.state()
    U1, V1, W1, P1, _ = o1.state()
    for a, b in ((U0, U1), (V0, V1), (W0, W1)):
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
    assert o0.max_divergence() < 1e-12 and o1.max_divergence() < 1e-12


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_step_is_divergence_free(rk):
    c = _small_case()
    c.rk_scheme = rk
    o = oracle.oracle_for(c)
    o.advance(3)
    assert o.max_divergence() < 1e-12
    U, V, W, P, t = o.state()
    assert np.isfinite(U).all() and t > 0


def test_compute_dt_uses_max_as_written():
    """compute_dt takes the MAX of spacing/|u| (time_integration.f90:550-558);
    with W == 0 somewhere the convective bound is +Inf and dt = dt_vis."""
    c = _small_case()
    o = oracle.oracle_for(c)
    dt = o.compute_dt()
    xg, yg, zg = cases.centres_ghost(c.x), cases.centres_ghost(c.y), cases.centres_ghost(c.z)
    dt_vis = min(c.cfl * np.diff(xg).min() ** 2, c.cfl * np.diff(yg).min() ** 2, c.cfl * np.diff(zg).min() ** 2) / c.nu
    assert dt == pytest.approx(dt_vis, rel=1e-15)


def test_lund_identity_when_inlet_is_station():
    """With the inlet plane equal to the recycling plane and delta_inlet set
    to the station's delta_99, gamma = 1 and every interpolation pair
    collapses to its own row: the rescaled plane is the station plane."""
    from blgpu import cases
    c = cases.turbulent_case(nx=40, ny=32, nz=16, seed=3)
    ir = 12
    for F in (c.U, c.V, c.W):
        F[0] = F[ir - 1]
    o = oracle.oracle_for(c)
    o.set_dt(0.01)
    o.set_rescaling(3, ir, 1.0, 10.0)
    o.rescaled_inflow()
    d = o.rescaling()["diag"]["delta_resc"]
    o.set_rescaling(3, ir, d, 10.0)
    o.rescaled_inflow()
    r = o.rescaling()
    assert r["diag"]["gamma"] == 1.0 and r["err"] == 0
    for F, L in ((c.U, r["U"]), (c.V, r["V"]), (c.W, r["W"])):
        assert np.abs(F[ir - 1][1:] - L[1:]).max() <= 1e-14 * np.abs(F).max()


def test_lund_gamma_follows_momentum_thickness():
    """gamma = (theta_resc/theta_inlet)^(1/8) (rescaled_inlet_bc.f90:230) and
    the running means move by dt/T_resc toward the instantaneous means."""
    from blgpu import cases
    c = cases.turbulent_case(nx=40, ny=32, nz=16, seed=4)
    o = oracle.oracle_for(c)
    o.set_dt(0.5)
    o.set_rescaling(3, 20, 1.0, 5.0)
    m0 = o.rescaling()["Umean_resc"].copy()
    o.rescaled_inflow()
    r = o.rescaling()
    d = r["diag"]
    assert abs(d["gamma"] - (d["theta_resc"] / d["theta_inlet"]) ** 0.125) < 1e-14
    inst = c.U[19, :, 1:-1].mean(axis=1)
    assert np.allclose(r["Umean_resc"], 0.1 * inst + 0.9 * m0, rtol=0, atol=1e-14)


def test_mlp_oracle_gradient_matches_finite_differences():
    """The oracle's back-propagation (plain FP64 mode) against central
    differences of its loss, and its BF16 mode within the BF16 rounding."""
    rng = np.random.default_rng(0)
    n = oracle.load().blo_mlp_nparams()
    assert n == 8770
    p = rng.standard_normal(n) * 0.2
    X = rng.standard_normal((40, 4)).astype(np.float32)
    T = rng.standard_normal((40, 2)).astype(np.float32)
    loss, g = oracle.mlp_gradient(p, X, T, exact=True)
    idx = rng.choice(n, 25, replace=False)
    h = 1e-6
    for q in idx:
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (oracle.mlp_gradient(pp, X, T, exact=True)[0] - oracle.mlp_gradient(pm, X, T, exact=True)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q]))
    lb, gb = oracle.mlp_gradient(p, X, T)
    assert abs(lb - loss) < 1e-2 * loss
    assert np.linalg.norm(gb - g) < 2e-2 * np.linalg.norm(g)


def test_wall_model_law_of_the_wall_on_log_profile():
    """On a mean profile that follows u+ = ln(y+)/kappa + B at the sampling
    row, the equilibrium wall model returns that profile's u_tau^2."""
    from blgpu import wallmodel
    c = wallmodel.wmles_case(nx=24, nz=8)
    o = oracle.oracle_for(c)
    o.set_wall_model(1, 3)
    tx, tz = o.wall_stress()
    assert abs(tx.mean() / c.utau ** 2 - 1) < 0.02
    assert np.all(tz == 0.0)


def _dyn_case(model, shift=0.0):
    """Noisy fields whose U, V planes in z are periodic and whose V, W
    columns in x follow the model's x helper (Neumann for 2, periodic for 3),
    so that the centre velocities agree with the ghosts of their products."""
    c = cases.laminar_case(nx=26, ny=14, nz=11, lx=20.0, ly=5.0, lz=3.0)
    rng = np.random.default_rng(41)
    U = c.U + 0.05 * rng.standard_normal(c.U.shape)
    V = c.V + 0.05 * rng.standard_normal(c.V.shape)
    W = c.W + 0.05 * rng.standard_normal(c.W.shape) + shift
    for a in (U, V):
        a[:, :, 0], a[:, :, -2], a[:, :, -1] = a[:, :, -3], a[:, :, 1], a[:, :, 2]
    for a in (V, W):
        if model == 2:
            a[0], a[-1] = a[1], a[-2]
        else:
            a[0], a[-2], a[-1] = a[-3], a[1], a[2]
    c.U, c.V, c.W = (np.asfortranarray(a) for a in (U, V, W))
    return c


def test_dynamic_smagorinsky_structure():
    """The oracle's dynamic model (subgrid.f90:261-583): nu_t >= 0 with
    Neumann y ghosts; LES = 2 keeps one coefficient per (i,j) column, so each
    column is all zero or all positive, and leaves the x / z ghosts at zero;
    LES = 3 has periodic x / z ghosts."""
    a = oracle.oracle_for(_dyn_case(2)).dynamic_smagorinsky(2)
    assert np.isfinite(a).all() and (a >= 0).all() and a.max() > 0
    assert np.array_equal(a[:, 0], a[:, 1]) and np.array_equal(a[:, -1], a[:, -2])
    assert not a[0].any() and not a[-1].any() and not a[:, :, 0].any() and not a[:, :, -1].any()
    col = a[1:-1, 1:-1, 1:-1] > 0
    assert np.all(col.all(axis=2) | ~col.any(axis=2)) and col.any() and not col.all()
    b = oracle.oracle_for(_dyn_case(3)).dynamic_smagorinsky(3)
    assert np.isfinite(b).all() and (b >= 0).all() and b.max() > 0
    assert np.array_equal(b[0], b[-3]) and np.array_equal(b[-2], b[1]) and np.array_equal(b[-1], b[2])
    assert np.array_equal(b[:, :, 0], b[:, :, -3]) and np.array_equal(b[:, :, -1], b[:, :, 2])
    assert np.array_equal(b[:, 0], b[:, 1])


@pytest.mark.parametrize("model", [2, 3])
def test_dynamic_smagorinsky_galilean_in_z(model):
    """A uniform shift of W changes neither the Leonard term (the filter
    weights sum to one) nor Mij (gradients only): nu_t moves by rounding."""
    a = oracle.oracle_for(_dyn_case(model)).dynamic_smagorinsky(model)
    b = oracle.oracle_for(_dyn_case(model, 0.3)).dynamic_smagorinsky(model)
    assert np.abs(a - b).max() <= 1e-8 * a.max()
