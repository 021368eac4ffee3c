"""Run set-up on the host: grids, Blasius tables, inflow/top vectors and the
synthetic initial fields of the benchmark configurations.

Restates the set-up half of the reference that feeds the step path:
  - grids and their centre/ghost extensions (input_output.f90:150-190,
    initialization.f90:174-222);
  - the Blasius similarity table in the reference's (eta, f, f') convention
    (laminar_test/generate_blasius.py: f''' + f f'' = 0, eta = y sqrt(U/(2 nu x)));
  - the inlet, top and outlet vectors of compute_blasius_solution_for_bc
    (boundary_conditions.f90:1452-1765) and of
    compute_turbulent_solution_for_bc (boundary_conditions.f90:1371-1425);
  - the Blasius initial condition of init_flow (input_output.f90:196-256).
All arrays follow the reference's Fortran layout and bounds.
"""
import math

import numpy as np


# ---------------------------------------------------------------------------
# grids
# ---------------------------------------------------------------------------
def uniform_faces(n, length, x0=0.0):
    """n faces from x0 to x0+length (init_flow x mesh, input_output.f90:152-157)."""
    return x0 + np.arange(n, dtype=np.float64) / (n - 1) * length


def periodic_faces(nz, length):
    """z faces of the periodic direction: z(k) = (k-1) Lz/(nz-2), so the
    nz-2 distinct centres k=2..nz-1 span one period (input_output.f90:159-163)."""
    return np.arange(nz, dtype=np.float64) / (nz - 2) * length


def tanh_faces(n, length, alpha):
    """wall-clustered faces y = L (1 - tanh(alpha (1-eta)) / tanh(alpha))."""
    eta = np.arange(n, dtype=np.float64) / (n - 1)
    y = length * (1.0 - np.tanh(alpha * (1.0 - eta)) / np.tanh(alpha))
    y[0] = 0.0
    return y


def sinh_faces(n, length, alpha):
    """the reference's own y mesh (input_output.f90:165-174)."""
    y = np.arange(n, dtype=np.float64)
    y = y / y.max()
    y = np.sinh(alpha * y) / np.sinh(alpha)
    y = y - y[0]
    return y / y.max() * length


def centres_ghost(f):
    """xg(1..n+1) from faces f(1..n) (initialization.f90:186-199)."""
    n = f.size
    m = 0.5 * (f[:-1] + f[1:])
    g = np.empty(n + 1)
    g[1:n] = m
    g[0] = m[0] - 2.0 * (m[0] - f[0])
    g[n] = m[-1] + 2.0 * (f[-1] - m[-1])
    return g


# ---------------------------------------------------------------------------
# Blasius similarity solution
# ---------------------------------------------------------------------------
def _blasius_integrate(fpp0, eta_max, nsteps, keep_every=0):
    """classical RK4 for (f, f', f'')' = (f', f'', -f f'')"""
    h = eta_max / nsteps
    f, g, q = 0.0, 0.0, fpp0
    rows = [(f, g)] if keep_every else None
    for i in range(nsteps):
        k1f, k1g, k1q = g, q, -f * q
        f2, g2, q2 = f + 0.5 * h * k1f, g + 0.5 * h * k1g, q + 0.5 * h * k1q
        k2f, k2g, k2q = g2, q2, -f2 * q2
        f3, g3, q3 = f + 0.5 * h * k2f, g + 0.5 * h * k2g, q + 0.5 * h * k2q
        k3f, k3g, k3q = g3, q3, -f3 * q3
        f4, g4, q4 = f + h * k3f, g + h * k3g, q + h * k3q
        k4f, k4g, k4q = g4, q4, -f4 * q4
        f += h / 6.0 * (k1f + 2 * k2f + 2 * k3f + k4f)
        g += h / 6.0 * (k1g + 2 * k2g + 2 * k3g + k4g)
        q += h / 6.0 * (k1q + 2 * k2q + 2 * k3q + k4q)
        if keep_every and (i + 1) % keep_every == 0:
            rows.append((f, g))
    return (f, g) if not keep_every else np.array(rows)


def blasius_table(n_points=1000, eta_max=20.0, substeps=20):
    """(eta, f, f') on n_points equispaced eta in [0, eta_max] for
    f''' + f f'' = 0, f(0)=f'(0)=0, f'(inf)=1; f''(0) by secant shooting."""
    nsteps = (n_points - 1) * substeps

    def miss(a):
        return _blasius_integrate(a, eta_max, nsteps)[1] - 1.0

    a0, a1 = 0.4, 0.5
    m0, m1 = miss(a0), miss(a1)
    for _ in range(50):
        a2 = a1 - m1 * (a1 - a0) / (m1 - m0)
        a0, m0 = a1, m1
        a1, m1 = a2, miss(a2)
        if abs(m1) < 1e-14 or a1 == a0:
            break
    sol = _blasius_integrate(a1, eta_max, nsteps, keep_every=substeps)
    eta = np.linspace(0.0, eta_max, n_points)
    return eta, sol[:, 0].copy(), sol[:, 1].copy(), a1


def write_blasius_file(path, eta, f, df):
    """text file in the reference format (n, eta row, f row, f' row)."""
    with open(path, "w") as fo:
        fo.write("%d\n" % len(eta))
        for row in (eta, f, df):
            fo.write(" ".join("%.15e" % v for v in row) + "\n")


def read_blasius_file(path):
    with open(path) as fi:
        toks = fi.read().split()
    n = int(toks[0])
    v = np.array([float(t) for t in toks[1:1 + 3 * n]])
    return v[:n], v[n:2 * n], v[2 * n:3 * n]


def _interp_eta(eta_src, eta):
    """the reference's bracket search: first k>=2 with eta_src(k) > eta;
    returns (j0, w0, w1) with 0-based j0, or None past the table."""
    k = int(np.searchsorted(eta_src[1:], eta, side="right")) + 1
    if k >= eta_src.size:
        return None
    j0 = k - 1
    w1 = (eta - eta_src[j0]) / (eta_src[k] - eta_src[j0])
    return j0, 1.0 - w1, w1


def blasius_boundary(x, y, nu, table, u_inf=1.0):
    """U_inlet(nyg), V_inlet(ny), W_inlet(nyg), U_top(nx), V_top(nxg), W_top(nxg)
    as compute_blasius_solution_for_bc with inflow_flag=1
    (boundary_conditions.f90:1485-1765)."""
    eta_s, f_s, df_s = table
    xg, yg = centres_ghost(x), centres_ghost(y)
    nyg, ny, nxg = yg.size, y.size, xg.size
    U_in = np.ones(nyg)
    for j in range(nyg):
        eta = yg[j] * (u_inf / (2.0 * nu * x[0])) ** 0.5
        r = _interp_eta(eta_s, eta)
        U_in[j] = 1.0 if r is None else r[1] * df_s[r[0]] + r[2] * df_s[r[0] + 1]
    V_in = np.zeros(ny)
    rex = 1.0 * xg[0] / nu
    for j in range(ny):
        eta = y[j] * (u_inf / (2.0 * nu * xg[0])) ** 0.5
        r = _interp_eta(eta_s, eta)
        if r is None:
            V_in[j] = V_in.max()
        else:
            j0, w0, w1 = r
            c = 1.0 / (2.0 * rex) ** 0.5
            V_in[j] = w0 * c * (eta_s[j0] * df_s[j0] - f_s[j0]) + w1 * c * (eta_s[j0 + 1] * df_s[j0 + 1] - f_s[j0 + 1])
    W_in = np.zeros(nyg)
    U_top = np.ones(x.size)
    V_top = np.empty(nxg)
    n = eta_s.size - 1
    for i in range(nxg):
        rex_i = 1.0 * xg[i] / nu
        V_top[i] = 1.0 / (2.0 * rex_i) ** 0.5 * (eta_s[n] * df_s[n] - f_s[n])
    W_top = np.zeros(nxg)
    return U_in, V_in, W_in, U_top, V_top, W_top


def blasius_initial(x, y, z, nu, table, u_inf=1.0):
    """U, V, W of init_flow (input_output.f90:196-256) on the given mesh."""
    eta_s, f_s, df_s = table
    xg, yg = centres_ghost(x), centres_ghost(y)
    nx, ny, nz = x.size, y.size, z.size
    nxg, nyg, nzg = nx + 1, ny + 1, nz + 1
    U = np.full((nx, nyg, nzg), u_inf, order="F")
    for ii in range(nx):
        for jj in range(nyg):
            eta = yg[jj] * math.sqrt(u_inf / (2.0 * nu * x[ii]))
            r = _interp_eta(eta_s, eta)
            U[ii, jj, :] = u_inf if r is None else u_inf * (r[1] * df_s[r[0]] + r[2] * df_s[r[0] + 1])
    V = np.zeros((nxg, ny, nzg), order="F")
    n = eta_s.size - 1
    for ii in range(nxg):
        rex = u_inf * xg[ii] / nu
        c = u_inf / math.sqrt(2.0 * rex)
        for jj in range(ny):
            eta = y[jj] * math.sqrt(u_inf / (2.0 * nu * xg[ii]))
            r = _interp_eta(eta_s, eta)
            if r is None:
                V[ii, jj, :] = c * (eta_s[n] * df_s[n] - f_s[n])
            else:
                j0, w0, w1 = r
                V[ii, jj, :] = c * (w0 * (eta_s[j0] * df_s[j0] - f_s[j0]) + w1 * (eta_s[j0 + 1] * df_s[j0 + 1] - f_s[j0 + 1]))
    W = np.zeros((nxg, nyg, nz), order="F")
    return U, V, W


def turbulent_top(x, nu, u_inf=1.0):
    """U_top, V_top, W_top of compute_turbulent_solution_for_bc
    (boundary_conditions.f90:1388-1397): V_top = U 0.0160 Re_x^(-1/7)."""
    xg = centres_ghost(x)
    U_top = np.full(x.size, u_inf)
    V_top = u_inf * 0.0160 * (u_inf * xg / nu) ** (-1.0 / 7.0)
    W_top = np.zeros(xg.size)
    return U_top, V_top, W_top


# ---------------------------------------------------------------------------
# turbulent mean profile (composite law of the wall + Coles wake)
# ---------------------------------------------------------------------------
# the reference's equilibrium wall-model constants (wallmodel.f90:1960-1961)
KAPPA_WM, B_WM = 0.38, 5.2


def reichardt_c(kappa, B):
    """Reichardt's constant for which his law tends to ln(y+)/kappa + B."""
    return B - math.log(kappa) / kappa


def composite_profile(y, delta, utau, nu, kappa=0.41, C=7.8, Pi=0.45, u_inf=1.0):
    """Reichardt's inner law (constant C) blended with Coles' wake, clipped at
    U_inf above delta."""
    yp = np.maximum(y, 0.0) * utau / nu
    up = (1.0 / kappa) * np.log1p(kappa * yp) + C * (1.0 - np.exp(-yp / 11.0) - (yp / 11.0) * np.exp(-yp / 3.0))
    eta = np.clip(y / delta, 0.0, 1.0)
    wake = 2.0 * Pi / kappa * np.sin(0.5 * np.pi * eta) ** 2
    u = utau * (up + wake)
    u = np.where(y >= delta, u_inf, np.minimum(u, u_inf))
    return np.where(y < 0, -u, u)


def turbulent_inflow_profile(retheta, delta=1.0, u_inf=1.0, n_fit=4000, kappa=0.41, C=7.8):
    """nu and utau for which the composite profile of thickness delta has
    momentum thickness Re_theta (Coles-Fernholz skin friction)."""
    # Coles-Fernholz: cf = 2 (1/0.384 ln Re_theta + 4.127)^-2
    cf = 2.0 * (1.0 / 0.384 * math.log(retheta) + 4.127) ** -2
    utau = u_inf * math.sqrt(cf / 2.0)
    yy = np.linspace(0.0, delta, n_fit)
    nu = 1e-4
    for _ in range(60):
        u = composite_profile(yy, delta, utau, nu, kappa=kappa, C=C, u_inf=u_inf) / u_inf
        theta = np.trapezoid(u * (1.0 - u), yy)
        nu_new = theta * u_inf / retheta
        if abs(nu_new - nu) < 1e-14:
            break
        nu = nu_new
    return nu, utau, theta


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------
class Case:
    """A complete input set for one box (what .turbb + snapshot provide)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def cells(self):
        return self.nx * self.ny * self.nz


def laminar_case(nx=128, ny=64, nz=32, lx=60.0, ly=6.0, lz=6.0, alpha=1.5, re_dstar=500.0, cfl=0.5,
                 rk_scheme=3, table=None):
    """Laminar flat-plate boundary layer in delta* units (inflow delta* = 1):
    nu = 1/Re_delta*, x0 with delta*(x0) = 1.7208 sqrt(nu x0) = 1."""
    nu = 1.0 / re_dstar
    x0 = (1.0 / 1.7208) ** 2 / nu
    x = uniform_faces(nx, lx, x0)
    y = tanh_faces(ny, ly, alpha)
    z = periodic_faces(nz, lz)
    if table is None:
        eta, f, df, _ = blasius_table()
        table = (eta, f, df)
    bc = blasius_boundary(x, y, nu, table)
    U, V, W = blasius_initial(x, y, z, nu, table)
    return Case(name="laminar", nx=nx, ny=ny, nz=nz, x=x, y=y, z=z, nu=nu, cfl=cfl, rk_scheme=rk_scheme,
                dpdx=0.0, dpdz=0.0, bc=bc, U=U, V=V, W=W, t=0.0, table=table)


def _smooth_noise(shape, seed, sigma_pts):
    """Gaussian-filtered white noise (FFT filter), unit rms."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    A = np.fft.rfftn(a)
    ks = [np.fft.fftfreq(n) for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1])]
    g = np.ones(A.shape)
    for d, k in enumerate(ks):
        sh = [1] * len(shape)
        sh[d] = k.size
        g = g * np.exp(-0.5 * (2 * np.pi * k * sigma_pts[d]) ** 2).reshape(sh)
    a = np.fft.irfftn(A * g, s=shape, axes=tuple(range(len(shape))))
    return a / a.std()


def turbulent_case(nx=814, ny=257, nz=193, lx=100.0, ly=4.0, lz=8.0, alpha=2.0, retheta=1100.0, cfl=0.5,
                   rk_scheme=3, seed=1234, noise=0.10, coarse=4, lund=3, T_resc=10.0, kappa=0.41, C=7.8):
    """Turbulent boundary layer in inflow delta99 units: composite mean profile
    plus divergence-free noise (curl of a Gaussian-filtered random vector
    potential, `noise` U_inf rms) confined below y = 1.5 delta.  The noise is
    built on a grid `coarse` times coarser and interpolated; the first
    projection of the solver makes the field discretely divergence free.
    Inflow: Lund recycling (inflow_flag `lund`, 0 for the fixed profile) from
    the station i = nx/10 (about 10 inflow delta99 downstream at the default
    length), delta_inlet = 1, averaging time T_resc."""
    nu, utau, theta = turbulent_inflow_profile(retheta, kappa=kappa, C=C)
    rex_theta = (retheta / 0.036) ** 1.25  # theta/x = 0.036 Re_x^-1/5
    x0 = rex_theta * nu
    x = uniform_faces(nx, lx, x0)
    y = tanh_faces(ny, ly, alpha)
    z = periodic_faces(nz, lz)
    xg, yg, zg = centres_ghost(x), centres_ghost(y), centres_ghost(z)
    prof_c = composite_profile(yg, 1.0, utau, nu, kappa=kappa, C=C)  # U at y centres (nyg)
    U_in = prof_c.copy()
    V_in = np.zeros(ny)
    W_in = np.zeros(ny + 1)
    U_top, V_top, W_top = turbulent_top(x, nu)
    # vector potential on a coarse uniform index grid
    cshape = (max(8, nx // coarse), max(8, (ny + 1) // coarse), max(8, nz // coarse))
    psi = [_smooth_noise(cshape, seed + c, (1.5, 1.5, 1.5)) for c in range(3)]
    # curl on the coarse index grid (unit spacing), then scale
    gx = [np.gradient(p, axis=0) for p in psi]
    gy = [np.gradient(p, axis=1) for p in psi]
    gz = [np.gradient(p, axis=2) for p in psi]
    u_c = gy[2] - gz[1]
    v_c = gz[0] - gx[2]
    w_c = gx[1] - gy[0]

    def resample(a, shape):
        from scipy.ndimage import zoom
        f = [s / c for s, c in zip(shape, a.shape)]
        r = zoom(a, f, order=1)
        out = np.zeros(shape)
        sl = tuple(slice(0, min(s, rs)) for s, rs in zip(shape, r.shape))
        out[sl] = r[sl]
        return out

    rms = np.sqrt((u_c ** 2 + v_c ** 2 + w_c ** 2).mean() / 3.0)
    mask_c = np.clip((1.5 - yg) / 0.3, 0.0, 1.0)  # smooth cut-off above 1.5 delta
    mask_f = np.clip((1.5 - y) / 0.3, 0.0, 1.0)
    wall_c = np.tanh(yg / 0.05)
    amp = noise / rms
    U = np.asfortranarray(resample(u_c, (nx, ny + 1, nz + 1)) * amp * (mask_c * wall_c)[None, :, None]
                          + prof_c[None, :, None])
    V = np.asfortranarray(resample(v_c, (nx + 1, ny, nz + 1)) * amp * (mask_f * np.tanh(y / 0.05))[None, :, None])
    W = np.asfortranarray(resample(w_c, (nx + 1, ny + 1, nz)) * amp * (mask_c * wall_c)[None, :, None])
    return Case(name="turbulent", nx=nx, ny=ny, nz=nz, x=x, y=y, z=z, nu=nu, cfl=cfl, rk_scheme=rk_scheme,
                dpdx=0.0, dpdz=0.0, bc=(U_in, V_in, W_in, U_top, V_top, W_top), U=U, V=V, W=W, t=0.0,
                utau=utau, theta=theta, retheta=retheta,
                lund=(lund, max(2, nx // 10), 1.0, T_resc) if lund else None)


def ensemble_cases(nbox=64, seed=2024, nx_set=(128, 192, 256), ny=65, nz_set=(64, 96),
                   retheta=(800.0, 1500.0), cfl=0.5):
    """Boxes of the batched training-data ensemble: nx drawn uniformly from
    nx_set, nz from nz_set, Re_theta uniform in `retheta`, each built with
    the turbulent recipe (seeded noise, Lund inflow) at the streamwise and
    spanwise resolution of the 814x257x193 box (dx = 100/814, dz = 8/193 in
    inflow delta99 units) and ly = 4."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(nbox):
        nx = int(rng.choice(nx_set))
        nz = int(rng.choice(nz_set))
        rt = float(rng.uniform(*retheta))
        out.append(turbulent_case(nx=nx, ny=ny, nz=nz, lx=nx * 100.0 / 814.0, ly=4.0, lz=nz * 8.0 / 193.0,
                                  retheta=rt, cfl=cfl, seed=seed + 7919 * (b + 1)))
    return out


def solver_for(case, precision=0, device=0, les_model=0, inflow=True, poisson=0):
    """Create a Solver loaded with a case (grid, boundary vectors, state and,
    unless inflow=False, the case's Lund recycling inflow).  poisson = 1
    selects the cuFFT comparison path of the Poisson solve."""
    from .solver import Solver
    s = Solver(case.nx, case.ny, case.nz, case.nu, case.cfl, case.dpdx, case.dpdz, case.rk_scheme,
               les_model=les_model, precision=precision, device=device, poisson=poisson)
    s.set_grid(case.x, case.y, case.z)
    s.set_boundary(*case.bc)
    s.upload_state(case.U, case.V, case.W, case.t)
    if case.cfl < 0:
        s.set_dt(-case.cfl)
    if inflow and getattr(case, "lund", None):
        s.set_rescaling(*case.lund)
    return s



def project_initial(case, device=0):
    """Make the initial field discretely divergence free: one boundary pass,
    projection and boundary pass of the FP64 path (the config-2 recipe's
    "one projection" of the noisy initial field).  Updates case.U/V/W."""
    from ._lib import FP64
    s = solver_for(case, precision=FP64, device=device, inflow=False)
    s.set_dt(abs(case.cfl) if case.cfl < 0 else 1.0)
    s.apply_boundary_conditions(3)
    s.compute_projection_step(3)
    s.apply_boundary_conditions(3)
    case.U, case.V, case.W = s.download_state()[:3]
    s.close()
    return case
