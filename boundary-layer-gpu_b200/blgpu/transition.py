"""Tollmien-Schlichting transition case: inflow modes from an Orr-Sommerfeld
solve of the Blasius profile, written in the reference's binary mode-file
format (read back through blgpu_read_temporal_modes, the inflow_flag = 1
branch of compute_blasius_solution_for_bc, boundary_conditions.f90:1652-1797),
and the growth rate of the forced wave.

Everything is in inflow displacement-thickness units (delta* = 1, U_inf = 1,
nu = 1/Re_delta*).  With the reference's Blasius convention f''' + f f'' = 0,
eta = y / sqrt(2 nu x), the profile in delta* units is U(y) = f'(c y) with
c = 1.7208 / sqrt(2) (delta* = 1.7208 sqrt(nu x)).

Orr-Sommerfeld (temporal, complex frequency omega at real alpha, k^2 =
alpha^2 + beta^2), Chebyshev collocation on y in [0, y_max] with clamped
walls:
    (alpha U - omega)(D^2 - k^2) v - alpha U'' v = (1/(i Re)) (D^2 - k^2)^2 v
The inflow shape of a mode of frequency omega is the eigenfunction at the
real alpha whose least stable eigenvalue has Re(omega) = omega (secant in
alpha); u and w follow from continuity with the wall-normal vorticity left
out: u = i alpha Dv / k^2, w = i beta Dv / k^2.
"""
import struct

import numpy as np

C_DSTAR = 1.7208 / np.sqrt(2.0)


def blasius_fine(eta_max=20.0, n=20000):
    """(eta, f, f', f'') of f''' + f f'' = 0 on a fine equispaced grid (RK4,
    f''(0) by secant shooting)."""
    h = eta_max / n

    def run(a, keep=False):
        y = np.array([0.0, 0.0, a])
        out = [y.copy()] if keep else None
        rhs = lambda s: np.array([s[1], s[2], -s[0] * s[2]])
        for _ in range(n):
            k1 = rhs(y)
            k2 = rhs(y + 0.5 * h * k1)
            k3 = rhs(y + 0.5 * h * k2)
            k4 = rhs(y + h * k3)
            y = y + h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
            if keep:
                out.append(y.copy())
        return np.array(out) if keep else y

    a0, a1 = 0.45, 0.48
    m0, m1 = run(a0)[1] - 1.0, run(a1)[1] - 1.0
    for _ in range(40):
        a2 = a1 - m1 * (a1 - a0) / (m1 - m0)
        a0, m0, a1 = a1, m1, a2
        m1 = run(a1)[1] - 1.0
        if abs(m1) < 1e-13:
            break
    sol = run(a1, keep=True)
    return np.linspace(0.0, eta_max, n + 1), sol[:, 0], sol[:, 1], sol[:, 2]


def cheb(n):
    """Chebyshev points x_j = cos(pi j / n) and the differentiation matrix."""
    x = np.cos(np.pi * np.arange(n + 1) / n)
    c = np.ones(n + 1)
    c[0] = c[-1] = 2.0
    c *= (-1.0) ** np.arange(n + 1)
    X = np.tile(x, (n + 1, 1)).T
    dX = X - X.T
    D = np.outer(c, 1.0 / c) / (dX + np.eye(n + 1))
    D -= np.diag(D.sum(axis=1))
    return x, D


class OrrSommerfeld:
    """Collocation operators of a parallel profile on y in [0, y_max]: the
    Blasius profile by default, or profile = (U(y), U''(y)) callables."""

    def __init__(self, re, n=120, y_max=20.0, profile=None):
        self.re = re
        xi, D = cheb(n)
        self.y = (xi + 1.0) * 0.5 * y_max       # y_max at j = 0, the wall at j = n
        D1 = D * (2.0 / y_max)
        self.D1, self.D2 = D1, D1 @ D1
        if profile is None:
            eta, f, fp, fpp = blasius_fine()
            e = C_DSTAR * self.y
            self.U = np.interp(e, eta, fp)
            self.Upp = -np.interp(e, eta, f) * np.interp(e, eta, fpp) * C_DSTAR ** 2
        else:
            self.U, self.Upp = profile[0](self.y), profile[1](self.y)
        self.n = n

    def modes(self, alpha, beta):
        """eigenvalues omega and eigenvectors v (columns) at real alpha"""
        import scipy.linalg
        k2 = alpha * alpha + beta * beta
        I = np.eye(self.n + 1)
        L = self.D2 - k2 * I
        A = alpha * np.diag(self.U) @ L - alpha * np.diag(self.Upp) - (L @ L) / (1j * self.re)
        B = L.astype(complex)
        # clamped walls: v = Dv = 0 at y = 0 (row n) and y = y_max (row 0)
        for r, row in ((0, I[0]), (1, self.D1[0]), (self.n, I[self.n]), (self.n - 1, self.D1[self.n])):
            A[r] = row
            B[r] = 0.0
        w, V = scipy.linalg.eig(A, B)
        # the four boundary rows leave infinite eigenvalues, which rounding
        # turns into huge finite ones: keep phase speeds of order one
        ok = np.isfinite(w) & (np.abs(w) < 1e3 * max(alpha, 1e-3))
        return w[ok], V[:, ok]

    def ts_mode(self, alpha, beta):
        """the least stable mode with a phase speed between 0 and 1"""
        w, V = self.modes(alpha, beta)
        c = w / alpha
        sel = np.where((c.real > 0.05) & (c.real < 0.95))[0]
        i = sel[np.argmax(w[sel].imag)]
        return w[i], V[:, i]

    def alpha_for(self, omega, beta, a0=0.25, a1=0.3):
        """real alpha whose TS eigenvalue has Re(omega) = omega (secant)"""
        f = lambda a: self.ts_mode(a, beta)[0].real - omega
        f0, f1 = f(a0), f(a1)
        for _ in range(30):
            a2 = a1 - f1 * (a1 - a0) / (f1 - f0)
            a0, f0, a1 = a1, f1, a2
            f1 = f(a1)
            if abs(f1) < 1e-10:
                break
        return a1

    def velocity(self, alpha, beta, v, y):
        """(u, v, w) of an eigenfunction on the points y (barycentric interpolation)"""
        from scipy.interpolate import BarycentricInterpolator
        k2 = alpha * alpha + beta * beta
        dv = self.D1 @ v
        u = 1j * alpha * dv / k2
        w = 1j * beta * dv / k2
        out = []
        for q in (u, v, w):
            re = BarycentricInterpolator(self.y, q.real)(y)
            im = BarycentricInterpolator(self.y, q.imag)(y)
            out.append(np.where(y <= self.y.max(), re + 1j * im, 0.0))
        return out


def write_mode_file(path, ymesh, zmode, tmode, beta, omega, qu, qv, qw):
    """The reference's binary mode file (native-order stream): ny_inlet, n, m
    (int32), beta, omega (f64), ymesh, zmode, tmode, then the real and
    imaginary parts of qu, qv, qw (ny_inlet, n, m) in Fortran order."""
    ny, n, m = qu.shape
    with open(path, "wb") as f:
        f.write(struct.pack("=3i", ny, n, m))
        f.write(struct.pack("=2d", beta, omega))
        for a in (ymesh, zmode, tmode):
            f.write(np.asarray(a, dtype=np.float64).tobytes())
        for q in (qu, qv, qw):
            f.write(np.asfortranarray(q.real).ravel(order="F").astype(np.float64).tobytes())
            f.write(np.asfortranarray(q.imag).ravel(order="F").astype(np.float64).tobytes())


def ts_mode_file(path, re=1000.0, omega=0.1, beta=0.2, amp2d=1e-3, amp3d=1e-4, seed=7, ly=20.0, ny_inlet=200,
                 n_cheb=120):
    """Mode file of a 2-D TS wave at omega (max |u| = amp2d) plus an oblique
    pair at +-beta (max |u| = amp3d each, seeded random phases).  Returns a
    dict with the chosen alphas and the temporal growth rates omega_i."""
    os_ = OrrSommerfeld(re, n=n_cheb, y_max=ly)
    ym = np.linspace(0.0, ly, ny_inlet)
    rng = np.random.default_rng(seed)
    zmode = np.array([0.0, 1.0, -1.0])
    tmode = np.array([1.0])
    qu = np.zeros((ny_inlet, 3, 1), complex)
    qv, qw = qu.copy(), qu.copy()
    info = {}
    for nidx, (bb, amp, phase) in enumerate(((0.0, amp2d, 0.0), (beta, amp3d, rng.uniform(0, 2 * np.pi)),
                                             (-beta, amp3d, rng.uniform(0, 2 * np.pi)))):
        a = os_.alpha_for(omega, abs(bb))
        w, v = os_.ts_mode(a, abs(bb))
        u_, v_, w_ = os_.velocity(a, bb, v, ym)
        s = amp * np.exp(1j * phase) / np.abs(u_).max()
        qu[:, nidx, 0], qv[:, nidx, 0], qw[:, nidx, 0] = s * u_, s * v_, s * w_
        info["beta=%+.2f" % bb] = {"alpha": float(a), "omega_i": float(w.imag)}
    write_mode_file(path, ym, zmode, tmode, beta, omega, qu, qv, qw)
    return info


def transition_case(nx=1024, ny=129, nz=128, lx=400.0, ly=20.0, lz=40.0, alpha=1.5, re_dstar=1000.0, cfl=0.4):
    """Blasius plate in delta* units at Re_delta* = re_dstar (inflow delta* = 1),
    laminar initial field; the TS forcing comes from a mode file."""
    from .cases import laminar_case
    c = laminar_case(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, lz=lz, alpha=alpha, re_dstar=re_dstar, cfl=cfl)
    c.name = "transition"
    return c


def growth_rate(x, amp, x0, x1):
    """slope of log(amp) over x in [x0, x1] (least squares): the spatial
    growth rate -alpha_i of the wave"""
    sel = (x >= x0) & (x <= x1) & (amp > 0)
    p = np.polyfit(x[sel], np.log(amp[sel]), 1)
    return float(p[0])


def run_growth(case, modes, precision, steps, period_steps=400, omega=0.1, device=0, x_fit=(20.0, 80.0)):
    """Force the case with the file's modes for `steps` steps at the fixed dt
    of period_steps per forcing period (graph-replayed steps), and again
    without forcing (the base).  The wave envelope at x is max over y of
    sqrt(<u'^2>_z(t) + <u'^2>_z(t + T/4)), u' = forced - base, from snapshots
    a quarter period apart; the spatial growth rate is the slope of its log
    over x - x(1) in x_fit.  Returns (growth rate, envelope, x)."""
    import copy
    from .cases import solver_for
    dt = 2.0 * np.pi / omega / period_steps
    c = copy.copy(case)
    c.cfl = -dt  # fixed dt (time_integration.f90:539)
    q = period_steps // 4
    snaps = {}
    for forced in (True, False):
        s = solver_for(c, precision=precision, device=device)
        if forced:
            s.set_inflow_modes(modes["zmode"], modes["tmode"], modes["qu"], modes["qv"], modes["qw"])
        out = []
        for n in (steps, q):
            s.advance(n)
            out.append(s.download_state()[0])
        snaps[forced] = out
        s.close()
    d0 = snaps[True][0] - snaps[False][0]
    d1 = snaps[True][1] - snaps[False][1]
    e2 = (d0[:, 1:-1, 1:-2] ** 2).mean(axis=2) + (d1[:, 1:-1, 1:-2] ** 2).mean(axis=2)
    env = np.sqrt(e2.max(axis=1))
    xr = case.x - case.x[0]
    return growth_rate(xr, env, *x_fit), env, xr
