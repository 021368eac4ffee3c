"""CPU parity oracle -- TEST INFRASTRUCTURE ONLY.

A plain-C FP64 restatement (bl_oracle.c) of the step path of the reference
CPU build of ms-alvaro/boundary-layer-gpu, loaded through ctypes.  Only the
tests, __graft_entry__.smoke() and bench.py's CPU-baseline/reference legs may
use it, and only as the checker or the timed CPU reference -- never as the
product path.

Parity status: the oracle is pinned component by component -- its FFT against
numpy.fft, its DCT against scipy.fft.dct, its ZGTSV restatement against
scipy's LAPACK zgtsv, its two Poisson variants (4N embedding + ZGTSV vs 2N
twiddle + precomputed Thomas) against each other, the host Blasius set-up
against the reference's shipped blasius_solution.dat (tests/golden).  The
reference solver itself cannot be built here (no Fortran compiler, MPI or
FFTW; Makefile.cpu also omits cufft_solver.o), and the reference ships no
solver outputs, so the full step is pinned by those components and by
physics checks (discrete divergence, Blasius skin friction), not by a
reference run.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "bl_oracle.c")
SRCS = [SRC, os.path.join(HERE, "mlp_oracle.c")]
LIB = os.path.join(HERE, "liboracle.so")
_dp = ctypes.POINTER(ctypes.c_double)


def build(force=False):
    """gcc -O2 -ffp-contract=off -fopenmp; output oracle/liboracle.so."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(
            [os.path.getmtime(p) for p in SRCS] + [os.path.getmtime(os.path.join(HERE, "bl_oracle.h"))]):
        return LIB
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-std=gnu99",
           "-o", LIB + ".tmp"] + SRCS + ["-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB)
        lib.blo_create.restype = ctypes.c_void_p
        lib.blo_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [ctypes.c_int, ctypes.c_int]
        lib.blo_destroy.argtypes = [ctypes.c_void_p]
        lib.blo_set_threads.argtypes = [ctypes.c_int]
        lib.blo_set_grid.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        lib.blo_set_bc.argtypes = [ctypes.c_void_p] + [_dp] * 6
        lib.blo_set_modes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [_dp] * 5
        lib.blo_set_state.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_double]
        lib.blo_get_state.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        lib.blo_set_nu_t.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int]
        lib.blo_compute_dt.restype = ctypes.c_double
        lib.blo_compute_dt.argtypes = [ctypes.c_void_p]
        lib.blo_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.blo_get_dt.restype = ctypes.c_double
        lib.blo_get_dt.argtypes = [ctypes.c_void_p]
        lib.blo_step.argtypes = [ctypes.c_void_p]
        lib.blo_rk3_stage.argtypes = [ctypes.c_void_p, ctypes.c_int]
        for n in ("blo_rhs_u", "blo_rhs_v", "blo_rhs_w"):
            getattr(lib, n).argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
        lib.blo_apply_bc.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.blo_projection.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.blo_max_divergence.restype = ctypes.c_double
        lib.blo_max_divergence.argtypes = [ctypes.c_void_p]
        lib.blo_get_rhs_p.argtypes = [ctypes.c_void_p, _dp]
        lib.blo_fft.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        lib.blo_zgtsv.restype = ctypes.c_int
        lib.blo_zgtsv.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
        lib.blo_dct2.argtypes = [ctypes.c_int, _dp, _dp]
        lib.blo_smagorinsky.argtypes = [ctypes.c_void_p]
        lib.blo_dynamic_smagorinsky.argtypes = [ctypes.c_void_p]
        lib.blo_set_les.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.blo_get_nu_t.argtypes = [ctypes.c_void_p, _dp]
        lib.blo_statistics.argtypes = [ctypes.c_void_p] + [_dp] * 5
        lib.blo_law_of_wall.restype = ctypes.c_int
        lib.blo_law_of_wall.argtypes = [ctypes.c_void_p, _dp]
        lib.blo_set_rescaling.restype = ctypes.c_int
        lib.blo_set_rescaling.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, _dp, _dp]
        lib.blo_rescaled_inflow.argtypes = [ctypes.c_void_p]
        lib.blo_get_rescaling.argtypes = [ctypes.c_void_p] + [_dp] * 8 + [ctypes.POINTER(ctypes.c_int)]
        _fp = ctypes.POINTER(ctypes.c_float)
        lib.blo_mlp_nparams.restype = ctypes.c_int
        lib.blo_mlp_forward.argtypes = [_dp, _fp, ctypes.c_int, _fp, ctypes.c_int]
        lib.blo_mlp_gradient.restype = ctypes.c_double
        lib.blo_mlp_gradient.argtypes = [_dp, _fp, _fp, ctypes.c_int, _dp, ctypes.c_int]
        lib.blo_set_wall_model.restype = ctypes.c_int
        lib.blo_set_wall_model.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        lib.blo_wall_stress.argtypes = [ctypes.c_void_p, _dp, _dp]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def fft(x, inverse=False):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).copy()
    load().blo_fft(a.size, _p(a.view(np.float64)), int(inverse))
    return a


def dct2(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    c = np.zeros_like(f)
    load().blo_dct2(f.size, _p(f), _p(c))
    return c


def zgtsv(dl, d, du, b):
    a = [np.ascontiguousarray(np.asarray(v, dtype=np.complex128)).copy() for v in (dl, d, du, b)]
    info = load().blo_zgtsv(a[1].size, *[_p(v.view(np.float64)) for v in a])
    return a[3], info


class Oracle:
    def __init__(self, nx, ny, nz, nu, cfl, dpdx=0.0, dpdz=0.0, rk_scheme=3, variant=0, threads=1):
        self.lib = load()
        self.lib.blo_set_threads(int(threads))
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nxg, self.nyg, self.nzg = nx + 1, ny + 1, nz + 1
        self.h = self.lib.blo_create(nx, ny, nz, nu, cfl, dpdx, dpdz, rk_scheme, variant)
        if not self.h:
            raise ValueError("oracle: bad sizes")

    def close(self):
        if self.h:
            self.lib.blo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_grid(self, x, y, z):
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        self.lib.blo_set_grid(self.h, _p(x), _p(y), _p(z))

    def set_bc(self, *vecs):
        self._bc = [np.ascontiguousarray(v, dtype=np.float64) for v in vecs]
        self.lib.blo_set_bc(self.h, *[_p(v) for v in self._bc])

    def set_modes(self, zmode, tmode, qu, qv, qw):
        zmode = np.ascontiguousarray(zmode, dtype=np.float64)
        tmode = np.ascontiguousarray(tmode, dtype=np.float64)
        n, m = zmode.size, tmode.size
        qs = []
        for q, ny_ in ((qu, self.nyg), (qv, self.ny), (qw, self.nyg)):
            q = np.asarray(q, dtype=np.complex128).reshape(ny_, n, m, order="F")
            qs.append(np.ascontiguousarray(q.ravel(order="F")).view(np.float64))
        self.lib.blo_set_modes(self.h, n, m, _p(zmode), _p(tmode), *[_p(q) for q in qs])

    def set_state(self, U, V, W, t=0.0):
        U, V, W = _f(U), _f(V), _f(W)
        self.lib.blo_set_state(self.h, _p(U), _p(V), _p(W), float(t))

    def set_les(self, les_model):
        self.lib.blo_set_les(self.h, int(les_model))

    def set_nu_t(self, nu_t, les_model=1):
        a = _f(nu_t)
        self.lib.blo_set_nu_t(self.h, _p(a), int(les_model))

    def state(self):
        U = np.zeros((self.nx, self.nyg, self.nzg), order="F")
        V = np.zeros((self.nxg, self.ny, self.nzg), order="F")
        W = np.zeros((self.nxg, self.nyg, self.nz), order="F")
        P = np.zeros((self.nxg, self.nyg, self.nzg), order="F")
        t = ctypes.c_double()
        self.lib.blo_get_state(self.h, _p(U), _p(V), _p(W), _p(P), ctypes.byref(t))
        return U, V, W, P, t.value

    def compute_dt(self):
        return self.lib.blo_compute_dt(self.h)

    def set_dt(self, dt):
        self.lib.blo_set_dt(self.h, float(dt))

    def dt(self):
        return self.lib.blo_get_dt(self.h)

    def step(self):
        self.lib.blo_step(self.h)

    def rk3_stage(self, stage):
        self.lib.blo_rk3_stage(self.h, int(stage))

    def advance(self, nsteps):
        """main.f90:87-96 loop body: compute_dt then one time step"""
        for _ in range(nsteps):
            self.compute_dt()
            self.step()

    def rhs(self, U, V, W):
        U, V, W = _f(U), _f(V), _f(W)
        nx, ny, nz, nxg, nyg, nzg = self.nx, self.ny, self.nz, self.nxg, self.nyg, self.nzg
        ru = np.zeros((nx - 2, nyg - 2, nzg - 2), order="F")
        rv = np.zeros((nxg - 2, ny - 2, nzg - 2), order="F")
        rw = np.zeros((nxg - 2, nyg - 2, nz - 2), order="F")
        self.lib.blo_rhs_u(self.h, _p(U), _p(V), _p(W), _p(ru))
        self.lib.blo_rhs_v(self.h, _p(U), _p(V), _p(W), _p(rv))
        self.lib.blo_rhs_w(self.h, _p(U), _p(V), _p(W), _p(rw))
        return ru, rv, rw

    def apply_bc(self, rk_step):
        self.lib.blo_apply_bc(self.h, int(rk_step))

    def projection(self, rk_step):
        self.lib.blo_projection(self.h, int(rk_step))

    def rhs_p(self):
        r = np.zeros((self.nxg - 2, self.nyg - 2, self.nzg - 1), order="F")
        self.lib.blo_get_rhs_p(self.h, _p(r))
        return r

    def max_divergence(self):
        return self.lib.blo_max_divergence(self.h)

    def smagorinsky(self):
        self.lib.blo_smagorinsky(self.h)
        a = np.zeros((self.nxg, self.nyg, self.nzg), order="F")
        self.lib.blo_get_nu_t(self.h, _p(a))
        return a

    def nu_t(self):
        a = np.zeros((self.nxg, self.nyg, self.nzg), order="F")
        self.lib.blo_get_nu_t(self.h, _p(a))
        return a

    def dynamic_smagorinsky(self, model):
        """nu_t of the dynamic model (subgrid.f90:261-583): model 2 with the
        coefficient averaged in z, 3 without; the oracle's LES flag is set to it."""
        self.lib.blo_set_les(self.h, int(model))
        self.lib.blo_dynamic_smagorinsky(self.h)
        return self.nu_t()

    def statistics(self):
        nx, ny = self.nx, self.ny
        means = np.zeros((9, ny, nx))
        ntm = np.zeros((self.nyg, self.nxg))
        cf, du, sc = np.zeros(nx), np.zeros(nx), np.zeros(5)
        self.lib.blo_statistics(self.h, _p(means), _p(ntm), _p(cf), _p(du), _p(sc))
        names = ["Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "UVmean", "Pmean", "P2mean"]
        out = {n: means[q].T.copy(order="F") for q, n in enumerate(names)}
        out.update(nu_t_mean=ntm.T.copy(order="F"), Cf=cf, dUdy_wall=du, theta_inlet=sc[0], delta99_inlet=sc[1],
                   Rex_inlet=sc[2], Retheta_inlet=sc[3], Redelta_inlet=sc[4])
        return out

    def law_of_the_wall(self, utau_guess):
        u = np.ascontiguousarray(utau_guess, dtype=np.float64).copy()
        it = self.lib.blo_law_of_wall(self.h, _p(u))
        return u, it

    def set_rescaling(self, mode, i_rescale, delta_inlet, T_resc, Umean0=None, Vmean0=None):
        u = None if Umean0 is None else np.ascontiguousarray(Umean0, dtype=np.float64)
        v = None if Vmean0 is None else np.ascontiguousarray(Vmean0, dtype=np.float64)
        rc = self.lib.blo_set_rescaling(self.h, mode, i_rescale, delta_inlet, T_resc,
                                        _p(u) if u is not None else None, _p(v) if v is not None else None)
        if rc:
            raise ValueError("blo_set_rescaling: %d" % rc)

    def rescaled_inflow(self):
        self.lib.blo_rescaled_inflow(self.h)

    def rescaling(self):
        """Running means, inflow planes (Fortran-ordered (nyg,nzg), (ny,nzg),
        (nyg,nz)) and diagnostics of the last Lund evaluation."""
        nyg, ny, nzg, nz = self.nyg, self.ny, self.nzg, self.nz
        um, vm, ui, vi = np.zeros(nyg), np.zeros(ny), np.zeros(nyg), np.zeros(ny)
        lu, lv, lw = (np.zeros((nyg, nzg), order="F"), np.zeros((ny, nzg), order="F"),
                      np.zeros((nyg, nz), order="F"))
        dg = np.zeros(8)
        err = ctypes.c_int(0)
        self.lib.blo_get_rescaling(self.h, _p(um), _p(vm), _p(ui), _p(vi), _p(lu), _p(lv), _p(lw), _p(dg),
                                   ctypes.byref(err))
        names = ["Uinf", "delta_resc", "delta_inlet", "theta_resc", "theta_inlet", "utau_resc", "utau_inlet",
                 "gamma"]
        return dict(Umean_resc=um, Vmean_resc=vm, Umean_inlet=ui, Vmean_inlet=vi, U=lu, V=lv, W=lw,
                    diag=dict(zip(names, dg)), err=err.value)

    def set_wall_model(self, mode, jh=3, params=None):
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        rc = self.lib.blo_set_wall_model(self.h, mode, jh, _p(p) if p is not None else None)
        if rc:
            raise ValueError("blo_set_wall_model: %d" % rc)

    def wall_stress(self):
        """(tau_x, tau_z) of the wall model on the current state, shape (nzg-3, nx-2)."""
        n = (self.nx - 2) * (self.nzg - 3)
        tx, tz = np.zeros(n), np.zeros(n)
        self.lib.blo_wall_stress(self.h, _p(tx), _p(tz))
        return tx.reshape(self.nzg - 3, self.nx - 2), tz.reshape(self.nzg - 3, self.nx - 2)


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mlp_forward(params, X, exact=False):
    """Network outputs Y[rows][2] for inputs X[rows][4] (the BF16 roundings of
    the tensor-core kernels unless exact)."""
    lib = load()
    p = np.ascontiguousarray(params, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.zeros((X.shape[0], 2), dtype=np.float32)
    lib.blo_mlp_forward(_p(p), _fptr(X), X.shape[0], _fptr(Y), 1 if exact else 0)
    return Y


def mlp_gradient(params, X, T, exact=False):
    """(loss, gradient[8770]) of the network over samples X, T."""
    lib = load()
    p = np.ascontiguousarray(params, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    g = np.zeros(lib.blo_mlp_nparams())
    loss = lib.blo_mlp_gradient(_p(p), _fptr(X), _fptr(T), X.shape[0], _p(g), 1 if exact else 0)
    return loss, g


def oracle_for(case, variant=0, threads=1):
    """An Oracle loaded with a blgpu.cases.Case (grid, boundary, state)."""
    o = Oracle(case.nx, case.ny, case.nz, case.nu, case.cfl, case.dpdx, case.dpdz, case.rk_scheme,
               variant=variant, threads=threads)
    o.set_grid(case.x, case.y, case.z)
    o.set_bc(*case.bc)
    o.set_state(case.U, case.V, case.W, case.t)
    if case.cfl < 0:
        o.set_dt(-case.cfl)
    if getattr(case, "lund", None):
        o.set_rescaling(*case.lund)
    return o
