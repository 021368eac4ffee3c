"""Host mirror of the reference's step-path subroutines, over the C ABI.

Method names follow the Fortran subroutines they replace
(time_integration.f90, projection.f90, boundary_conditions.f90,
equations.f90); arrays are numpy arrays in the reference's Fortran layout
and bounds:  U(nx,nyg,nzg), V(nxg,ny,nzg), W(nxg,nyg,nz), P(nxg,nyg,nzg).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import FP64, MIXED, POISSON_NATIVE, check


def _p(a):
    return a.ctypes.data_as(_lib.c_double_p)


def _f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


class Solver:
    """One box on one GPU (a blgpu context)."""

    def __init__(self, nx, ny, nz, nu, cfl, dpdx=0.0, dpdz=0.0, rk_scheme=3, les_model=0,
                 precision=FP64, poisson=POISSON_NATIVE, device=0):
        self.lib = _lib.load()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.nxg, self.nyg, self.nzg = self.nx + 1, self.ny + 1, self.nz + 1
        cfg = _lib.Config(self.nx, self.ny, self.nz, float(nu), float(cfl), float(dpdx), float(dpdz),
                          int(rk_scheme), int(les_model), int(precision), int(poisson), int(device))
        h = ctypes.c_void_p()
        check(self.lib.blgpu_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.ctx = h
        self.cfg = cfg

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.blgpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        check(rc, self.ctx)

    # -- set-up (initialization.f90) ---------------------------------------
    def set_grid(self, x, y, z):
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        assert x.size == self.nx and y.size == self.ny and z.size == self.nz
        self._ck(self.lib.blgpu_set_grid(self.ctx, _p(x), _p(y), _p(z)))
        self.x, self.y, self.z = x.copy(), y.copy(), z.copy()

    def set_boundary(self, U_inlet, V_inlet, W_inlet, U_top, V_top, W_top):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (U_inlet, V_inlet, W_inlet, U_top, V_top, W_top)]
        want = [self.nyg, self.ny, self.nyg, self.nx, self.nxg, self.nxg]
        for a, n in zip(arrs, want):
            assert a.size == n, (a.size, n)
        self._bc_keep = arrs
        self._ck(self.lib.blgpu_set_boundary(self.ctx, *[_p(a) for a in arrs]))

    def set_inflow_modes(self, zmode, tmode, qu, qv, qw):
        zmode = np.ascontiguousarray(zmode, dtype=np.float64)
        tmode = np.ascontiguousarray(tmode, dtype=np.float64)
        n, m = zmode.size, tmode.size
        qs = []
        for q, ny_ in ((qu, self.nyg), (qv, self.ny), (qw, self.nyg)):
            q = np.asfortranarray(np.asarray(q, dtype=np.complex128).reshape(ny_, n, m, order="F"))
            qs.append(np.ascontiguousarray(q.ravel(order="F")).view(np.float64))
        self._ck(self.lib.blgpu_set_inflow_modes(self.ctx, n, m, _p(zmode), _p(tmode), *[_p(q) for q in qs]))

    def set_rescaling(self, mode, i_rescale, delta_inlet, T_resc, Umean0=None, Vmean0=None):
        """Lund recycling inflow (inflow_flag 3 or 5; 0 switches it off).
        i_rescale is the reference's 1-based Lund_ix."""
        u = None if Umean0 is None else np.ascontiguousarray(Umean0, dtype=np.float64)
        v = None if Vmean0 is None else np.ascontiguousarray(Vmean0, dtype=np.float64)
        self._ck(self.lib.blgpu_set_rescaling(self.ctx, int(mode), int(i_rescale), float(delta_inlet),
                                              float(T_resc), _p(u) if u is not None else None,
                                              _p(v) if v is not None else None))

    def rescaled_inflow(self):
        """One compute_rescaled_inflow from the current state and dt."""
        self._ck(self.lib.blgpu_rescaled_inflow(self.ctx))

    def rescaling(self):
        """Running means, last inflow planes and diagnostics of the Lund inflow."""
        nyg, ny, nzg, nz = self.nyg, self.ny, self.nzg, self.nz
        um, vm, ui, vi = np.zeros(nyg), np.zeros(ny), np.zeros(nyg), np.zeros(ny)
        lu, lv, lw = (np.zeros((nyg, nzg), order="F"), np.zeros((ny, nzg), order="F"),
                      np.zeros((nyg, nz), order="F"))
        dg = np.zeros(8)
        err = ctypes.c_int(0)
        self._ck(self.lib.blgpu_get_rescaling(self.ctx, _p(um), _p(vm), _p(ui), _p(vi), _p(lu), _p(lv), _p(lw),
                                              _p(dg), ctypes.byref(err)))
        names = ["Uinf", "delta_resc", "delta_inlet", "theta_resc", "theta_inlet", "utau_resc", "utau_inlet",
                 "gamma"]
        return dict(Umean_resc=um, Vmean_resc=vm, Umean_inlet=ui, Vmean_inlet=vi, U=lu, V=lv, W=lw,
                    diag=dict(zip(names, dg)), err=err.value)

    def set_nu_t(self, nu_t):
        a = _f64(nu_t)
        assert a.shape == (self.nxg, self.nyg, self.nzg)
        self._ck(self.lib.blgpu_set_nu_t(self.ctx, _p(a)))

    # -- state ------------------------------------------------------------
    def upload_state(self, U, V, W, t=0.0):
        U, V, W = _f64(U), _f64(V), _f64(W)
        assert U.shape == (self.nx, self.nyg, self.nzg)
        assert V.shape == (self.nxg, self.ny, self.nzg)
        assert W.shape == (self.nxg, self.nyg, self.nz)
        self._ck(self.lib.blgpu_upload_state(self.ctx, _p(U), _p(V), _p(W), float(t)))

    def download_state(self):
        U = np.zeros((self.nx, self.nyg, self.nzg), order="F")
        V = np.zeros((self.nxg, self.ny, self.nzg), order="F")
        W = np.zeros((self.nxg, self.nyg, self.nz), order="F")
        P = np.zeros((self.nxg, self.nyg, self.nzg), order="F")
        t = ctypes.c_double()
        self._ck(self.lib.blgpu_download_state(self.ctx, _p(U), _p(V), _p(W), _p(P), ctypes.byref(t)))
        return U, V, W, P, t.value

    def upload_state_async(self, U, V, W, t=0.0):
        """Streamed upload (returns at once): U, V, W must be Fortran-ordered
        float64 arrays of the state's shapes, pinned for the copy to overlap,
        and left untouched until sync()."""
        for a, sh in ((U, (self.nx, self.nyg, self.nzg)), (V, (self.nxg, self.ny, self.nzg)),
                      (W, (self.nxg, self.nyg, self.nz))):
            assert a.dtype == np.float64 and a.flags.f_contiguous and a.shape == sh
        self._ck(self.lib.blgpu_upload_state_async(self.ctx, _p(U), _p(V), _p(W), float(t)))

    def download_state_async(self, U, V, W):
        """Streamed download of U, V, W into the given arrays (as
        upload_state_async), complete after sync()."""
        for a, sh in ((U, (self.nx, self.nyg, self.nzg)), (V, (self.nxg, self.ny, self.nzg)),
                      (W, (self.nxg, self.nyg, self.nz))):
            assert a.dtype == np.float64 and a.flags.f_contiguous and a.shape == sh
        self._ck(self.lib.blgpu_download_state_async(self.ctx, _p(U), _p(V), _p(W)))

    # -- the reference's files -------------------------------------------------
    def output_data(self, fileout, step, rescaling=False):
        """output_data: writes fileout.<step> (one-process layout), links
        fileout.restart to it and, with rescaling, the Lund means file."""
        _lib.check_io(self.lib.blgpu_output_data(self.ctx, str(fileout).encode(), int(step), int(bool(rescaling))))

    def output_statistics(self, fileout, istep, nstep_init=0):
        """output_statistics: the device statistics written to
        fileout.<istep+nstep_init>.stats.txt in the reference's text layout."""
        _lib.check_io(self.lib.blgpu_output_statistics(self.ctx, str(fileout).encode(), int(istep), int(nstep_init)))

    def read_input_data(self, filein):
        """read_input_data: grid (replaces the current one), U, V, W and t
        from a snapshot; returns the file's step (-1 when absent)."""
        st = ctypes.c_int(0)
        _lib.check_io(self.lib.blgpu_read_input_data(self.ctx, str(filein).encode(), ctypes.byref(st)))
        x, y, z = np.zeros(self.nx), np.zeros(self.ny), np.zeros(self.nz)
        self._ck(self.lib.blgpu_get_grid(self.ctx, _p(x), _p(y), _p(z)))
        self.x, self.y, self.z = x, y, z
        return st.value

    # -- the step path ------------------------------------------------------
    def compute_dt(self):
        dt = ctypes.c_double()
        self._ck(self.lib.blgpu_compute_dt(self.ctx, ctypes.byref(dt)))
        return dt.value

    def set_dt(self, dt):
        self._ck(self.lib.blgpu_set_dt(self.ctx, float(dt)))

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._ck(self.lib.blgpu_get_time(self.ctx, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def time_step(self):
        """compute_time_step_{Euler,RK2,RK3} with the current dt."""
        self._ck(self.lib.blgpu_time_step(self.ctx))

    compute_time_step = time_step

    def advance(self, nsteps=1):
        """nsteps of the main loop body: compute_dt + time step (CUDA graph)."""
        self._ck(self.lib.blgpu_advance(self.ctx, int(nsteps)))

    def advance_timed(self, nsteps):
        """advance(nsteps) timed with CUDA events on the solver stream (ms)."""
        ms = ctypes.c_double()
        self._ck(self.lib.blgpu_advance_timed(self.ctx, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def sync(self):
        self._ck(self.lib.blgpu_sync(self.ctx))

    def compute_rhs(self, U, V, W):
        """compute_rhs_u/v/w: returns the compact interior arrays."""
        U, V, W = _f64(U), _f64(V), _f64(W)
        nx, ny, nz, nxg, nyg, nzg = self.nx, self.ny, self.nz, self.nxg, self.nyg, self.nzg
        ru = np.zeros((nx - 2, nyg - 2, nzg - 2), order="F")
        rv = np.zeros((nxg - 2, ny - 2, nzg - 2), order="F")
        rw = np.zeros((nxg - 2, nyg - 2, nz - 2), order="F")
        self._ck(self.lib.blgpu_compute_rhs(self.ctx, _p(U), _p(V), _p(W), _p(ru), _p(rv), _p(rw)))
        return ru, rv, rw

    def apply_boundary_conditions(self, rk_step):
        self._ck(self.lib.blgpu_apply_bc(self.ctx, int(rk_step)))

    def compute_projection_step(self, rk_step):
        self._ck(self.lib.blgpu_projection(self.ctx, int(rk_step)))

    def rhs_p(self):
        r = np.zeros((self.nxg - 2, self.nyg - 2, self.nzg - 1), order="F")
        self._ck(self.lib.blgpu_get_rhs_p(self.ctx, _p(r)))
        return r

    def check_divergence(self):
        d = ctypes.c_double()
        self._ck(self.lib.blgpu_max_divergence(self.ctx, ctypes.byref(d)))
        return d.value

    # -- models and diagnostics -------------------------------------------
    def compute_eddy_viscosity(self):
        """The context's LES model on the resident state (LES = 1
        sgs_Smagorinsky; 2, 3 the dynamic model); returns nu_t(nxg,nyg,nzg)."""
        self._ck(self.lib.blgpu_eddy_viscosity(self.ctx))
        return self.nu_t()

    def nu_t(self):
        a = np.zeros((self.nxg, self.nyg, self.nzg), order="F")
        self._ck(self.lib.blgpu_get_nu_t(self.ctx, _p(a)))
        return a

    def compute_statistics(self):
        """compute_statistics: dict of z-means, Cf, dUdy_wall and inlet scalars."""
        nx, ny = self.nx, self.ny
        means = np.zeros((9, ny, nx))
        ntm = np.zeros((self.nyg, self.nxg))
        cf = np.zeros(nx)
        du = np.zeros(nx)
        sc = np.zeros(5)
        self._ck(self.lib.blgpu_statistics(self.ctx, _p(means), _p(ntm), _p(cf), _p(du), _p(sc)))
        names = ["Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "UVmean", "Pmean", "P2mean"]
        out = {n: means[q].T.copy(order="F") for q, n in enumerate(names)}
        out.update(nu_t_mean=ntm.T.copy(order="F"), Cf=cf, dUdy_wall=du, theta_inlet=sc[0], delta99_inlet=sc[1],
                   Rex_inlet=sc[2], Retheta_inlet=sc[3], Redelta_inlet=sc[4])
        return out

    def law_of_the_wall(self, utau_guess):
        """compute_law_of_the_wall_model: (utau_model, iters_max)."""
        u = np.ascontiguousarray(utau_guess, dtype=np.float64).copy()
        it = ctypes.c_int()
        self._ck(self.lib.blgpu_law_of_wall(self.ctx, _p(u), ctypes.byref(it)))
        return u, it.value

    def device_bytes(self):
        return int(self.lib.blgpu_device_bytes(self.ctx))

    def kernel_launches(self):
        return int(self.lib.blgpu_kernel_launches(self.ctx))

    # -- wall model ----------------------------------------------------------
    def set_wait_limit(self, polls):
        """Test hook: mbarrier polls of the tiled y-solve before a copy counts
        as lost (< 0: the built-in limit)."""
        self._ck(self.lib.blgpu_set_wait_limit(self.ctx, int(polls)))

    def set_wall_model(self, mode, jh=3, net=None):
        """0 no-slip, 1 law of the wall at row jh, 2 the WallNet `net` at row jh."""
        self._wall_net = net  # the solver reads the network's device weights every substep
        self._ck(self.lib.blgpu_set_wall_model(self.ctx, int(mode), int(jh), net.h if net is not None else None))

    def wall_stress(self):
        """(tau_x, tau_z) of the wall model on the current state, shape (nzg-3, nx-2)."""
        n = (self.nx - 2) * (self.nzg - 3)
        tx, tz = np.zeros(n), np.zeros(n)
        self._ck(self.lib.blgpu_wall_stress(self.ctx, _p(tx), _p(tz)))
        return tx.reshape(self.nzg - 3, self.nx - 2), tz.reshape(self.nzg - 3, self.nx - 2)

    # -- launch shapes -----------------------------------------------------
    TILE_NAMES = ("rhs_kc", "rhs_by", "dct_nw", "dftz_rk", "proj_by", "zdft", "rhs_pts", "thomas", "idct_nw",
                  "xfft")

    def tiles(self):
        t = (ctypes.c_int * 10)()
        self._ck(self.lib.blgpu_get_tiles(self.ctx, t, 10))
        return dict(zip(self.TILE_NAMES, list(t)))

    def set_tiles(self, **kw):
        cur = self.tiles()
        for k, v in kw.items():
            if k not in cur:
                raise KeyError(k)
            cur[k] = int(v)
        t = (ctypes.c_int * 10)(*[cur[k] for k in self.TILE_NAMES])
        self._ck(self.lib.blgpu_set_tiles(self.ctx, t, 10))

    def autotune(self, steps=3):
        """Choose the launch shapes by timing; returns (ms/step before, after)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._ck(self.lib.blgpu_autotune(self.ctx, int(steps), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def phase_times(self, nsteps=1):
        """{phase: (ms total, kernels)} over nsteps eager steps (CUDA events)."""
        n = len(_lib.PHASES)
        ms = (ctypes.c_double * n)()
        kn = (ctypes.c_longlong * n)()
        self._ck(self.lib.blgpu_phase_times(self.ctx, int(nsteps), ms, kn, n))
        return {p: (ms[i], kn[i]) for i, p in enumerate(_lib.PHASES)}
