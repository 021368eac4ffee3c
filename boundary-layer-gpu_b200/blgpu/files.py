"""The reference's files through the C ABI (host code, no device needed).

read_params       .turbb run parameters (params.f90:119-207, miscel.f90:13-262)
read_snapshot     flow snapshot (read_input_data, input_output.f90:288-487)
write_snapshot    flow snapshot in the one-process layout (output_data, input_output.f90:496-680)
read_rescaling,
write_rescaling   <snapshot>.mean.rescaling Lund means (input_output.f90:440-458, 668-676)
snapshot_name     fileout.%08d
read_temporal_modes  the binary temporal inflow-mode file of the transition case
                  (compute_blasius_solution_for_bc, boundary_conditions.f90:1652-1797)
read_inflow_profile  the inflow_file of inflow flags 2 and 5 (boundary_conditions.f90:1405, 1550)
write_statistics,
read_statistics   <fileout>.<step>.stats.txt (output_statistics, input_output.f90:685-746)
"""
import ctypes

import numpy as np

from ._lib import Config, ModesInfo, Params, PARAM_KEYS, SnapshotInfo, check_io, load


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _f64(a):
    return np.asfortranarray(a, dtype=np.float64)


def read_params(path):
    """dict of the .turbb keys that were given (reference key names), plus
    'found' (list of those names) and 'config' (the blgpu_config fields)."""
    p = Params()
    check_io(load().blgpu_read_params(str(path).encode(), ctypes.byref(p)))
    out = {}
    vals = {
        "nu": p.nu, "CFL": p.cfl, "Vmax": p.vmax, "x0": p.x0, "sigma": p.sigma, "phi": p.phi,
        "nsteps": p.nsteps, "nsave": p.nsave, "nstats": p.nstats, "nmonitor": p.nmonitor,
        "nxyz": list(p.nxyz), "boxsize": list(p.boxsize), "inflow_flag": p.inflow_flag, "top_flag": p.top_flag,
        "inflow_file": p.inflow_file.decode(), "Lund_ix": p.lund_ix, "Lund_deltai": p.lund_deltai,
        "Lund_T": p.lund_T, "dPdx": p.dpdx, "dPdz": p.dpdz, "LES": p.les, "WM": p.wm,
        "TauwModel": p.tauw_model, "nutBC": p.nut_bc, "WMnutflag": p.wm_nut_flag, "WMnut": p.wm_nut,
        "Amplitude": p.amplitude, "init_step": p.init_step, "init_rand": p.init_rand,
        "filein": p.filein.decode(), "fileout": p.fileout.decode(), "timeinflow_file": p.timeinflow_file.decode(),
        "RKscheme": p.rk_scheme, "alphas": list(p.alphas),
    }
    found = [k for q, k in enumerate(PARAM_KEYS) if p.found >> q & 1]
    for k in found:
        out[k] = vals[k]
    out["found"] = found
    out["init_step"] = p.init_step  # -45 when not given
    cfg = Config()
    check_io(load().blgpu_params_config(ctypes.byref(p), ctypes.byref(cfg)))
    out["config"] = {f: getattr(cfg, f) for f, _ in Config._fields_ if f in
                     ("nx", "ny", "nz", "nu", "cfl", "dpdx", "dpdz", "rk_scheme", "les_model")}
    return out


def snapshot_info(path):
    h = SnapshotInfo()
    check_io(load().blgpu_snapshot_info_read(str(path).encode(), ctypes.byref(h)))
    return {f: getattr(h, f) for f, _ in SnapshotInfo._fields_}


def read_snapshot(path):
    """dict with t, nu, step, x, y, z, U, V, W, nu_t, P (Fortran-layout arrays)."""
    info = snapshot_info(path)
    nx, ny, nz = info["nx"], info["ny"], info["nz"]
    nxg, nyg, nzg = nx + 1, ny + 1, nz + 1
    x, y, z = np.zeros(nx), np.zeros(ny), np.zeros(nz)
    U = np.zeros((nx, nyg, nzg), order="F")
    V = np.zeros((nxg, ny, nzg), order="F")
    W = np.zeros((nxg, nyg, nz), order="F")
    nt = np.zeros((nxg, nyg, nzg), order="F")
    P = np.zeros((nxg, nyg, nzg), order="F")
    h = SnapshotInfo()
    check_io(load().blgpu_read_snapshot(str(path).encode(), ctypes.byref(h), _p(x), _p(y), _p(z), _p(U), _p(V),
                                        _p(W), _p(nt), _p(P)))
    out = {f: getattr(h, f) for f, _ in SnapshotInfo._fields_}
    out.update(x=x, y=y, z=z, U=U, V=V, W=W, nu_t=nt, P=P)
    return out


def write_snapshot(path, t, nu, step, x, y, z, U, V, W, nu_t=None, P=None):
    nx, ny, nz = len(x), len(y), len(z)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    U, V, W = _f64(U), _f64(V), _f64(W)
    nu_t = _f64(nu_t) if nu_t is not None else None
    P = _f64(P) if P is not None else None
    assert U.shape == (nx, ny + 1, nz + 1) and V.shape == (nx + 1, ny, nz + 1) and W.shape == (nx + 1, ny + 1, nz)
    check_io(load().blgpu_write_snapshot(str(path).encode(), nx, ny, nz, float(t), float(nu), int(step), _p(x),
                                         _p(y), _p(z), _p(U), _p(V), _p(W), _p(nu_t), _p(P)))


def read_rescaling(path, ny):
    um, vm = np.zeros(ny + 1), np.zeros(ny)
    check_io(load().blgpu_read_rescaling(str(path).encode(), ny + 1, ny, _p(um), _p(vm)))
    return um, vm


def write_rescaling(path, Umean, Vmean):
    um, vm = np.ascontiguousarray(Umean, dtype=np.float64), np.ascontiguousarray(Vmean, dtype=np.float64)
    check_io(load().blgpu_write_rescaling(str(path).encode(), len(um), len(vm), _p(um), _p(vm)))


def read_inflow_profile(path, ny=None):
    """inflow_file of inflow flags 2 and 5: (U_inlet at the ny+1 centres,
    V_inlet at the ny faces); ny (the grid's) defaults to the file's."""
    lib = load()
    n = ctypes.c_int()
    check_io(lib.blgpu_read_inflow_profile_info(str(path).encode(), ctypes.byref(n)))
    ny = n.value if ny is None else int(ny)
    U, V = np.zeros(ny + 1), np.zeros(ny)
    check_io(lib.blgpu_read_inflow_profile(str(path).encode(), ny, _p(U), _p(V)))
    return U, V


def write_statistics(path, t, nu, nz, istep, Cf, x, y, means):
    """means: the nine (nx, ny) arrays of Solver.statistics, in its order
    (Umean, Vmean, Wmean, U2mean, V2mean, W2mean, UVmean, Pmean, P2mean)."""
    Cf, x, y = (np.ascontiguousarray(a, dtype=np.float64) for a in (Cf, x, y))
    nx, ny = len(x), len(y)
    m = np.asarray(means, dtype=np.float64)
    assert m.shape == (9, nx, ny)
    buf = np.ascontiguousarray(np.stack([np.asfortranarray(a).ravel(order="F") for a in m]))
    check_io(load().blgpu_write_statistics(str(path).encode(), float(t), float(nu), nx, ny, int(nz), int(istep),
                                           _p(Cf), _p(x), _p(y), _p(buf)))


def read_statistics(path):
    """The text of a stats file back as arrays: header (t, nu, nx, ny, nz,
    istep), Cf, x, y and the eight (nx, ny) arrays the file holds."""
    lines = open(path).read().splitlines()
    h = lines[0][1:]
    t, nu = float(h[0:15]), float(h[15:30])
    nx, ny, nz, istep = (int(h[30 + 8 * q:38 + 8 * q]) for q in range(4))
    def num(f):  # a field that did not fit its width reads as NaN
        return np.nan if f.strip().startswith("*") else float(f)

    row = lambda s: np.array([num(s[15 * q:15 * q + 15]) for q in range(len(s) // 15)])
    Cf, x, y = row(lines[1]), row(lines[2]), row(lines[3])
    arrays = [np.array([row(lines[4 + q * nx + i]) for i in range(nx)]) for q in range(8)]
    names = ("Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "Pmean", "P2mean")
    return dict(t=t, nu=nu, nx=nx, ny=ny, nz=nz, istep=istep, Cf=Cf, x=x, y=y, **dict(zip(names, arrays)))


def snapshot_name(fileout, step):
    buf = ctypes.create_string_buffer(4096)
    check_io(load().blgpu_snapshot_name(str(fileout).encode(), int(step), buf, 4096))
    return buf.value.decode()


def temporal_modes_info(path):
    h = ModesInfo()
    check_io(load().blgpu_read_temporal_modes_info(str(path).encode(), ctypes.byref(h)))
    return dict(ny_inlet=h.ny_inlet, n_modes=h.n_modes, m_modes=h.m_modes, beta=h.beta, omega=h.omega)


def read_temporal_modes(path, y):
    """The file's modes on the face grid y(ny) and its centres: zmode (n,),
    tmode (m,) already scaled by beta / omega; qu (ny+1, n, m), qv (ny, n, m),
    qw (ny+1, n, m) complex; ymesh (ny_inlet,).  The arguments of
    Solver.set_inflow_modes."""
    h = temporal_modes_info(path)
    y = np.ascontiguousarray(y, dtype=np.float64)
    ny, n, m = len(y), h["n_modes"], h["m_modes"]
    zm, tm = np.zeros(n), np.zeros(m)
    qu, qw = np.zeros(2 * (ny + 1) * n * m), np.zeros(2 * (ny + 1) * n * m)
    qv, ym = np.zeros(2 * ny * n * m), np.zeros(h["ny_inlet"])
    check_io(load().blgpu_read_temporal_modes(str(path).encode(), ny, _p(y), _p(zm), _p(tm), _p(qu), _p(qv),
                                              _p(qw), _p(ym)))
    cplx = lambda a, n1: a.view(np.complex128).reshape((n1, n, m), order="F")
    return dict(zmode=zm, tmode=tm, qu=cplx(qu, ny + 1), qv=cplx(qv, ny), qw=cplx(qw, ny + 1), ymesh=ym, info=h)
