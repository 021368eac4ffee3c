"""ctypes binding of lib/libblgpu.so (the C ABI declared in include/blgpu.h).

The library is the only compute path: if it is missing or fails to load the
import raises, there is no CPU fallback.
"""
import ctypes
import os

from ._build import LIB_PATH

c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)


class Config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nu", ctypes.c_double), ("cfl", ctypes.c_double),
        ("dpdx", ctypes.c_double), ("dpdz", ctypes.c_double),
        ("rk_scheme", ctypes.c_int), ("les_model", ctypes.c_int),
        ("precision", ctypes.c_int), ("poisson", ctypes.c_int), ("device", ctypes.c_int),
    ]


class Params(ctypes.Structure):
    """blgpu_params: the .turbb keys of initparams (params.f90:119-197)."""
    _fields_ = [
        ("nu", ctypes.c_double), ("cfl", ctypes.c_double), ("vmax", ctypes.c_double),
        ("x0", ctypes.c_double), ("sigma", ctypes.c_double), ("phi", ctypes.c_double),
        ("nsteps", ctypes.c_int), ("nsave", ctypes.c_int), ("nstats", ctypes.c_int), ("nmonitor", ctypes.c_int),
        ("nxyz", ctypes.c_int * 3), ("boxsize", ctypes.c_double * 4),
        ("inflow_flag", ctypes.c_int), ("top_flag", ctypes.c_int), ("inflow_file", ctypes.c_char * 201),
        ("lund_ix", ctypes.c_int), ("lund_deltai", ctypes.c_double), ("lund_T", ctypes.c_double),
        ("dpdx", ctypes.c_double), ("dpdz", ctypes.c_double),
        ("les", ctypes.c_int), ("wm", ctypes.c_int), ("tauw_model", ctypes.c_int), ("nut_bc", ctypes.c_int),
        ("wm_nut_flag", ctypes.c_int), ("wm_nut", ctypes.c_double), ("amplitude", ctypes.c_double),
        ("init_step", ctypes.c_int), ("init_rand", ctypes.c_int),
        ("filein", ctypes.c_char * 201), ("fileout", ctypes.c_char * 201), ("timeinflow_file", ctypes.c_char * 201),
        ("rk_scheme", ctypes.c_int), ("alphas", ctypes.c_double * 5), ("found", ctypes.c_ulonglong),
    ]


# .turbb keys in the order of the bits of Params.found
PARAM_KEYS = ["nu", "CFL", "Vmax", "x0", "sigma", "phi", "nsteps", "nsave", "nstats", "nmonitor", "nxyz",
              "boxsize", "inflow_flag", "top_flag", "inflow_file", "Lund_ix", "Lund_deltai", "Lund_T", "dPdx",
              "dPdz", "LES", "WM", "TauwModel", "nutBC", "WMnutflag", "WMnut", "Amplitude", "init_step",
              "init_rand", "filein", "fileout", "timeinflow_file", "RKscheme", "alphas"]


class ModesInfo(ctypes.Structure):
    _fields_ = [("ny_inlet", ctypes.c_int), ("n_modes", ctypes.c_int), ("m_modes", ctypes.c_int),
                ("beta", ctypes.c_double), ("omega", ctypes.c_double)]


class SnapshotInfo(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("nu", ctypes.c_double), ("step", ctypes.c_int),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("full_planes", ctypes.c_int), ("has_nu_t_p", ctypes.c_int)]


FP64 = 0
MIXED = 1
POISSON_NATIVE = 0
POISSON_CUFFT = 1
LES_HOST = -1  # les_model: eddy viscosity supplied by the host

_SIGS = {
    "blgpu_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    "blgpu_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "blgpu_set_grid": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p, c_double_p]),
    "blgpu_set_boundary": (ctypes.c_int, [ctypes.c_void_p] + [c_double_p] * 6),
    "blgpu_set_inflow_modes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [c_double_p] * 5),
    "blgpu_set_rescaling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, c_double_p, c_double_p]),
    "blgpu_rescaled_inflow": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_get_rescaling": (ctypes.c_int, [ctypes.c_void_p] + [c_double_p] * 8 + [ctypes.POINTER(ctypes.c_int)]),
    "blgpu_set_nu_t": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "blgpu_upload_state": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p, c_double_p, ctypes.c_double]),
    "blgpu_download_state": (ctypes.c_int, [ctypes.c_void_p] + [c_double_p] * 5),
    "blgpu_upload_state_async": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p, c_double_p, ctypes.c_double]),
    "blgpu_download_state_async": (ctypes.c_int, [ctypes.c_void_p] + [c_double_p] * 3),
    "blgpu_compute_dt": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "blgpu_set_dt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "blgpu_get_time": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p]),
    "blgpu_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "blgpu_time_step": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_compute_rhs": (ctypes.c_int, [ctypes.c_void_p] + [c_double_p] * 6),
    "blgpu_apply_bc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "blgpu_projection": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "blgpu_get_rhs_p": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "blgpu_max_divergence": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "blgpu_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_device_bytes": (ctypes.c_longlong, [ctypes.c_void_p]),
    "blgpu_phase_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p,
                                         ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    "blgpu_kernel_launches": (ctypes.c_longlong, [ctypes.c_void_p]),
    "blgpu_advance_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p]),
    "blgpu_eddy_viscosity": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_get_nu_t": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "blgpu_statistics": (ctypes.c_int, [ctypes.c_void_p] + [c_double_p] * 5),
    "blgpu_law_of_wall": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.POINTER(ctypes.c_int)]),
    "blgpu_check_divergence_noalloc": (ctypes.c_int, [ctypes.c_void_p] * 6 + [ctypes.c_int] * 3
                                       + [ctypes.c_void_p, ctypes.c_void_p]),
    "blgpu_set_tiles": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "blgpu_get_tiles": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "blgpu_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p, c_double_p]),
    "blgpu_ensemble_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_void_p)]),
    "blgpu_ensemble_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_ensemble_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "blgpu_ensemble_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "blgpu_ensemble_advance_sequential": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "blgpu_ensemble_time": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_double_p]),
    "blgpu_ensemble_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_ensemble_launches": (ctypes.c_longlong, [ctypes.c_void_p]),
    "blgpu_ensemble_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "blgpu_mlp_nparams": (ctypes.c_int, []),
    "blgpu_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_void_p)]),
    "blgpu_mlp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_mlp_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "blgpu_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "blgpu_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "blgpu_mlp_forward": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int, c_float_p]),
    "blgpu_mlp_gradient": (ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_int, c_float_p, c_float_p]),
    "blgpu_mlp_add_data": (ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_int]),
    "blgpu_mlp_sample": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "blgpu_mlp_clear_data": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_mlp_num_samples": (ctypes.c_int, [ctypes.c_void_p]),
    "blgpu_mlp_get_data": (ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_int]),
    "blgpu_mlp_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, c_float_p]),
    "blgpu_mlp_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "blgpu_mlp_loss_history": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "blgpu_mlp_eval": (ctypes.c_int, [ctypes.c_void_p, c_float_p]),
    "blgpu_set_wall_model": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "blgpu_wall_stress": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p]),
    "blgpu_box": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 3 + [c_double_p]),
    "blgpu_get_grid": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p, c_double_p]),
    "blgpu_io_last_error": (ctypes.c_char_p, []),
    "blgpu_read_params": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Params)]),
    "blgpu_params_config": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.POINTER(Config)]),
    "blgpu_snapshot_info_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(SnapshotInfo)]),
    "blgpu_read_snapshot": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(SnapshotInfo)] + [c_double_p] * 8),
    "blgpu_write_snapshot": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 3 + [ctypes.c_double] * 2
                             + [ctypes.c_int] + [c_double_p] * 8),
    "blgpu_read_rescaling": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p]),
    "blgpu_write_rescaling": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p]),
    "blgpu_read_inflow_profile_info": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "blgpu_write_statistics": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p,
                                              c_double_p, c_double_p]),
    "blgpu_output_statistics": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "blgpu_read_inflow_profile": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, c_double_p, c_double_p]),
    "blgpu_snapshot_name": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "blgpu_output_data": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "blgpu_read_input_data": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "blgpu_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "blgpu_read_temporal_modes_info": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ModesInfo)]),
    "blgpu_read_temporal_modes": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int] + [c_double_p] * 7),
}

PHASES = ["rhs_rk", "bc", "div_dct", "dft_z", "thomas", "idft_z", "idct", "project", "compute_dt", "time"]

_lib = None


def exported_symbols():
    """Names of the C-ABI entry points this binding declares."""
    return sorted(_SIGS)


def load():
    """Load libblgpu.so; raises OSError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libblgpu.so not built (%s); run __graft_entry__.build()" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class BlgpuError(RuntimeError):
    pass


def check(rc, ctx=None):
    if rc != 0:
        msg = load().blgpu_last_error(ctx)
        raise BlgpuError("blgpu error %d: %s" % (rc, msg.decode() if msg else "?"))


def check_io(rc):
    if rc != 0:
        msg = load().blgpu_io_last_error()
        raise BlgpuError("blgpu error %d: %s" % (rc, msg.decode() if msg else "?"))


def check_mlp(rc, net=None):
    if rc != 0:
        msg = load().blgpu_mlp_last_error(net) if net is not None else load().blgpu_last_error(None)
        raise BlgpuError("blgpu error %d: %s" % (rc, msg.decode() if msg else "?"))


def check_ensemble(rc, ens=None):
    if rc != 0:
        msg = load().blgpu_ensemble_last_error(ens)
        raise BlgpuError("blgpu error %d: %s" % (rc, msg.decode() if msg else "?"))
