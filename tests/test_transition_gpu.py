"""Forced Tollmien-Schlichting wave on the device (inflow_flag = 1 modes from
the Orr-Sommerfeld solve, read back from the reference-format mode file):
the wave grows downstream, and the mixed form's spatial growth rate matches
the FP64 form's."""
import numpy as np
import pytest

from blgpu import files, transition, FP64, MIXED

pytestmark = pytest.mark.gpu


def test_ts_growth_mixed_matches_fp64(gpu, tmp_path):
    beta = 0.2
    lz = 2.0 * np.pi / beta  # one spanwise period of the oblique pair
    p = tmp_path / "ts_modes.dat"
    transition.ts_mode_file(p, beta=beta, n_cheb=100)
    c = transition.transition_case(nx=256, ny=65, nz=32, lx=100.0, ly=20.0, lz=lz)
    modes = files.read_temporal_modes(p, c.y)
    g64, env64, x = transition.run_growth(c, modes, FP64, steps=1100, x_fit=(10.0, 45.0))
    g32, env32, _ = transition.run_growth(c, modes, MIXED, steps=1100, x_fit=(10.0, 45.0))
    print("TS growth rate per delta*: FP64 %.5f, mixed %.5f" % (g64, g32))
    assert np.all(np.isfinite(env64)) and np.all(np.isfinite(env32))
    assert g64 > 0.0
    assert abs(g32 - g64) <= 0.02 * abs(g64)
