"""The transition case's inflow modes (host side): the Orr-Sommerfeld solver
against Orszag's known answer for plane Poiseuille flow, the Blasius TS mode
it forces, and the mode file it writes read back through the C ABI
(blgpu_read_temporal_modes)."""
import numpy as np
import pytest

from blgpu import files, transition


def test_orr_sommerfeld_poiseuille_known_answer():
    """Plane Poiseuille flow, Re = 10000, alpha = 1: the least stable
    eigenvalue c = 0.23752649 + 0.00373967 i (Orszag, J. Fluid Mech. 50, 1971)."""
    prof = (lambda y: 1.0 - (y - 1.0) ** 2, lambda y: -2.0 * np.ones_like(y))
    os_ = transition.OrrSommerfeld(10000.0, n=100, y_max=2.0, profile=prof)
    w, _ = os_.modes(1.0, 0.0)
    c = w[np.argmax(w.imag)] / 1.0
    assert abs(c.real - 0.23752649) < 1e-7 and abs(c.imag - 0.00373967) < 1e-7, c


def test_blasius_ts_mode():
    """Re_delta* = 1000, omega = 0.1: an unstable TS wave (phase speed about
    0.36, temporal growth rate a few 1e-3), converged in the resolution."""
    a = transition.OrrSommerfeld(1000.0, n=100).alpha_for(0.1, 0.0)
    b = transition.OrrSommerfeld(1000.0, n=140).alpha_for(0.1, 0.0)
    assert abs(a - b) < 1e-7
    w, v = transition.OrrSommerfeld(1000.0, n=140).ts_mode(b, 0.0)
    assert 0.3 < 0.1 / b < 0.42 and 1e-3 < w.imag < 6e-3


def test_mode_file_round_trip(tmp_path):
    p = tmp_path / "ts_modes.dat"
    info = transition.ts_mode_file(p, n_cheb=100, ny_inlet=150)
    assert set(info) == {"beta=+0.00", "beta=+0.20", "beta=-0.20"}
    y = transition.transition_case(nx=16, ny=33, nz=8, lx=10.0).y
    r = files.read_temporal_modes(p, y)
    assert r["info"]["n_modes"] == 3 and r["info"]["m_modes"] == 1
    assert np.allclose(r["zmode"], [0.0, 0.2, -0.2]) and np.allclose(r["tmode"], [0.1])
    # amplitudes as written: max |u| 1e-3 for the 2-D wave, 1e-4 for each oblique mode
    # (on the coarser solver mesh the interpolated maxima sit slightly below)
    amp = np.abs(r["qu"][:, :, 0]).max(axis=0)
    assert 0.95e-3 < amp[0] <= 1.0e-3 + 1e-12 and np.all((amp[1:] > 0.95e-4) & (amp[1:] <= 1.0e-4 + 1e-13))
    # the wall-normal velocity vanishes at the wall face, the 2-D mode has no w
    assert np.abs(r["qv"][0]).max() < 1e-12 and np.abs(r["qw"][:, 0]).max() == 0.0
