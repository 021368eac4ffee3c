"""output_data / read_input_data for a context: a run restarted from its
own snapshot continues as the uninterrupted run does, and the Lund means
file carries the running means."""
import os

import numpy as np
import pytest

from blgpu import cases, files, FP64, MIXED

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_restart_continues_bit_identically(gpu, tmp_path, precision):
    c = cases.turbulent_case(nx=66, ny=33, nz=20, lx=8.0, ly=2.0, lz=3.0, seed=5, cfl=-0.01)
    a = cases.solver_for(c, precision=precision, inflow=False)
    a.advance(3)
    out = str(tmp_path / "data" / "BL")
    a.output_data(out, 3)
    name = files.snapshot_name(out, 3)
    assert os.path.realpath(out + ".restart") == os.path.realpath(name)
    b = cases.solver_for(c, precision=precision, inflow=False)
    assert b.read_input_data(name) == 3
    assert np.array_equal(b.x, c.x) and np.array_equal(b.y, c.y) and np.array_equal(b.z, c.z)
    assert b.time()[0] == a.time()[0]
    a.advance(2)
    b.advance(2)
    for p, q in zip(a.download_state()[:3], b.download_state()[:3]):
        assert np.array_equal(p, q)
    a.close()
    b.close()


def test_rescaling_means_file(gpu, tmp_path):
    c = cases.turbulent_case(nx=66, ny=33, nz=20, lx=8.0, ly=2.0, lz=3.0, seed=6, cfl=-0.01)
    a = cases.solver_for(c, precision=FP64)
    a.advance(2)
    out = str(tmp_path / "BL")
    a.output_data(out, 2, rescaling=True)
    um, vm = files.read_rescaling(files.snapshot_name(out, 2) + ".mean.rescaling", c.ny)
    r = a.rescaling()
    assert np.array_equal(um, r["Umean_resc"]) and np.array_equal(vm, r["Vmean_resc"])
    s = files.read_snapshot(files.snapshot_name(out, 2))
    U, V, W, P, t = a.download_state()
    assert s["t"] == t and np.array_equal(s["U"][:, :, :-1], U[:, :, :-1]) and np.array_equal(s["P"], P)
    a.close()


def test_unknown_les_model_refused(gpu):
    """An LES flag outside 0..3 (and the host-supplied -1) is refused by
    blgpu_create instead of running another model."""
    from blgpu import Solver, BlgpuError
    for les in (4, -2):
        with pytest.raises(BlgpuError, match="unknown LES model"):
            Solver(34, 17, 12, 1e-3, -0.01, les_model=les)


def test_output_statistics(gpu, tmp_path):
    """output_statistics for a context: the device statistics in the
    reference's text layout, named with istep + nstep_init and headed with
    istep; every value equals compute_statistics' to the file's 8 decimals."""
    c = cases.laminar_case(nx=34, ny=17, nz=12)
    s = cases.solver_for(c)
    s.advance(2)
    st = s.compute_statistics()
    out = str(tmp_path / "stats" / "BL")
    s.output_statistics(out, 5, nstep_init=10)
    r = files.read_statistics(files.snapshot_name(out, 15) + ".stats.txt")
    assert (r["nx"], r["ny"], r["nz"], r["istep"]) == (34, 17, 12, 5)
    assert abs(r["t"] - s.time()[0]) <= 5.01e-9 and r["nu"] == round(c.nu, 8)
    assert np.abs(r["x"] - s.x).max() <= 5.01e-9 and np.abs(r["y"] - s.y).max() <= 5.01e-9
    assert np.abs(r["Cf"] - st["Cf"]).max() <= 5.01e-9
    for name in ("Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "Pmean", "P2mean"):
        assert r[name].shape == (34, 17)
        assert np.abs(r[name] - st[name]).max() <= 5.01e-9 * max(1.0, np.abs(st[name]).max()), name
    s.close()
