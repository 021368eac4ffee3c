"""Failure detection on the device, without faulting it.

A NaN or an infinity in host arrays handed to the upload entry points is
found by the repack kernel (a flag bit, no trap) and reported as
BLGPU_EDEVICE; the context stays usable and takes a clean state afterwards.
"""
import numpy as np
import pytest

from blgpu import cases, BlgpuError, FP64, MIXED

pytestmark = pytest.mark.gpu


def _case():
    c = cases.laminar_case(nx=40, ny=13, nz=18, lx=20.0, ly=5.0, lz=3.0)
    rng = np.random.default_rng(3)
    c.W = np.asfortranarray(c.W + 1e-3 * rng.standard_normal(c.W.shape))
    return c


@pytest.mark.parametrize("precision", [FP64, MIXED])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_upload_rejects_non_finite(gpu, precision, bad):
    c = _case()
    s = cases.solver_for(c, precision=precision)
    V = np.array(c.V, order="F")
    V[7, 4, 9] = bad
    with pytest.raises(BlgpuError, match="NaN or an infinity"):
        s.upload_state(c.U, V, c.W)
    # the context still works: a clean state steps and matches a fresh context
    s.upload_state(c.U, c.V, c.W)
    s.advance(2)
    r = cases.solver_for(c, precision=precision)
    r.advance(2)
    for a, b in zip(s.download_state()[:3], r.download_state()[:3]):
        assert np.array_equal(a, b)
    s.close()
    r.close()


def test_streamed_upload_reports_non_finite_at_sync(gpu):
    c = _case()
    s = cases.solver_for(c)
    U = np.array(c.U, order="F")
    U[3, 2, 1] = np.nan
    s.upload_state_async(U, c.V, c.W)
    with pytest.raises(BlgpuError, match="NaN or an infinity"):
        s.sync()
    s.close()


@pytest.mark.parametrize("thomas", [2, 3])
def test_y_solve_wait_limit_reports_and_recovers(gpu, thomas):
    """The tiled y-solve's mbarrier wait given zero polls (one lane per mode,
    and the rows split over the lanes): every tile's wait gives up at once,
    the CTAs drain their copies (normal limit) and leave, the step reports
    BLGPU_EDEVICE through the device flag; with the limit restored and the
    state uploaded again the context steps exactly as a fresh one."""
    c = _case()
    c.cfl = -1e-3
    s = cases.solver_for(c, precision=FP64)
    assert s.tiles()["thomas"] == 0
    s.set_tiles(thomas=thomas)
    s.set_wait_limit(0)
    s.time_step()
    with pytest.raises(BlgpuError, match="y-solve"):
        s.sync()
    s.sync()  # reported once
    s.set_wait_limit(-1)
    s.upload_state(c.U, c.V, c.W)
    s.set_dt(1e-3)
    s.advance(2)
    r = cases.solver_for(c, precision=FP64)
    r.set_tiles(thomas=thomas)
    r.advance(2)
    for a, b in zip(s.download_state()[:3], r.download_state()[:3]):
        assert np.array_equal(a, b)
    s.close()
    r.close()


def test_rhs_plane_wait_limit_reports_and_recovers(gpu):
    """The TMA-fed RHS (mixed form, rhs_pts 4) given zero polls: every CTA's
    first plane wait gives up, the CTA drains the copies it issued and
    leaves, the step reports BLGPU_EDEVICE; with the limit restored and the
    state uploaded again the context steps exactly as a fresh one."""
    c = _case()
    c.cfl = -1e-3
    s = cases.solver_for(c, precision=MIXED)
    s.set_tiles(rhs_pts=4, thomas=1)  # the register-ring y-solve waits on no mbarrier
    s.set_wait_limit(0)
    s.time_step()
    with pytest.raises(BlgpuError, match="RHS"):
        s.sync()
    s.sync()  # reported once
    s.set_wait_limit(-1)
    s.upload_state(c.U, c.V, c.W)
    s.set_dt(1e-3)
    s.advance(2)
    r = cases.solver_for(c, precision=MIXED)
    r.set_tiles(rhs_pts=4, thomas=1)
    r.advance(2)
    for a, b in zip(s.download_state()[:3], r.download_state()[:3]):
        assert np.array_equal(a, b)
    s.close()
    r.close()
