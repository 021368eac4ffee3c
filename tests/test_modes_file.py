"""The binary temporal inflow-mode file of the transition case (inflow_flag
= 1) through the C ABI (host code, no device): header, scaling by beta and
omega, and the linear interpolation onto the solver's centres and faces of
compute_blasius_solution_for_bc (boundary_conditions.f90:1652-1797).  A
numpy restatement is the check; the reference's own file
(transition_test/temporal_modes_inlet.dat) is read when BLGPU_REFERENCE_DIR
points at the reference tree and compared with the committed golden header."""
import json
import os
import struct

import numpy as np
import pytest

from blgpu import files, BlgpuError

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("BLGPU_REFERENCE_DIR", "")


def write_modes(path, ym, zm, tm, beta, omega, qu, qv, qw, order="<"):
    ny, n, m = qu.shape
    with open(path, "wb") as f:
        f.write(struct.pack(order + "3i", ny, n, m))
        f.write(struct.pack(order + "2d", beta, omega))
        for a in (ym, zm, tm):
            f.write(np.asarray(a, order + "f8").tobytes())
        for q in (qu, qv, qw):
            f.write(np.asfortranarray(q.real).ravel(order="F").astype(order + "f8").tobytes())
            f.write(np.asfortranarray(q.imag).ravel(order="F").astype(order + "f8").tobytes())


def centres_ghost(y):
    c = 0.5 * (y[:-1] + y[1:])
    return np.concatenate([[c[0] - 2.0 * (c[0] - y[0])], c, [c[-1] + 2.0 * (y[-1] - c[-1])]])


def interp_np(ym, q, tgt):
    """boundary_conditions.f90:1730-1774, as numpy"""
    nyi = len(ym)
    out = np.zeros((len(tgt),) + q.shape[1:], dtype=complex)
    for j, yt in enumerate(tgt):
        j1 = nyi
        for jj in range(2, nyi + 1):
            if ym[jj - 1] >= yt:
                j1 = jj
                break
        if j1 == nyi:
            continue
        j0 = j1 - 1
        dy, span = yt - ym[j0 - 1], ym[j1 - 1] - ym[j0 - 1]
        d = q[j1 - 1] - q[j0 - 1]
        out[j] = q[j0 - 1] + (dy * d.real / span + 1j * (dy * d.imag / span))
    return out


@pytest.mark.parametrize("order", ["<", ">"])
def test_synthetic_modes_file(tmp_path, order):
    """Native and big-endian files (the GPU build's runtime reads big-endian)."""
    rng = np.random.default_rng(5)
    nyi, n, m = 40, 3, 2
    ym = np.concatenate([[0.0], np.cumsum(rng.uniform(0.01, 0.05, nyi - 1))])
    zm, tm = np.array([0.0, 1.0, -1.0]), np.array([1.0, 2.0])
    q = [rng.standard_normal((nyi, n, m)) + 1j * rng.standard_normal((nyi, n, m)) for _ in range(3)]
    p = tmp_path / "modes.dat"
    write_modes(p, ym, zm, tm, 2.5, 0.3, *q, order=order)
    y = np.linspace(0.0, ym[-1] * 1.3, 23)  # rows past the mesh end read zero
    r = files.read_temporal_modes(p, y)
    assert r["info"] == dict(ny_inlet=nyi, n_modes=n, m_modes=m, beta=2.5, omega=0.3)
    assert np.array_equal(r["zmode"], 2.5 * zm) and np.array_equal(r["tmode"], 0.3 * tm)
    assert np.array_equal(r["ymesh"], ym)
    yg = centres_ghost(y)
    for got, qq, tgt in ((r["qu"], q[0], yg), (r["qv"], q[1], y), (r["qw"], q[2], yg)):
        ref = interp_np(ym, qq, tgt)
        assert got.shape == ref.shape
        assert np.array_equal(got, ref)
    assert np.all(r["qv"][y >= ym[-1]] == 0)


def test_modes_file_size_checked(tmp_path):
    p = tmp_path / "bad.dat"
    write_modes(p, np.linspace(0, 1, 5), [0.0], [1.0], 1.0, 1.0, *[np.ones((5, 1, 1), complex)] * 3)
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:-8])
    with pytest.raises(BlgpuError, match="bytes"):
        files.temporal_modes_info(p)


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="BLGPU_REFERENCE_DIR not set")
def test_reference_modes_file():
    p = os.path.join(REF, "transition_test", "temporal_modes_inlet.dat")
    gold = json.load(open(os.path.join(HERE, "golden", "temporal_modes_ref.json")))
    h = files.temporal_modes_info(p)
    assert (h["ny_inlet"], h["n_modes"], h["m_modes"]) == (gold["ny_inlet"], gold["n_modes"], gold["m_modes"])
    assert h["beta"] == gold["beta"] and h["omega"] == gold["omega"]
    y = np.linspace(0.0, 0.41, 129)  # the transition case's Ly
    r = files.read_temporal_modes(p, y)
    assert np.allclose(r["zmode"], gold["beta"] * np.array(gold["zmode"]), rtol=0, atol=0)
    assert np.allclose(r["tmode"], gold["omega"] * np.array(gold["tmode"]), rtol=0, atol=0)
    assert [r["ymesh"][0], r["ymesh"][-1]] == gold["ymesh_first_last"]
    # the interpolation against the numpy restatement on the raw payload
    raw = open(p, "rb").read()
    nyi, n, m = h["ny_inlet"], h["n_modes"], h["m_modes"]
    off = 28 + 8 * (nyi + n + m)
    nq = nyi * n * m
    arr = np.frombuffer(raw, "<f8", 6 * nq, off)
    assert [float(np.abs(arr[i * nq:(i + 1) * nq]).sum()) for i in range(6)] == pytest.approx(gold["q_abs_sum"],
                                                                                           rel=1e-14)
    qs = [(arr[2 * c * nq:(2 * c + 1) * nq] + 1j * arr[(2 * c + 1) * nq:(2 * c + 2) * nq]).reshape((nyi, n, m),
                                                                                                   order="F")
          for c in range(3)]
    yg = centres_ghost(y)
    assert np.array_equal(r["qu"], interp_np(r["ymesh"], qs[0], yg))
    assert np.array_equal(r["qv"], interp_np(r["ymesh"], qs[1], y))
    assert np.array_equal(r["qw"], interp_np(r["ymesh"], qs[2], yg))
