"""Host set-up (no GPU): Blasius table and inflow vectors against the
reference's shipped data (golden fixtures from tests/golden/make_golden.py)."""
import json
import os

import numpy as np

from blgpu import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_blasius_table_matches_reference_file():
    g = json.load(open(os.path.join(GOLD, "blasius_ref.json")))
    eta, f, df, fpp0 = cases.blasius_table(n_points=g["n"])
    idx = np.array(g["index"])
    assert np.abs(eta[idx] - np.array(g["eta"])).max() < 1e-14
    # the reference integrates with f''(0) = 0.46960 (rounded); ours shoots f'(inf)=1
    assert np.abs(f[idx] - np.array(g["f"])).max() < 1e-6
    assert np.abs(df[idx] - np.array(g["df"])).max() < 1e-7
    assert abs(fpp0 - 0.46960) < 1e-6


def test_blasius_inflow_vectors():
    c = cases.laminar_case(nx=32, ny=24, nz=8)
    U_in, V_in, W_in, U_top, V_top, W_top = c.bc
    assert U_in.size == c.ny + 1 and V_in.size == c.ny and V_top.size == c.nx + 1
    # wall value below zero (ghost, extrapolated), free stream -> 1
    assert U_in[0] < 0 < U_in[1] and abs(U_in[-1] - 1.0) < 1e-6
    # V_top = (eta f' - f)/sqrt(2 Re_x) at eta_max: ~0.8604/sqrt(2 Re_x) * sqrt(2)
    rex = cases.centres_ghost(c.x) / c.nu
    assert np.allclose(V_top * np.sqrt(2 * rex), V_top[0] * np.sqrt(2 * rex[0]))
    assert np.all(W_in == 0) and np.all(W_top == 0)


def test_grid_builders():
    z = cases.periodic_faces(10, 3.0)
    zg = cases.centres_ghost(z)
    # nz-2 distinct centres span one period: zg(nz-1)-zg(1)... zg[k] for k=1..nz-2
    assert abs((zg[8] - zg[0]) - 3.0) < 1e-14
    y = cases.tanh_faces(33, 6.0, 1.5)
    assert y[0] == 0.0 and abs(y[-1] - 6.0) < 1e-12 and np.all(np.diff(y) > 0)
    assert np.diff(y)[0] < np.diff(y)[-1]


def test_temporal_mode_file_fixture():
    g = json.load(open(os.path.join(GOLD, "temporal_modes_ref.json")))
    assert g["bytes"] == 28 + 8 * (g["ny_inlet"] + g["n_modes"] + g["m_modes"]) + 48 * g["ny_inlet"] * g["n_modes"] * g["m_modes"]


def test_ensemble_cases_follow_the_recipe():
    bs = cases.ensemble_cases(nbox=12, seed=5)
    assert len(bs) == 12
    for c in bs:
        assert c.nx in (128, 192, 256) and c.ny == 65 and c.nz in (64, 96)
        assert 800.0 <= c.retheta <= 1500.0
        assert c.lund[0] == 3 and 2 <= c.lund[1] <= c.nx
        assert abs((c.x[1] - c.x[0]) - 100.0 / 814.0) < 1e-3
    assert len({(c.nx, c.nz) for c in bs}) > 1
