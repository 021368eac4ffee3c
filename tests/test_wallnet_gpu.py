"""The learned wall-stress model on the GPU: the tensor-core network against
the CPU oracle (forward pass and gradient), deterministic training, the
training-sample extractor, the wall-model hooks of the step against the
oracle, and the learned model checked against the equilibrium law of the wall
(wallmodel.f90:1951-1985): mean skin friction within 2 % of it on a coarse
wall-modelled grid, and what it gains over the no-slip wall there."""
import numpy as np
import pytest

import oracle
from blgpu import cases, wallmodel, FP64, MIXED, WallNet, BlgpuError

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def inputs(rows, seed):
    rng = np.random.default_rng(seed)
    X = np.stack([rng.uniform(0.3, 1.0, rows), rng.normal(0, 0.05, rows), rng.uniform(0.4, 0.9, rows),
                  rng.normal(0, 0.05, rows)], -1).astype(np.float32)
    T = np.stack([1.5 + 2.0 * (X[:, 0] - 0.65) - 1.2 * (X[:, 2] - 0.65), 3.0 * X[:, 1]], -1).astype(np.float32)
    return X, T


def test_forward_matches_oracle(gpu):
    net = WallNet(seed=3)
    X, _ = inputs(1003, 1)
    Y = net.forward(X)
    Yo = oracle.mlp_forward(net.params.astype(np.float64), X)
    assert np.abs(Y - Yo).max() <= 2e-3 * np.abs(Yo).max()
    assert np.abs(Y - Yo).mean() <= 1e-5 * np.abs(Yo).max()


def test_gradient_matches_oracle(gpu):
    net = WallNet(seed=4)
    X, T = inputs(1003, 2)
    loss, g = net.gradient(X, T)
    p = net.params.astype(np.float64)
    lo, go = oracle.mlp_gradient(p, X, T)
    le, ge = oracle.mlp_gradient(p, X, T, exact=True)
    assert abs(loss - lo) <= 1e-5 * lo
    # per tensor: W0 b0 W1 b1 W2 b2 W3 b3
    edges = [0, 256, 320, 4416, 4480, 8576, 8640, 8768, 8770]
    for a, b in zip(edges[:-1], edges[1:]):
        assert rel(g[a:b], go[a:b]) < 5e-3, (a, b, rel(g[a:b], go[a:b]))
        assert rel(g[a:b], ge[a:b]) < 5e-2, (a, b, rel(g[a:b], ge[a:b]))


def test_training_is_deterministic_and_fits(gpu):
    X, T = inputs(20000, 3)
    out = []
    for _ in range(2):
        net = WallNet(seed=5)
        net.add_data(X, T)
        l0 = net.eval()
        net.train(400, batch=4096, lr=2e-3)
        net.train(200, batch=4096, lr=5e-4)
        out.append((l0, net.eval(), net.params))
    assert np.array_equal(out[0][2], out[1][2])
    assert out[0][1] < 0.02 * out[0][0], out[0][:2]
    hist = net.loss_history(600)
    assert np.isfinite(hist).all() and hist[-50:].mean() < hist[:50].mean()


def test_wall_samples_match_fields(gpu):
    c = wallmodel.dns_boxes(retheta=(1100.0,), nx=40, nz=12)[0]
    s = cases.solver_for(c, precision=FP64, inflow=False)
    s.advance(2)
    net = WallNet()
    jh = wallmodel.rows_between(c, 0.05, 0.15)[0]
    net.sample(s, jh)
    X, T = net.data()
    U, V, W, P, _ = s.download_state()
    yg, xg = cases.centres_ghost(c.y), cases.centres_ghost(c.x)
    i = np.arange(2, c.nx)[None, :]
    k = np.arange(2, c.nz)[:, None]
    u = U[i - 1, jh - 1, k - 1]
    w = 0.25 * (W[i - 1, jh - 1, k - 1] + W[i, jh - 1, k - 1] + W[i - 1, jh - 1, k - 2] + W[i, jh - 1, k - 2])
    dp = (P[i, jh - 1, k - 1] - P[i - 1, jh - 1, k - 1]) / (xg[i] - xg[i - 1])
    h = yg[jh - 1]
    Xr = np.stack([u, w, np.log(np.maximum(h * np.abs(u) / c.nu, 1.0)) / 10.0, 100 * h * dp], -1).reshape(-1, 4)
    tx = c.nu * (U[i - 1, 1, k - 1] - U[i - 1, 0, k - 1]) / (yg[1] - yg[0])
    assert np.allclose(X, Xr, rtol=1e-6, atol=1e-7)
    assert np.allclose(T[:, 0], 1000 * tx.reshape(-1), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("mode", [1, 2])
def test_wall_model_step_matches_oracle(gpu, mode):
    c = wallmodel.wmles_case(nx=40, nz=16)
    c.cfl = -0.02
    net = WallNet(seed=7) if mode == 2 else None
    params = net.params.astype(np.float64) if net else None
    s = cases.solver_for(c, precision=FP64, les_model=1, inflow=False)
    s.set_wall_model(mode, 3, net)
    o = oracle.oracle_for(c)
    o.set_les(1)
    o.set_wall_model(mode, 3, params)
    for _ in range(3):
        s.time_step()
        o.step()
    U, V, W, _, _ = s.download_state()
    Ur, Vr, Wr, _, _ = o.state()
    tol = 1e-10 if mode == 1 else 1e-5
    assert rel(U, Ur) < tol and rel(V, Vr) < tol and rel(W, Wr) < tol, (rel(U, Ur), rel(V, Vr), rel(W, Wr))
    tx, _ = s.wall_stress()
    txo, _ = o.wall_stress()
    if mode == 1:
        assert np.abs(tx - txo).max() <= 1e-10 * np.abs(txo).max()
    else:  # FP32 sums in a different order may flip a BF16 rounding of an activation
        assert np.abs(tx - txo).max() <= 5e-3 * np.abs(txo).max() and rel(tx, txo) < 2e-4


def test_wall_model_errors(gpu):
    c = wallmodel.wmles_case(nx=40, nz=16)
    s = cases.solver_for(c, inflow=False)
    with pytest.raises(BlgpuError):
        s.set_wall_model(3, 3)
    with pytest.raises(BlgpuError):
        s.set_wall_model(2, 3, None)
    with pytest.raises(BlgpuError):
        s.set_wall_model(1, 0)
    with pytest.raises(BlgpuError):
        s.wall_stress()


def test_learned_wall_model_reproduces_equilibrium_cf(gpu):
    """Train on the solver's own wall-resolved boxes, then on a coarse
    wall-modelled grid: the network's mean Cf is within 2 % of the
    equilibrium law of the wall's, and the no-slip wall (the method without
    a wall model) misses it by far more."""
    net = WallNet(seed=11)
    n = wallmodel.generate_samples(net, wallmodel.dns_boxes())
    assert n == net.num_samples and n > 100000
    l0 = net.eval()
    wallmodel.train(net)
    assert net.eval() < 0.01 * l0
    c = wallmodel.wmles_case()
    # the two models on the same states
    s = cases.solver_for(c, precision=MIXED, les_model=1, inflow=False)
    s.set_wall_model(1, 3)
    cf_eq, cf_net = [], []
    for _ in range(20):
        s.advance(1)
        cf_eq.append(wallmodel.mean_cf(s.wall_stress()[0]))
        s.set_wall_model(2, 3, net)
        cf_net.append(wallmodel.mean_cf(s.wall_stress()[0]))
        s.set_wall_model(1, 3)
    err_same = abs(np.mean(cf_net[10:]) / np.mean(cf_eq[10:]) - 1)
    assert err_same < 0.02, err_same
    # runs with each model as the wall condition
    eq = wallmodel.run_cf(c, 1)
    learned = wallmodel.run_cf(c, 2, net)
    noslip = wallmodel.run_cf(c, 0)
    err = abs(learned / eq - 1)
    gain = abs(noslip / eq - 1)
    assert err < 0.02, (eq, learned)
    assert gain > 10 * err and gain > 0.2, (eq, noslip)
