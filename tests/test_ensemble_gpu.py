"""Ensembles of uneven boxes advanced by one CUDA-graph launch per step, the
sequential baseline, launch shapes (tiles) and their autotuner.  Tiles and
concurrency change speed only: every comparison here is bit-exact."""
import numpy as np
import pytest

from blgpu import cases, FP64, MIXED, BlgpuError, Ensemble

pytestmark = pytest.mark.gpu


def small_boxes(n=4, seed=11):
    shapes = [(40, 17, 18), (56, 17, 24), (40, 17, 24), (72, 17, 18)]
    out = []
    for b in range(n):
        nx, ny, nz = shapes[b % len(shapes)]
        out.append(cases.turbulent_case(nx=nx, ny=ny, nz=nz, lx=nx * 0.12, ly=4.0, lz=nz * 0.04,
                                        retheta=900.0 + 100 * b, seed=seed + b))
    return out


def states(solvers):
    return [s.download_state()[:3] for s in solvers]


def same(a, b):
    return all(np.array_equal(x, y) for p, q in zip(a, b) for x, y in zip(p, q))


@pytest.mark.parametrize("precision", [MIXED, FP64])
def test_ensemble_equals_individual_boxes(gpu, precision):
    cs = small_boxes()
    ref = [cases.solver_for(c, precision=precision) for c in cs]
    nl = 0
    for s in ref:
        l0 = s.kernel_launches()
        s.advance(4)
        nl += s.kernel_launches() - l0
    box = [cases.solver_for(c, precision=precision) for c in cs]
    ens = Ensemble(box)
    ens.advance(4)
    ens.sync()
    assert same(states(ref), states(box))
    assert ens.launches() == nl
    ens.close()


def test_sequential_baseline_equals_concurrent(gpu):
    cs = small_boxes(seed=12)
    a = [cases.solver_for(c, precision=MIXED) for c in cs]
    b = [cases.solver_for(c, precision=MIXED) for c in cs]
    ea, eb = Ensemble(a), Ensemble(b)
    ea.advance(3)
    eb.advance_sequential(3)
    ea.sync()
    eb.sync()
    assert same(states(a), states(b))
    t_conc = ea.time(2)
    t_seq = eb.time(2, sequential=True)
    assert t_conc > 0 and t_seq > 0
    ea.close()
    eb.close()


@pytest.mark.parametrize("precision", [MIXED, FP64])
def test_tiles_do_not_change_results(gpu, precision):
    c = small_boxes(1, seed=13)[0]
    s0 = cases.solver_for(c, precision=precision)
    s0.advance(3)
    kc = 16 if precision == MIXED else 4
    s1 = cases.solver_for(c, precision=precision)
    s1.set_tiles(rhs_kc=kc, rhs_by=4, dct_nw=2, dftz_rk=4, proj_by=4, idct_nw=3)
    assert s1.tiles() == dict(rhs_kc=kc, rhs_by=4, dct_nw=2, dftz_rk=4, proj_by=4, zdft=0, rhs_pts=0, thomas=0,
                              idct_nw=3, xfft=0)
    s1.advance(3)
    assert same(states([s0]), states([s1]))


def test_autotune_restores_state_and_keeps_results(gpu):
    c = small_boxes(1, seed=14)[0]
    s = cases.solver_for(c, precision=MIXED)
    s.advance(2)
    before = states([s])
    t0, t1 = s.autotune(steps=2)
    assert t0 > 0 and 0 < t1 <= t0
    assert same(before, states([s]))
    ref = cases.solver_for(c, precision=MIXED)
    ref.advance(2)  # the built-in tiles, as s before tuning
    # the z-transform, RHS-form, x-transform and y-solve choices are the knobs that move roundings
    ref.set_tiles(zdft=s.tiles()["zdft"], rhs_pts=s.tiles()["rhs_pts"], xfft=s.tiles()["xfft"],
                  thomas=s.tiles()["thomas"])
    s.advance(3)
    ref.advance(3)
    assert same(states([ref]), states([s]))


def test_ensemble_autotune_shares_tiles_by_shape(gpu):
    cs = small_boxes(4, seed=15) + small_boxes(2, seed=16)
    box = [cases.solver_for(c, precision=MIXED) for c in cs]
    ens = Ensemble(box)
    n = ens.autotune(steps=1)
    assert n == 4
    assert box[4].tiles() == box[0].tiles() and box[5].tiles() == box[1].tiles()
    ens.advance(2)
    ens.close()


def test_ensemble_errors(gpu):
    cs = small_boxes(2, seed=17)
    box = [cases.solver_for(c, precision=MIXED) for c in cs]
    with pytest.raises(BlgpuError):
        Ensemble([box[0], box[0]])
    ens = Ensemble(box)
    box[0].advance(1)  # rotations now differ
    with pytest.raises(BlgpuError):
        ens.advance(1)
    ens.close()
    with pytest.raises(BlgpuError):
        box[1].set_tiles(dftz_rk=5)
    with pytest.raises(BlgpuError):
        box[1].set_tiles(rhs_by=3)
