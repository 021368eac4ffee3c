"""Training and judging the learned wall-stress model.

Pipeline.  Wall-resolved boundary-layer boxes (the turbulent mean profile
at several Re_theta, first cell centre below y+ = 1, closed top) are made
divergence free and stepped by the solver; at a few early snapshots every
wall point of the rows between `lo` and `hi` (delta99 units) gives a sample
(u, w, ln(h|u|/nu)/10, 100 h dP/dx) -> 1000 (tau_x, tau_z), the stress of
the resolved wall gradient.  The WallNet is trained on those samples on the
GPU.  It is checked against the equilibrium law of the wall
(wallmodel.f90:1951-1985) on a coarse wall-modelled grid: the mean skin
friction 2 <tau_x> of the two models on the same states, and of runs that
use each model as the Neumann wall condition.  The same grid with the
no-slip wall shows what the model gains.
"""
import numpy as np

from . import cases
from ._lib import MIXED

# mean profiles whose log layer follows the equilibrium model's law
# u+ = ln(y+)/0.38 + 5.2, so the comparison is like with like
LOG_LAW = dict(kappa=cases.KAPPA_WM, C=cases.reichardt_c(cases.KAPPA_WM, cases.B_WM))


def closed_top(case):
    """The case with V_top = 0 (no transpiration through the top)."""
    U_in, V_in, W_in, U_top, V_top, W_top = case.bc
    case.bc = (U_in, V_in, W_in, U_top, np.zeros_like(V_top), W_top)
    return case


def dns_boxes(retheta=(700.0, 900.0, 1100.0, 1400.0, 1700.0, 2000.0, 2400.0), nx=64, ny=97, nz=16, seed=77):
    """Wall-resolved boxes (first cell centre below y+ = 1), 2 delta99 high."""
    return [closed_top(cases.turbulent_case(nx=nx, ny=ny, nz=nz, lx=nx * 0.125, ly=2.0, lz=nz * 0.0625,
                                            alpha=2.5, retheta=rt, seed=seed + q, lund=0, noise=0.0, **LOG_LAW))
            for q, rt in enumerate(retheta)]


def rows_between(case, lo, hi):
    """1-based centre rows j with lo <= yg(j) <= hi."""
    yg = cases.centres_ghost(case.y)
    return [j + 1 for j in range(1, case.ny) if lo <= yg[j] <= hi]


def generate_samples(net, boxes, snapshots=(0, 2, 4), lo=0.04, hi=0.16, precision=MIXED, device=0):
    """Append the wall samples of every box at the given step counts; returns
    the number of samples added."""
    n0 = net.num_samples
    for case in boxes:
        cases.project_initial(case, device=device)
        s = cases.solver_for(case, precision=precision, device=device, inflow=False)
        rows = rows_between(case, lo, hi)
        done = 0
        for snap in snapshots:
            if snap > done:
                s.advance(snap - done)
                done = snap
            for jh in rows:
                net.sample(s, jh)
        s.close()
    return net.num_samples - n0


def train(net, schedule=((2000, 2e-3), (1500, 5e-4), (1000, 1e-4)), batch=8192):
    """Adam with a step schedule; returns the loss of the last batch."""
    loss = None
    for steps, lr in schedule:
        loss = net.train(steps, batch=batch, lr=lr)
    return loss


def wmles_case(retheta=1100.0, nx=128, ny=33, nz=32, seed=5):
    """Coarse wall-modelled grid: nearly uniform y (dy = delta/16), so the
    reference's sampling row jref = 3 (yg(3) ~ 0.094 delta, y+ ~ 95 at
    Re_theta 1100) sits in the log layer and the first cell centre is at
    y+ ~ 30, far from resolving the wall."""
    return closed_top(cases.turbulent_case(nx=nx, ny=ny, nz=nz, lx=nx * 0.125, ly=2.0, lz=nz * 0.0625, alpha=0.05,
                                           retheta=retheta, seed=seed, lund=0, noise=0.05, **LOG_LAW))


def mean_cf(tau_x):
    """2 <tau_x> over the wall points (U_inf = 1)."""
    return 2.0 * float(np.mean(tau_x))


def resolved_cf(solver):
    """Skin friction of the resolved wall gradient (no wall model)."""
    U = solver.download_state()[0]
    yg = cases.centres_ghost(solver.y)
    tau = solver.cfg.nu * (U[1:-1, 1, 1:-2] - U[1:-1, 0, 1:-2]) / (yg[1] - yg[0])
    return 2.0 * float(np.mean(tau))


def run_cf(case, mode, net=None, jh=3, steps=40, precision=MIXED, device=0):
    """Wall-modelled LES (Smagorinsky) of `case` with wall model `mode`
    (0 no-slip, 1 law of the wall, 2 network); mean skin friction over the
    second half of the run."""
    s = cases.solver_for(case, precision=precision, device=device, les_model=1, inflow=False)
    if mode:
        s.set_wall_model(mode, jh, net)
    cfs = []
    for n in range(steps):
        s.advance(1)
        if n >= steps // 2:
            cfs.append(mean_cf(s.wall_stress()[0]) if mode else resolved_cf(s))
    s.close()
    return float(np.mean(cfs))
