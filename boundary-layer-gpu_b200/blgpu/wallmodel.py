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


def row_at(case, h):
    """1-based centre row whose yg is closest to h (delta99 units)"""
    yg = cases.centres_ghost(case.y)
    return int(np.argmin(np.abs(yg[1:-1] - h))) + 2


def config2_training(net, holdout, h=0.1, spinup=300, snaps=12, every=25, held=2, dt=0.012, precision=MIXED,
                     device=0, **case_kw):
    """Training data from the turbulent DNS recipe (814 x 257 x 193 by default:
    composite mean profile with the equilibrium law's log layer, 10 % U_inf
    divergence-free noise, Lund inflow), run `spinup` steps past the noisy
    initial field and then sampled every `every` steps: `snaps` snapshots of
    every wall point of the row at h = 0.1 delta go to `net`'s training set,
    the `held` snapshots after them to `holdout` (never trained on), together
    with the equilibrium model's stress at the same row on those states.
    The steps use a fixed dt (delta99 / U_inf units): compute_dt's CFL mode
    takes the largest spacing/|u| (time_integration.f90:546-558), so at
    CFL 0.5 its dt is the viscous limit and this noisy field breaks up after
    about 130 steps; 0.012 keeps the convective CFL below about 0.5.
    Returns a dict: jh, steps run, samples, and the held-out equilibrium
    stresses tau_eq (flattened in the sample order)."""
    case = cases.turbulent_case(noise=0.10, cfl=-dt, **LOG_LAW, **case_kw)
    cases.project_initial(case, device=device)
    s = cases.solver_for(case, precision=precision, device=device)
    jh = row_at(case, h)
    s.advance(spinup)
    n0 = net.num_samples
    for _ in range(snaps):
        s.advance(every)
        net.sample(s, jh)
    tau_eq = []
    for _ in range(held):
        s.advance(every)
        holdout.sample(s, jh)
        s.set_wall_model(1, jh)  # the equilibrium law on this state (no step taken)
        tau_eq.append(s.wall_stress()[0].ravel())
        s.set_wall_model(0, jh)
    s.close()
    return dict(jh=jh, h=float(cases.centres_ghost(case.y)[jh - 1]), steps=spinup + (snaps + held) * every,
                samples=net.num_samples - n0, held_samples=holdout.num_samples, tau_eq=np.concatenate(tau_eq),
                grid=(case.nx, case.ny, case.nz))


def holdout_errors(net, holdout, tau_eq):
    """The network and the equilibrium model against the resolved wall stress
    of the held-out states: rms pointwise error, mean Cf and their errors."""
    X, T = holdout.data()
    tau = T[:, 0].astype(np.float64) / 1000.0
    tau_net = net.forward(X)[:, 0].astype(np.float64) / 1000.0
    rms = lambda a: float(np.sqrt(np.mean((a - tau) ** 2)))
    cf, cf_net, cf_eq = mean_cf(tau), mean_cf(tau_net), mean_cf(tau_eq)
    return dict(cf_dns=cf, cf_net=cf_net, cf_eq=cf_eq, rms_net=rms(tau_net), rms_eq=rms(tau_eq),
                cf_err_net=abs(cf_net / cf - 1.0), cf_err_eq=abs(cf_eq / cf - 1.0))


def config4_case(retheta=2000.0, nx=512, ny=96, nz=256, seed=5, dt=0.04):
    """The wall-modelled LES grid the closure is assessed on: 512 x 96 x 256 over
    64 x 2 x 16 delta99, nearly uniform y (dy = delta/48), so h = 0.1 delta is
    the sixth row and the first cell centre sits at y+ ~ 7 (Re_theta 2000),
    far from resolving the wall gradient.  Fixed dt = 0.04 delta99/U_inf
    (convective CFL about 0.35 in x): compute_dt's CFL mode would take the
    viscous limit, about 4 on this grid."""
    c = wmles_case(retheta=retheta, nx=nx, ny=ny, nz=nz, seed=seed)
    c.cfl = -dt
    return c
