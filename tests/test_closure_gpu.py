"""The learned wall-stress closure trained on the turbulent DNS recipe's own
data and assessed against the equilibrium law of the wall
(wallmodel.f90:1951-1985, Newton_solver.f90:13-79).

Data: the 814 x 257 x 193 turbulent box (10 % divergence-free noise, Lund
inflow), 300 steps past the noisy initial field, then 12 snapshots 25 steps
apart of every wall point of the row at h = 0.1 delta99 (812 x 191 points
each, about 1.86 M samples); the 2 snapshots after them are held out.

Measured on the held-out states against the resolved wall stress: the
network's mean Cf error and pointwise rms error, and the equilibrium law's
(evaluated at the same row on the same states).  The gain over the method
without the network is the ratio of those errors.  Then both models drive
the wall of the 512 x 96 x 256 wall-modelled LES (Smagorinsky, LES = 1), and
the runs' mean Cf are compared.

The training DNS is not in equilibrium: over the steps this noisy field can
be run its near-wall region relaxes and its Cf falls about 30 % below the
log-law value the equilibrium model returns at h, so the network (which
learns the DNS) and the equilibrium law differ by about that much in the LES;
the test states the numbers and checks the network against the DNS."""
import numpy as np
import pytest

from blgpu import cases, wallmodel, WallNet

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def test_closure_from_dns_data(gpu):
    net, hold = WallNet(seed=11), WallNet(seed=12)
    info = wallmodel.config2_training(net, hold)
    assert info["samples"] == 12 * 812 * 191 and info["held_samples"] == 2 * 812 * 191
    l0 = net.eval()
    wallmodel.train(net)
    l1 = net.eval()
    e = wallmodel.holdout_errors(net, hold, info["tau_eq"])
    c = wallmodel.config4_case()
    jh = wallmodel.row_at(c, 0.1)
    cf_eq = wallmodel.run_cf(c, 1, jh=jh, steps=200)
    cf_net = wallmodel.run_cf(c, 2, net, jh=jh, steps=200)
    print("closure: %d samples from %d DNS steps (row %d, h = %.4f); loss %.3f -> %.3f" %
          (info["samples"], info["steps"], info["jh"], info["h"], l0, l1))
    print("held out vs resolved DNS: Cf %.5f, network %.5f (err %.3f), equilibrium %.5f (err %.3f); "
          "rms network %.3e, equilibrium %.3e" % (e["cf_dns"], e["cf_net"], e["cf_err_net"], e["cf_eq"],
                                                   e["cf_err_eq"], e["rms_net"], e["rms_eq"]))
    print("512x96x256 WMLES, wall at row %d: Cf equilibrium %.5f, network %.5f (ratio %.3f)" %
          (jh, cf_eq, cf_net, cf_net / cf_eq))
    assert l1 < l0
    # the network reproduces the DNS's wall stress better than the equilibrium law
    assert e["cf_err_net"] < 0.5 * e["cf_err_eq"]
    assert e["rms_net"] < e["rms_eq"]
    assert np.isfinite(cf_eq) and np.isfinite(cf_net) and cf_eq > 0 and cf_net > 0
