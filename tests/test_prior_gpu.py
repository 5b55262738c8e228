"""The window solve with a marginal prior over pose slots, on the device, against the reference's own window.solve and
final_linearisation with the same prior (tests/golden/prior_golden.npz, made by tests/golden/make_golden_prior.py from
src/xclean/vio/marg.py and window.py).

Tolerances as the other float64 window tests: the starting cost to 1e-9 relative, the accepted count exactly, the
final states to 1e-6 (the device sums in another order; the reference's Cholesky is LAPACK's); final_linearisation's
H and b to 1e-9 of their scale.  Mixed precision (slot 0 held, as the other mixed tests) against the float64 device
solve of the same windows: the first pose step to 1e-6 relative."""
import os

import numpy as np
import pytest

from xclean_b200.backend import marg as M
from xclean_b200.backend.synth_ba import Window

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prior_golden.npz")
FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLD))


def _window(G, c, with_prior=True):
    kw = {k: G["c%d_%s" % (c, k)].copy() for k in FIELDS}
    kw.update({k: float(v) for k, v in zip(SCAL, G["c%d_scal" % c])})
    w = Window(**kw)
    w.prior = None
    if with_prior:
        t = "c%d_prior" % c
        sids = [int(s) for s in G[t + "_sids"]]
        pr = M.Prior(sids, [6] * len(sids), [(R, p, None, None, None) for R, p in zip(G[t + "_R0"], G[t + "_p0"])],
                     G[t + "_S"], G[t + "_r"])
        pr.bind({s: s for s in range(w.Rwb.shape[0])})
        w.prior = pr
    return w


@pytest.mark.parametrize("c", [0, 1])
def test_solve_with_prior_matches_the_reference(G, c):
    from xclean_b200.backend import ba
    w = _window(G, c)
    st = ba.solve(w, iters=5, lam0=1e-4)
    ref = G["c%d_stats" % c]
    assert abs(st["cost0"] - ref[0]) <= 1e-9 * abs(ref[0])
    assert st["accepted"] == int(ref[2])
    assert abs(st["cost"] - ref[1]) <= 1e-7 * abs(ref[1])
    assert np.abs(w.Rwb - G["c%d_Rwb_n" % c]).max() < 1e-6
    assert np.abs(w.pwb - G["c%d_pwb_n" % c]).max() < 1e-6
    ln = G["c%d_lmp_n" % c]
    assert np.abs(w.lmp - ln).max() < 1e-5 * max(1.0, np.abs(ln).max())


@pytest.mark.parametrize("c", [0, 1])
def test_final_linearisation_with_prior(G, c):
    from xclean_b200.backend import ba
    w = _window(G, c)
    w.Rwb[:] = G["c%d_Rwb_n" % c]
    w.pwb[:] = G["c%d_pwb_n" % c]
    w.lmp[:] = G["c%d_lmp_n" % c]
    H, b, _chi, _ok, _Hi, imu, off = ba.final_linearisation(w)
    Hr, br = G["c%d_final_H" % c], G["c%d_final_b" % c]
    assert np.abs(H - Hr).max() <= 1e-9 * np.abs(Hr).max()
    assert np.abs(b - br).max() <= 1e-9 * max(np.abs(br).max(), 1.0)
    assert imu == [] and off[-1] == 6 * w.Rwb.shape[0]


def test_batch_mixed_with_priors_and_the_newton_refusal(G):
    import torch
    from xclean_b200 import _lib
    from xclean_b200.backend import ba
    ws64 = [_window(G, 0), _window(G, 1), _window(G, 0, with_prior=False)]
    wsm = [_window(G, 0), _window(G, 1), _window(G, 0, with_prior=False)]
    r64 = ba.solve_batch(ws64, iters=5, lam0=1e-4, precision="fp64", hold=0)
    rm = ba.solve_batch(wsm, iters=5, lam0=1e-4, precision="mixed", hold=0)
    for i in range(3):
        a, b = rm["dx0_list"][i], r64["dx0_list"][i]
        assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b), i
        assert rm["accepted"][i] == r64["accepted"][i]
        assert (rm["status"] == 0).all() and (r64["status"] == 0).all()
    # a prior moves the solution: the unprioured twin of window 0 ends elsewhere
    assert np.abs(ws64[0].pwb - ws64[2].pwb).max() > 1e-6
    # the exact-Newton / adjoint calls do not carry priors: they answer XCB_BA_STATUS_PRIOR for such windows
    bs = ba.BatchSolver([_window(G, 0), _window(G, 0, with_prior=False)], "cuda", hold=0)
    st = bs.newton(0)
    torch.cuda.synchronize()
    assert int(st[0, 3]) == _lib.XCB_BA_STATUS_PRIOR and int(st[1, 3]) == 0
