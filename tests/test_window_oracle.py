"""The window-BA oracle (oracle/ba_oracle.c, float64 restatement of src/xclean/vio/window.py) against outputs of the
reference itself (tests/golden/window_golden.npz, made by tests/golden/make_golden_window.py).  CPU only.

build_system must agree bit for bit (same operation order); the 5-iteration solve to 1e-9 (the Cholesky and the
triangular solves are LAPACK's in the reference, a plain loop in the oracle, and the window's gauge is free)."""
import os

import numpy as np
import pytest

from oracle import ba_oracle as BO
from xclean_b200.backend.synth_ba import Window

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "window_golden.npz")
FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLD))


def _window(G, c):
    kw = {k: G["c%d_%s" % (c, k)].copy() for k in FIELDS}
    kw.update({k: float(v) for k, v in zip(SCAL, G["c%d_scal" % c])})
    return Window(**kw)


@pytest.mark.parametrize("c", [0, 1, 2])
def test_build_system_is_bit_exact(G, c):
    w = _window(G, c)
    H, b, cost, Hi, bl, Hlp, ok = BO.build_system(w, 1e-4)
    assert np.array_equal(ok, G["c%d_ok" % c])
    assert cost == G["c%d_cost" % c][0]
    for a, k in ((H, "H"), (b, "b"), (bl, "bl"), (Hi, "Hi"), (Hlp, "Hlp")):
        ref = G["c%d_%s" % (c, k)]
        if k in ("Hi", "Hlp", "bl"):        # per-landmark outputs are defined only where the landmark entered
            a, ref = a[ok], ref[ok]
        assert np.array_equal(a.view(np.uint64), ref.view(np.uint64)), k


@pytest.mark.parametrize("c", [0, 1, 2])
def test_solve_matches_the_reference(G, c):
    w = _window(G, c)
    st = BO.solve(w, iters=5, lam0=1e-4, hold=None)
    ref = G["c%d_stats" % c]
    np.testing.assert_allclose([st["cost0"], st["cost"]], ref[:2], rtol=1e-12)
    assert st["accepted"] == int(ref[2]) and st["lam"] == pytest.approx(ref[3], rel=1e-12)
    np.testing.assert_allclose(w.Rwb, G["c%d_Rwb_n" % c], rtol=0, atol=1e-9)
    np.testing.assert_allclose(w.pwb, G["c%d_pwb_n" % c], rtol=0, atol=1e-9)
    np.testing.assert_allclose(w.lmp, G["c%d_lmp_n" % c], rtol=1e-8, atol=1e-10)
