"""The pose-free landmark block of the window solve (src/xclean/vio/window.py:550-765) against outputs of the
reference itself (tests/golden/posefree_golden.npz, made by tests/golden/make_golden_posefree.py).  CPU only.

posefree_cost / posefree_step of the oracle agree bit for bit.  The batched solve carries the block as ordinary
landmarks with one host observation (xclean_b200.backend.ba.merge_posefree); the oracle's solve of that merged window
reproduces the reference's solve with the block attached to 1e-9 (the cost sum is associated differently and the
Cholesky is LAPACK's in the reference)."""
import os

import numpy as np
import pytest

from oracle import ba_oracle as BO
from xclean_b200.backend.ba import PoseFree, merge_posefree
from xclean_b200.backend.synth_ba import Window

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "posefree_golden.npz")
FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLD))


def window(G, c, pf_tag=None):
    kw = {k: G["c%d_%s" % (c, k)].copy() for k in FIELDS}
    kw.update({k: float(v) for k, v in zip(SCAL, G["c%d_scal" % c])})
    w = Window(**kw)
    if pf_tag:
        g = lambda k: G["c%d_%s_%s" % (c, pf_tag, k)]
        w.pf = PoseFree(g("host"), g("z"), float(g("isg")), g("rmeas"), g("ris"), g("lmp").copy())
    return w


def pf_args(G, c, w):
    g = lambda k: G["c%d_pf_%s" % (c, k)]
    return (w.Rwb, w.pwb, w.Rbc, w.pbc, g("lmp"), g("host"), g("rmeas"), g("ris"), g("z"), float(g("isg")))


@pytest.mark.parametrize("c", [0, 1])
def test_posefree_cost_and_step_bit_exact(G, c):
    w = window(G, c)
    a = pf_args(G, c, w)
    with np.errstate(all="ignore"):
        for behind in (0, 1):
            got = BO.posefree_cost(*a, w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k, behind)
            ref = G["c%d_cost_%d" % (c, behind)][0]
            assert np.array_equal(np.float64(got).view(np.uint64), np.float64(ref).view(np.uint64)), behind
        n = len(a[4])
        for tag, lam in (("d", 1e-3), ("u", 0.0)):
            lo, Hi, ok = np.full((n, 3), 7.0), np.full((n, 3, 3), 5.0), np.zeros(n, np.bool_)
            BO.posefree_step(*a, w.fx, w.fy, w.cx, w.cy, w.huber_k, lam, lo, Hi, ok)
            assert np.array_equal(ok, G["c%d_%s_ok" % (c, tag)])
            for x, k in ((lo, "lmp"), (Hi, "Hinv")):
                assert np.array_equal(x.view(np.uint64), G["c%d_%s_%s" % (c, tag, k)].view(np.uint64)), (tag, k)
    assert not ok.all() and ok.sum() > n // 2            # the degenerate landmarks are refused, the rest solved


@pytest.mark.parametrize("c", [0, 1])
def test_merged_solve_matches_the_reference(G, c):
    w = window(G, c, "pfs")
    m = merge_posefree(w)
    st = BO.solve(m, iters=5, lam0=1e-4, hold=None)
    ref = G["c%d_stats" % c]
    np.testing.assert_allclose([st["cost0"], st["cost"]], ref[:2], rtol=1e-12)
    assert st["accepted"] == int(ref[2]) and st["lam"] == pytest.approx(ref[3], rel=1e-12)
    L = w.lmp.shape[0]
    np.testing.assert_allclose(m.Rwb, G["c%d_Rwb_n" % c], rtol=0, atol=1e-9)
    np.testing.assert_allclose(m.pwb, G["c%d_pwb_n" % c], rtol=0, atol=1e-9)
    np.testing.assert_allclose(m.lmp[:L], G["c%d_lmp_n" % c], rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(m.lmp[L:], G["c%d_pflmp_n" % c], rtol=1e-8, atol=1e-10)


def test_posefree_argument_checks_without_a_device():
    """The device entry refuses a host slot outside the window and returns 0 for an empty block, before any device
    call."""
    from xclean_b200.backend import ba
    w = window(dict(np.load(GOLD)), 0)
    with pytest.raises(ValueError):
        ba.posefree_cost(w.Rwb, w.pwb, w.Rbc, w.pbc, np.zeros((1, 3)), np.array([99]), np.zeros(1), np.zeros(1),
                         np.zeros((1, 2)), 1.0, w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k, False)
    assert ba.posefree_cost(w.Rwb, w.pwb, w.Rbc, w.pbc, np.zeros((0, 3)), np.zeros(0, np.int64), np.zeros(0),
                            np.zeros(0), np.zeros((0, 2)), 1.0, w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k, False) == 0.0
    with pytest.raises(ValueError):
        ba.pack_windows([window(dict(np.load(GOLD)), 0, "pfs")][:0] + [_bad_host(window(dict(np.load(GOLD)), 0,
                                                                                         "pfs"))])


def _bad_host(w):
    w.pf.host = w.pf.host.copy()
    w.pf.host[0] = w.Rwb.shape[0]
    return w


def test_pack_windows_appends_the_posefree_block(G):
    """The packed batch carries each pose-free landmark after the window's own, with one observation (host slot, left
    camera, its pixel and whitening) and its prior; a window without a block packs as before."""
    from xclean_b200.backend.ba import pack_windows
    w = window(G, 1, "pfs")
    plain = window(G, 1)
    pk = pack_windows([w, plain], hold=None)
    L, M, n = plain.lmp.shape[0], int(plain.ob_start[-1]), len(w.pf.host)
    assert list(pk["L"]) == [L + n, L]
    lo = pk["lm_off"]
    assert np.array_equal(pk["lmp"][lo[0] + L:lo[0] + L + n], w.pf.lmp)
    assert np.array_equal(pk["lm_host"][lo[0] + L:lo[0] + L + n], w.pf.host)
    assert np.array_equal(pk["rho_isig"][lo[0] + L:lo[0] + L + n], w.pf.ris)
    ob = pk["lm_ob"]
    assert np.array_equal(np.diff(ob[lo[0] + L:lo[0] + L + n + 1]), np.ones(n))
    k0 = ob[lo[0] + L]
    assert k0 == M
    assert np.array_equal(pk["ob_pose"][k0:k0 + n], w.pf.host) and (pk["ob_cam"][k0:k0 + n] == 0).all()
    assert np.array_equal(pk["ob_z"][k0:k0 + n], w.pf.z) and (pk["ob_isig"][k0:k0 + n] == w.pf.isg).all()
    assert np.array_equal(pk["lmp"][lo[1]:lo[1] + L], plain.lmp)
