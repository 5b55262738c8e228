"""The pose-free landmark block on the device: window.posefree_cost / posefree_step bit for bit against the
reference's outputs, and the batched window solve with the block attached against the reference's solve
(tests/golden/posefree_golden.npz).  Tolerances of the solve as for the windows without a block: the first cost to
1e-9 relative, the accepted count identical, the states to 1e-6 (float64 mode; atomics change the summation order)."""
import numpy as np
import pytest

from oracle import ba_oracle as BO
from tests.test_posefree_oracle import GOLD, pf_args, window

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLD))


@pytest.mark.parametrize("c", [0, 1])
def test_posefree_cost_and_step_bit_exact(G, c):
    from xclean_b200.backend import ba
    w = window(G, c)
    a = pf_args(G, c, w)
    for behind in (False, True):
        got = ba.posefree_cost(*a, w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k, behind)
        ref = G["c%d_cost_%d" % (c, int(behind))][0]
        assert np.array_equal(np.float64(got).view(np.uint64), np.float64(ref).view(np.uint64)), behind
    n = len(a[4])
    for tag, lam in (("d", 1e-3), ("u", 0.0)):
        lo, Hi, ok = np.full((n, 3), 7.0), np.full((n, 3, 3), 5.0), np.zeros(n, np.bool_)
        assert ba.posefree_step(*a, w.fx, w.fy, w.cx, w.cy, w.huber_k, lam, lo, Hi, ok) == 0
        assert np.array_equal(ok, G["c%d_%s_ok" % (c, tag)])
        for x, k in ((lo, "lmp"), (Hi, "Hinv")):
            assert np.array_equal(x.view(np.uint64), G["c%d_%s_%s" % (c, tag, k)].view(np.uint64)), (tag, k)


def test_batched_solve_with_posefree_block(G, precision="fp64", tol=1e-6):
    """Both fixture windows with their pose-free blocks and one window without, in one float64 batch with the gauge
    free (as the reference solves them): every window as the reference's solve leaves it; then final_linearisation's
    pose-free marginals at the solution equal the oracle's."""
    from xclean_b200.backend import ba
    ws = [window(G, 0, "pfs"), window(G, 1, "pfs"), window(G, 1)]
    plain_ref = BO.solve(window(G, 1), iters=5, lam0=1e-4, hold=None)
    res = ba.solve_batch(ws, iters=5, lam0=1e-4, precision=precision, hold=None)
    for i, c in enumerate((0, 1)):
        ref = G["c%d_stats" % c]
        w = ws[i]
        assert res["status"][i] == 0
        assert abs(res["cost0"][i] - ref[0]) <= 1e-9 * abs(ref[0])
        assert res["accepted"][i] == int(ref[2])
        assert np.abs(w.Rwb - G["c%d_Rwb_n" % c]).max() < tol and np.abs(w.pwb - G["c%d_pwb_n" % c]).max() < tol
        for got, k in ((w.lmp, "lmp_n"), (w.pf.lmp, "pflmp_n")):
            r = G["c%d_%s" % (c, k)]
            assert np.abs(got - r).max() < 10 * tol * max(1.0, np.abs(r).max()), k
        ba.posefree_marginals(w)
        pf = w.pf
        n = len(pf.host)
        lo, Hi, ok = np.zeros((n, 3)), np.zeros((n, 3, 3)), np.zeros(n, np.bool_)
        BO.posefree_step(w.Rwb, w.pwb, w.Rbc, w.pbc, pf.lmp, pf.host, pf.rmeas, pf.ris, pf.z, pf.isg, w.fx, w.fy,
                         w.cx, w.cy, w.huber_k, 0.0, lo, Hi, ok)
        assert np.array_equal(pf.ok, ok) and np.array_equal(pf.Hinv[ok], Hi[ok])
    assert res["accepted"][2] == plain_ref["accepted"]
    assert abs(res["cost0"][2] - plain_ref["cost0"]) <= 1e-9 * abs(plain_ref["cost0"])


def test_mixed_solve_with_posefree_block(G):
    """Mixed precision (its step target assumes a fixed gauge: slot 0 held, as the other mixed-precision tests) with
    the blocks attached, against the oracle's float64 solve of the merged windows: the first pose step to 1e-6
    relative, the same accepted count, the states to 1e-6."""
    from xclean_b200.backend import ba
    ws = [window(G, 0, "pfs"), window(G, 1, "pfs")]
    refs = [ba.merge_posefree(window(G, c, "pfs")) for c in (0, 1)]
    outs = [BO.solve(r, iters=5, lam0=1e-4, hold=0) for r in refs]
    res = ba.solve_batch(ws, iters=5, lam0=1e-4, precision="mixed", hold=0)
    for i, (w, r, o) in enumerate(zip(ws, refs, outs)):
        dx = res["dx0_list"][i]
        assert np.linalg.norm(dx - o["dx0"]) <= 1e-6 * np.linalg.norm(o["dx0"]), i
        assert res["accepted"][i] == o["accepted"], i
        assert np.abs(w.pwb - r.pwb).max() < 1e-6 and np.abs(w.Rwb - r.Rwb).max() < 1e-6
        L = w.lmp.shape[0]
        assert np.abs(w.pf.lmp - r.lmp[L:]).max() < 1e-5 * max(1.0, np.abs(r.lmp[L:]).max())


def test_final_linearisation_systems(G):
    """final_linearisation's visual outputs (lam = 0) from the batched kernel against the oracle's build_system (which
    the reference pins bit for bit): H, b and the kept landmarks' Hll_inv to 1e-9 of their scale, lm_ok exactly, the
    observations' chi2 to 1e-9 (inf at the same rows), the cost to 1e-12; a window's pose-free block leaves its system
    unchanged (no pose coupling) and gets its marginals."""
    from tests.test_window_oracle import GOLD as WGOLD, _window as wwindow
    from xclean_b200.backend import ba
    WG = dict(np.load(WGOLD))
    ws = [wwindow(WG, c) for c in (0, 1, 2)] + [window(G, 1, "pfs"), window(G, 1)]
    systems, cost = ba.final_linearisation_batch(ws)
    for i, w in enumerate(ws):
        ref = w if getattr(w, "pf", None) is None else window(G, 1)
        H, b, c, Hi, _bl, _Hlp, ok, chi = BO.build_system(ref, 0.0, want_chi2=True)
        sy = systems[i]
        Hd, bd = sy["H"], sy["b"]
        assert Hd.shape == H.shape and bd.shape == b.shape
        assert np.abs(Hd - H).max() <= 1e-9 * np.abs(H).max(), i
        assert np.abs(bd - b).max() <= 1e-9 * np.abs(b).max(), i
        assert np.array_equal(sy["lm_ok"], ok), i
        assert np.abs(sy["Hll_inv"][ok] - Hi[ok]).max() <= 1e-9 * np.abs(Hi[ok]).max(), i
        assert (sy["Hll_inv"][~ok] == 0).all()
        fin = np.isfinite(chi)
        assert np.array_equal(np.isfinite(sy["ob_chi2"]), fin), i
        assert np.allclose(sy["ob_chi2"][fin], chi[fin], rtol=1e-9, atol=1e-12), i
        if getattr(w, "pf", None) is None:
            assert abs(cost[i] - c) <= 1e-12 * abs(c), i
    pf = ws[3].pf
    n = len(pf.host)
    lo, Hi, ok = np.zeros((n, 3)), np.zeros((n, 3, 3)), np.zeros(n, np.bool_)
    w = ws[3]
    BO.posefree_step(w.Rwb, w.pwb, w.Rbc, w.pbc, pf.lmp, pf.host, pf.rmeas, pf.ris, pf.z, pf.isg, w.fx, w.fy, w.cx,
                     w.cy, w.huber_k, 0.0, lo, Hi, ok)
    assert np.array_equal(pf.ok, ok) and np.array_equal(pf.Hinv[ok], Hi[ok])
    assert cost[3] > cost[4]                             # the block's cost joins the window's


def test_marg_system(G):
    """window.marg_system: the masked landmarks' reduced system against the oracle's build_system with that mask
    (lam = 0), H and b to 1e-9 of their scale; the offsets are 6 per slot."""
    from xclean_b200.backend import ba
    w = window(G, 1, "pfs")
    rng = np.random.default_rng(4)
    mask = rng.random(w.lmp.shape[0]) < 0.3
    (H, b, off), = ba.marg_system_batch([w], [mask])
    ref = window(G, 1)
    ref.lm_mask = mask
    Hr, br = BO.build_system(ref, 0.0)[:2]
    assert np.abs(H - Hr).max() <= 1e-9 * np.abs(Hr).max() and np.abs(b - br).max() <= 1e-9 * np.abs(br).max()
    assert np.array_equal(off, np.arange(w.Rwb.shape[0] + 1) * 6)


def test_single_window_signatures(G):
    """window.solve / final_linearisation / marg_system with the reference's signatures and return shapes: solve
    equals the reference's solve with the block attached (float64, free gauge) and returns its stats dict; the
    linearisation tuple matches the batched outputs; a prior or IMU terms are refused."""
    from xclean_b200.backend import ba
    w = window(G, 1, "pfs")
    st = ba.solve(w, iters=5, lam0=1e-4)
    ref = G["c1_stats"]
    assert set(st) == {"cost0", "cost", "accepted", "iters", "lam"} and st["accepted"] == int(ref[2])
    assert abs(st["cost0"] - ref[0]) <= 1e-9 * abs(ref[0])
    assert np.abs(w.pwb - G["c1_pwb_n"]).max() < 1e-6
    H, b, chi2, ok, Hi, imu, off = ba.final_linearisation(w)
    (sy,), _c = ba.final_linearisation_batch([w])
    # two linearisations agree to rounding (the reduced system is accumulated by atomics in any order)
    assert np.abs(H - sy["H"]).max() <= 1e-12 * np.abs(H).max()
    assert np.array_equal(chi2, sy["ob_chi2"]) and np.array_equal(ok, sy["lm_ok"])
    assert imu == [] and np.array_equal(off, np.arange(w.Rwb.shape[0] + 1) * 6) and w.pf.ok.any()
    Hm, bm, offm = ba.marg_system(w, np.asarray(w.lm_mask, np.bool_))      # the window's own mask: its H again
    assert np.allclose(Hm, H, rtol=0, atol=1e-9 * np.abs(H).max())
    w.prior = object()                    # not a marg.Prior (bound priors are solved: tests/test_prior_gpu.py)
    with pytest.raises(ValueError):
        ba.solve(w)
