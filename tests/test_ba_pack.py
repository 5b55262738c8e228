"""The host packing of the batched window solve (xclean_b200/backend/ba.py) on the CPU: pack_windows' batch layout
(the xcb_ba_windows arrays: per-window slot / landmark / observation offsets, the concatenated state and
observations, the largest-first work order), its refusals (the kernel's per-window and per-landmark limits, slots
outside the window), and the marginal-prior layout (_prior_slots, _pack_priors: a bound marg.Prior's 6-dim pose
blocks, src/xclean/vio/marg.py:57-213) with its refusals."""
from types import SimpleNamespace

import numpy as np
import pytest

from xclean_b200.backend import ba as B


def _windows():
    from xclean_b200.backend import synth_ba as S
    return [S.make_window(None, K=k, L=l, obs_min=2, obs_max=4, rng=np.random.default_rng(s))
            for k, l, s in ((3, 10, 1), (6, 25, 2), (4, 7, 3))]


def _tiny(P, obs_pose, lm_host=0):
    """One landmark observed in the left image of the slots `obs_pose` (one row each)."""
    n = len(obs_pose)
    return SimpleNamespace(
        Rwb=np.tile(np.eye(3), (P, 1, 1)), pwb=np.zeros((P, 3)), Rbc=np.eye(3), pbc=np.zeros(3), fx=400.0, fy=400.0,
        cx=300.0, cy=200.0, B=0.1, huber_k=1.345, lmp=np.array([[0.0, 0.0, 0.2]]), lm_host=np.array([lm_host]),
        lm_mask=np.array([True]), rho_meas=np.zeros(1), rho_isig=np.zeros(1), ob_start=np.array([0, n]),
        ob_pose=np.asarray(obs_pose, np.int64), ob_cam=np.zeros(n, np.int64), ob_z=np.zeros((n, 2)),
        ob_isig=np.ones(n), ob_valid=np.ones(n, bool))


def test_batch_layout():
    ws = _windows()
    pk = B.pack_windows(ws, hold=0)
    P = [w.Rwb.shape[0] for w in ws]
    L = [w.lmp.shape[0] for w in ws]
    M = [w.ob_pose.shape[0] for w in ws]
    assert pk["nw"] == 3 and pk["max_slots"] == max(P)
    assert pk["P"].tolist() == P and pk["L"].tolist() == L
    assert pk["slot_off"].tolist() == [0, P[0], P[0] + P[1]]
    assert pk["lm_off"].tolist() == [0, L[0], L[0] + L[1]]
    assert pk["hold"].tolist() == [0, 0, 0]
    assert B.pack_windows(ws, hold=None)["hold"].tolist() == [-1, -1, -1]
    ob0 = np.concatenate([[0], np.cumsum(M)])
    assert pk["lm_ob"].shape == (sum(L) + 1,) and pk["lm_ob"][-1] == sum(M)
    for i, w in enumerate(ws):
        so, lo = pk["slot_off"][i], pk["lm_off"][i]
        assert np.array_equal(pk["Rwb"][so:so + P[i]], w.Rwb.reshape(-1, 9))
        assert np.array_equal(pk["pwb"][so:so + P[i]], w.pwb)
        assert np.array_equal(pk["lmp"][lo:lo + L[i]], w.lmp)
        assert np.array_equal(pk["lm_host"][lo:lo + L[i]], w.lm_host)
        assert np.array_equal(pk["lm_ob"][lo:lo + L[i]], np.asarray(w.ob_start[:-1]) + ob0[i])
        assert np.array_equal(pk["ob_pose"][ob0[i]:ob0[i + 1]], w.ob_pose)
        assert np.array_equal(pk["ob_z"][ob0[i]:ob0[i + 1]], w.ob_z)
        assert np.array_equal(pk["cam"][i], [w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k])
        assert np.array_equal(pk["ext"][i], np.concatenate([np.ravel(w.Rbc), np.ravel(w.pbc)]))
    work = np.array(P, np.int64) ** 2 * 36 + np.array(M, np.int64) * 64
    assert sorted(pk["order"].tolist()) == [0, 1, 2]
    assert (np.diff(work[pk["order"]]) <= 0).all()
    assert not any(k.startswith("pr_") for k in pk)


def test_batch_refusals():
    with pytest.raises(ValueError, match="slots"):
        B.pack_windows([_tiny(B.MAX_SLOTS + 1, [0, 1])])
    with pytest.raises(ValueError, match="outside"):
        B.pack_windows([_tiny(3, [0, 1], lm_host=3)])
    with pytest.raises(ValueError, match="outside"):
        B.pack_windows([_tiny(3, [0, -1])])
    with pytest.raises(ValueError, match="observation rows"):
        B.pack_windows([_tiny(2, [0, 1] * ((B.MAX_ROWS_PER_LANDMARK + 2) // 2))])
    with pytest.raises(ValueError, match="touches"):
        B.pack_windows([_tiny(B.MAX_TOUCHED_SLOTS + 2, list(range(1, B.MAX_TOUCHED_SLOTS + 2)))])
    # at the limits: accepted
    B.pack_windows([_tiny(B.MAX_SLOTS, [0, 1])])
    B.pack_windows([_tiny(B.MAX_TOUCHED_SLOTS, list(range(B.MAX_TOUCHED_SLOTS)))])


def _prior(slots, rows=None, dims=6, bound=True):
    nb = len(slots)
    cols = np.concatenate([6 * s + np.arange(6) for s in slots]) if bound else None
    m = 6 * nb if rows is None else rows
    rng = np.random.default_rng(len(slots))
    return SimpleNamespace(dims=[dims] * nb, cols=cols, S=rng.normal(size=(m, 6 * nb)), r=rng.normal(size=m),
                           x0=[(np.eye(3) * (k + 1), np.arange(3.0) + k) for k in range(nb)])


def test_prior_slots_and_refusals():
    assert B._prior_slots(_prior([2, 0]), 4).tolist() == [2, 0]
    with pytest.raises(ValueError, match="not a marginal prior"):
        B._prior_slots(SimpleNamespace(S=np.zeros((6, 6))), 4)
    with pytest.raises(ValueError, match="not bound"):
        B._prior_slots(_prior([0], bound=False), 4)
    with pytest.raises(NotImplementedError):
        B._prior_slots(_prior([0], dims=15), 4)
    half = _prior([1])
    half.cols = half.cols + 3
    with pytest.raises(ValueError, match="whole pose slot"):
        B._prior_slots(half, 4)
    with pytest.raises(ValueError, match="distinct slots"):
        B._prior_slots(_prior([1, 1]), 4)
    with pytest.raises(ValueError, match="distinct slots"):
        B._prior_slots(_prior([4]), 4)


def test_prior_layout():
    P = np.array([4, 3, 5], np.int32)
    wins = [SimpleNamespace(prior=_prior([2, 0], rows=9)), SimpleNamespace(prior=None),
            SimpleNamespace(prior=_prior([4]))]
    pr = B._pack_priors(wins, P)
    assert pr["pr_m"].tolist() == [9, 0, 6] and pr["pr_nb"].tolist() == [2, 0, 1]
    assert pr["pr_boff"].tolist() == [0, 2, 2]
    assert pr["pr_soff"].tolist() == [0, 9 * 12, 9 * 12]
    assert pr["pr_roff"].tolist() == [0, 9, 9]
    assert pr["pr_blk"].tolist() == [2, 0, 4]
    assert pr["pr_x0"].shape == (3, 12)
    assert np.array_equal(pr["pr_x0"][1], np.concatenate([np.ravel(np.eye(3) * 2), np.arange(3.0) + 1]))
    assert np.array_equal(pr["pr_S"], np.concatenate([wins[0].prior.S.ravel(), wins[2].prior.S.ravel()]))
    assert np.array_equal(pr["pr_r"], np.concatenate([wins[0].prior.r, wins[2].prior.r]))
    assert B._pack_priors([SimpleNamespace(prior=None)], P[:1]) == {}
    with pytest.raises(ValueError, match="more rows than columns"):
        B._pack_priors([SimpleNamespace(prior=_prior([0], rows=7))], P[:1])
