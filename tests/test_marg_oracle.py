"""The marginal prior's host algebra (xclean_b200.backend.marg) against the reference's own outputs
(tests/golden/prior_golden.npz, made by tests/golden/make_golden_prior.py from src/xclean/vio/marg.py and window.py).

The square-root factor S of a prior is defined only up to the sign of each row (eigenvectors), so the comparisons are
on the sign-free quantities S^T S, S^T r, the kept rank, and everything computed from them; tolerance 1e-9 relative
(float64, the same LAPACK on both sides)."""
import os

import numpy as np
import pytest

from xclean_b200.backend import marg as M

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prior_golden.npz")


@pytest.fixture(scope="module")
def z():
    return np.load(GOLD)


def _close(a, b, tol=1e-9):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert a.shape == b.shape
    assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max()), np.abs(a - b).max()


def _prior(z, tag):
    sids = [int(s) for s in z[tag + "_sids"]]
    x0 = [(R, p, None, None, None) for R, p in zip(z[tag + "_R0"], z[tag + "_p0"])]
    return M.Prior(sids, [6] * len(sids), x0, z[tag + "_S"], z[tag + "_r"])


def _same_prior(a, b):
    assert a.sids == b.sids and a.S.shape == b.S.shape
    _close(a.S.T @ a.S, b.S.T @ b.S)
    _close(a.S.T @ a.r, b.S.T @ b.r)
    for (Ra, pa, *_), (Rb, pb, *_) in zip(a.x0, b.x0):
        _close(Ra, Rb, 0.0)
        _close(pa, pb, 0.0)


@pytest.mark.parametrize("ci", [0, 1])
def test_schur_and_combine_make_the_reference_prior(z, ci):
    c = "c%d" % ci
    K = z[c + "_Rwb"].shape[0]
    H2, b2 = M.schur(z[c + "_marg_H"], z[c + "_marg_b"], np.arange(6, 6 * K), np.arange(6))
    _close(H2, z[c + "_schur_H"])
    _close(b2, z[c + "_schur_b"])
    sids = list(range(1, K))
    R, p = z[c + "_solved_Rwb"], z[c + "_solved_pwb"]
    pr = M.combine(None, sids, [6] * len(sids), [(R[s], p[s], None, None, None) for s in sids], H2, b2)
    g = M.gauge_prior(1, R[1], p[1], info=1e8)
    Hc, bc = pr.info()
    Hg, bg = g.info()
    Hc[:6, :6] += Hg
    bc[:6] += bg
    pr = M.Prior.from_info(pr.sids, pr.dims, pr.x0, Hc, bc)
    _same_prior(pr, _prior(z, c + "_prior"))


@pytest.mark.parametrize("ci", [0, 1])
def test_terms_cost_drop_and_refold(z, ci):
    c = "c%d" % ci
    K = z[c + "_Rwb"].shape[0]
    pr = _prior(z, c + "_prior")
    pr.bind({s: s for s in range(K)})
    st = (z[c + "_moved_Rwb"], z[c + "_moved_pwb"], None, None, None)
    H, b, cost = pr.terms(st, 6 * K)
    _close(H, z[c + "_terms_H"])
    _close(b, z[c + "_terms_b"])
    _close([cost, pr.cost(st)], z[c + "_terms_cost"])
    _same_prior(pr.drop_slot(pr.sids[0]), _prior(z, c + "_drop"))
    sids = pr.sids
    cb = M.combine(pr, sids, [6] * len(sids), [(st[0][s], st[1][s], None, None, None) for s in sids],
                   z[c + "_combine_H"], z[c + "_combine_b"])
    _same_prior(cb, _prior(z, c + "_comb"))


def test_pose_blocks_only_and_log_branches():
    with pytest.raises(NotImplementedError):
        M.Prior([0], [15], [(np.eye(3), np.zeros(3), None, None, None)], np.eye(15), np.zeros(15))
    from xclean_b200.backend.synth_ba import so3_exp
    for w in (np.array([1e-8, -2e-8, 3e-9]), np.array([0.3, -0.2, 0.1]), np.array([np.pi - 2e-5, 0.0, 0.0]),
              np.array([0.0, -(np.pi - 3e-5), 0.0])):
        got = M.so3_log(so3_exp(w))
        assert np.abs(got - w).max() < 1e-7, (w, got)
