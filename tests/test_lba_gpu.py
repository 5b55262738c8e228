"""Local BA on the device: the stage kernels of src/xclean/backend/kernels.py and the solvers _solve_gpu /
_solve_gpu_id of src/xclean/backend/ba.py, through libxcb200's C ABI.

Parity: each stage kernel against its float64 restatement in oracle/lba_oracle.py on the golden problems' start
state (relative 1e-4: float32 arithmetic with float atomics, whose order is unspecified); each solver against the
float64 restatement of the reference's device LM loop (poses 2e-4 m) and against the reference's own CPU solver
outputs in tests/golden/lba_golden.npz with the reference's GPU-vs-numpy tolerance (src/xclean/tests/test_ba.py:
translation 5e-3 m, |rms difference| 0.05 px), plus its convergence bar (pose error below 0.6x the initial)."""
import os

import numpy as np
import pytest

from oracle import lba_oracle as LO

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lba_golden.npz")


class _Rig:
    def __init__(self, v):
        self.fx_rect, self.cx, self.cy = float(v[0]), float(v[1]), float(v[2])


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLD))


def _err(a, b):
    return float(np.sqrt(np.mean(np.sum((a[:, :3, 3] - b[:, :3, 3]) ** 2, 1))))


def _rotf(G):
    return [(int(a), int(b), M, float(s)) for a, b, M, s in zip(G["p_rot_a"], G["p_rot_b"], G["p_rot_M"],
                                                                 G["p_rot_sig"])]


def _close(a, b, rel, what):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(float(np.abs(b).max()), 1e-12)
    err = float(np.abs(a - b).max()) / scale
    assert err <= rel, "%s: max abs diff %.3e relative to max |ref| %.3e = %.3e > %.1e" % (
        what, float(np.abs(a - b).max()), scale, err, rel)


# ------------------------------------------------------------------------------------------------- solvers
def test_solve_gpu_agrees_with_the_reference(G):
    from xclean_b200.backend.local_ba import _solve_gpu
    rig = _Rig(G["rig"])
    p, q, st = _solve_gpu(G["e_poses0"].copy(), G["e_pts0"].copy(), G["e_okf"], G["e_olm"], G["e_ouv"], rig, 0, 5)
    assert np.abs(p[:, :3, 3] - G["e_poses"][:, :3, 3]).max() < 5e-3
    assert abs(st["rms_n"] - G["e_stats"][3]) < 0.05
    assert _err(p, G["e_poses_true"]) < 0.6 * _err(G["e_poses0"], G["e_poses_true"])
    assert st["n_obs"] == len(G["e_okf"]) and st["npair"] == int((np.bincount(G["e_olm"]) ** 2).sum())
    # against the float64 restatement of the same device loop
    fx, cx, cy = G["rig"][:3]
    po, qo, _r, so = LO.solve_gpu_loop("euclid", G["e_poses0"], G["e_pts0"], G["e_okf"], G["e_olm"], G["e_ouv"], fx,
                                       cx, cy, 0, 5)
    assert np.abs(p[:, :3, 3] - po[:, :3, 3]).max() < 2e-4
    assert np.abs(p[:, :3, :3] - po[:, :3, :3]).max() < 2e-4
    assert np.abs(q - qo).max() < 5e-3
    assert abs(st["chi2_n"] - so["chi2_n"]) <= 1e-3 * so["chi2_n"]
    assert abs(st["rms_0"] - so["rms_0"]) <= 1e-4 * so["rms_0"]
    # the rotations come back orthonormal (one projection at the end)
    R = p[:, :3, :3]
    assert np.abs(np.einsum("nij,nkj->nik", R, R) - np.eye(3)).max() < 1e-12


def test_solve_gpu_with_prior_rotation_factors_and_held_keyframes(G):
    from xclean_b200.backend.local_ba import _solve_gpu
    rig = _Rig(G["rig"])
    prior = (G["p_c"], G["p_rho0"], G["p_invsig"], G["p_valid"])
    p, q, st = _solve_gpu(G["e_poses0"].copy(), G["e_pts0"].copy(), G["e_okf"], G["e_olm"], G["e_ouv"], rig,
                          G["p_free"], 5, prior=prior, rotf=_rotf(G))
    fx, cx, cy = G["rig"][:3]
    po, qo, _r, so = LO.solve_gpu_loop("euclid", G["e_poses0"], G["e_pts0"], G["e_okf"], G["e_olm"], G["e_ouv"], fx,
                                       cx, cy, G["p_free"], 5, prior=prior, rotf=_rotf(G))
    assert np.abs(p[:, :3, 3] - po[:, :3, 3]).max() < 2e-4
    assert abs(st["chi2_n"] - so["chi2_n"]) <= 1e-3 * so["chi2_n"]
    # held keyframes do not move
    for i in np.nonzero(~G["p_free"])[0]:
        assert np.abs(p[i] - G["e_poses0"][i]).max() < 1e-9
    # (keyframe 4 is held at its perturbed pose, so the truth is out of reach; the fit still improves)
    assert st["rms_n"] < st["rms_0"]


def test_solve_gpu_id_agrees_with_the_reference(G):
    from xclean_b200.backend.local_ba import _solve_gpu_id
    rig = _Rig(G["rig"])
    prior = (G["i_m0"], G["i_prho0"], G["i_wbear"], G["i_invsig"], G["i_valid"])
    p, rho, m, st = _solve_gpu_id(G["i_poses0"].copy(), G["i_rho0"].copy(), G["i_mbear0"].copy(), G["i_hidx"],
                                  G["i_hpose"], G["i_okf"], G["i_olm"], G["i_ouv"], rig, 0, 5, prior=prior)
    assert np.abs(p[:, :3, 3] - G["i_poses"][:, :3, 3]).max() < 5e-3
    assert _err(p, G["i_poses_true"]) < 0.6 * _err(G["i_poses0"], G["i_poses_true"])
    np.testing.assert_allclose(rho, G["i_rho"], rtol=5e-3)
    fx, cx, cy = G["rig"][:3]
    po, mo, ro, so = LO.solve_gpu_loop("id", G["i_poses0"], G["i_mbear0"], G["i_okf"], G["i_olm"], G["i_ouv"], fx, cx,
                                       cy, 0, 5, prior=prior, rho=G["i_rho0"], hidx=G["i_hidx"],
                                       hpose_ext=G["i_hpose"])
    assert np.abs(p[:, :3, 3] - po[:, :3, 3]).max() < 2e-4
    np.testing.assert_allclose(rho, ro, rtol=1e-3)
    np.testing.assert_allclose(m[:, :2], mo[:, :2], atol=1e-5)
    assert np.array_equal(m[:, 2], G["i_mbear0"][:, 2])
    assert abs(st["chi2_n"] - so["chi2_n"]) <= 1e-3 * so["chi2_n"]


def test_solve_gpu_on_generated_problems_and_edge_cases():
    from xclean_b200.backend import local_ba as LB
    from xclean_b200.backend.synth_lba import make_problem, make_problem_id
    pb = make_problem(nk=8, nl=200, seed=3)
    p, q, st = LB._solve_gpu(pb["poses0"], pb["pts0"], pb["okf"], pb["olm"], pb["ouv"], pb["rig"], 0, 5)
    assert _err(p, pb["poses_true"]) < 0.6 * _err(pb["poses0"], pb["poses_true"])
    assert st["rms_n"] < st["rms_0"]
    pi = make_problem_id(make_problem(nk=10, nl=300, seed=4))
    p, rho, m, st = LB._solve_gpu_id(pi["poses0"], pi["rho0"], pi["mbear0"], pi["hidx"], pi["hpose_ext"], pi["okf"],
                                     pi["olm"], pi["ouv"], pi["rig"], 0, 5, prior=pi["prior"])
    assert _err(p, pi["poses_true"]) < 0.6 * _err(pi["poses0"], pi["poses_true"])
    assert (rho >= 1e-4).all()
    # zero iterations: the state comes back (rotations projected), stats of the start state
    p0, q0, st0 = LB._solve_gpu(pb["poses0"], pb["pts0"], pb["okf"], pb["olm"], pb["ouv"], pb["rig"], 0, 0)
    assert np.abs(p0 - pb["poses0"]).max() < 1e-12 and np.abs(q0 - pb["pts0"]).max() == 0.0
    # a landmark without observations keeps a finite state
    pts = np.concatenate([pb["pts0"], [[0.5, 0.2, 4.0]]])
    p1, q1, _ = LB._solve_gpu(pb["poses0"], pts, pb["okf"], pb["olm"], pb["ouv"], pb["rig"], 0, 3)
    assert np.isfinite(q1).all()
    with pytest.raises(ValueError):
        LB._solve_gpu(np.repeat(pb["poses0"], 10, 0), pb["pts0"], pb["okf"], pb["olm"], pb["ouv"], pb["rig"], 0, 1)
    bad = pb["okf"].copy()
    bad[0] = 99
    with pytest.raises(ValueError):
        LB._solve_gpu(pb["poses0"], pb["pts0"], bad, pb["olm"], pb["ouv"], pb["rig"], 0, 1)


# -------------------------------------------------------------------------------------------- stage kernels
def _dev(a, dt):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dt)).cuda()


def _sorted_problem(G):
    order = np.argsort(G["e_olm"], kind="stable")
    return G["e_okf"][order].astype(np.int32), G["e_olm"][order].astype(np.int32), G["e_ouv"][order]


def test_stage_kernels_euclidean(G):
    import torch
    from xclean_b200.backend import kernels as K
    fx, cx, cy = G["rig"][:3]
    okf, olm, ouv = _sorted_problem(G)
    nk, nl, N = len(G["e_poses0"]), len(G["e_pts0"]), len(okf)
    d, n = 6, 6 * nk
    Tcw = LO.se3_inv(G["e_poses0"])[:, :3, :].reshape(nk, 12)
    ref = LO.k_build_blocks(Tcw.astype(np.float32).astype(np.float64), G["e_pts0"].astype(np.float32), okf, olm,
                            ouv.astype(np.float32), fx, cx, cy, LO.HUBER_K, nl)
    z = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")
    g_T, g_pts = _dev(Tcw, np.float32), _dev(G["e_pts0"], np.float32)
    g_okf, g_olm, g_ouv = _dev(okf, np.int32), _dev(olm, np.int32), _dev(ouv, np.float32)
    Jpose, Jlm, resw, Hll, bl, Hpl = z(N, 2, 6), z(N, 2, 3), z(N, 2), z(nl, 9), z(nl, 3), z(N, 6, 3)
    K.build_blocks(g_T, g_pts, g_okf, g_olm, g_ouv, Jpose, Jlm, resw, Hll, bl, Hpl, N, fx, cx, cy, LO.HUBER_K)
    for name, t in (("Jpose", Jpose), ("Jlm", Jlm), ("resw", resw), ("Hll", Hll), ("bl", bl), ("Hpl", Hpl)):
        _close(t.cpu().numpy(), ref[name], 1e-4, name)
    # depth prior (some invalid), inverse, Schur over the pair list, gradient, pose blocks
    rng = np.random.default_rng(0)
    valid = (rng.random(nl) < 0.7).astype(np.float32)
    h_p, b_p = LO.k_depth_prior(G["e_pts0"].astype(np.float32), G["p_c"], G["p_rho0"], G["p_invsig"], valid,
                                LO.HUBER_K)
    Hll2, bl2 = z(nl, 9), z(nl, 3)
    K.depth_prior(g_pts, _dev(G["p_c"], np.float32), _dev(G["p_rho0"], np.float32), _dev(G["p_invsig"], np.float32),
                  _dev(valid, np.float32), Hll2, bl2, nl, LO.HUBER_K)
    _close(Hll2.cpu().numpy(), h_p, 1e-4, "depth_prior Hll")
    _close(bl2.cpu().numpy(), b_p, 1e-4, "depth_prior bl")
    lam = 1e-3
    Hlli = z(nl, 9)
    K.inv3_damped(Hll, Hlli, nl, lam)
    # float32 cofactor inverse: compare where the damped block is well conditioned (its error grows with cond * eps)
    Hh = Hll.cpu().numpy().astype(np.float64)
    Hi_ref = LO.k_inv3_damped(Hh, lam)
    Hd = Hh.reshape(-1, 3, 3) + lam * np.maximum(np.trace(Hh.reshape(-1, 3, 3), axis1=1, axis2=2) / 3, 1e-9)[
        :, None, None] * np.eye(3)
    good = np.linalg.cond(Hd) < 1e4
    assert good.sum() > nl // 4
    _close(Hlli.cpu().numpy()[good], Hi_ref[good], 1e-3, "inv3_damped")
    from xclean_b200.backend.local_ba import build_pairs
    offs, pa, pb = build_pairs(olm, nl)
    o2, pa2, pb2 = LO.build_pairs(olm, nl)
    assert np.array_equal(offs, o2) and np.array_equal(pa, pa2) and np.array_equal(pb, pb2)
    Hred, grad = z(n, n), z(n)
    Hpl_h, Hi_h, bl_h = Hpl.cpu().numpy(), Hlli.cpu().numpy(), bl.cpu().numpy()
    K.pose_blocks(Jpose, resw, g_okf, Hred, grad, N, 2, d, n)
    Hp_ref, gp_ref = LO.k_pose_blocks(Jpose.cpu().numpy(), resw.cpu().numpy(), okf, n)
    _close(Hred.cpu().numpy(), Hp_ref, 1e-4, "pose_blocks H")
    _close(grad.cpu().numpy(), gp_ref, 1e-4, "pose_blocks g")
    Hs, gs = z(n, n), z(n)
    K.schur_pairs(Hpl, Hlli, g_okf, g_olm, _dev(pa, np.int32), _dev(pb, np.int32), Hs, len(pa), d, n)
    K.schur_grad(Hpl, Hlli, bl, g_okf, g_olm, gs, N, d)
    _close(Hs.cpu().numpy(), LO.k_schur_pairs(Hpl_h, Hi_h, okf, olm, pa, pb, n), 1e-4, "schur_pairs")
    _close(gs.cpu().numpy(), LO.k_schur_grad(Hpl_h, Hi_h, bl_h, okf, olm, n), 1e-4, "schur_grad")
    # Cholesky + solve on a well-conditioned SPD system (both the shared-memory and the global-memory form)
    for nn in (90, 200):
        A = rng.standard_normal((nn, nn))
        S = (A @ A.T / nn + np.eye(nn)).astype(np.float32)
        b = rng.standard_normal(nn).astype(np.float32)
        gH, gx = _dev(S, np.float32), z(nn)
        st = K.chol_solve(gH, _dev(b, np.float32), gx, nn)
        assert int(st.item()) == 0
        L_ref, x_ref = LO.k_chol_solve(S.astype(np.float64), b.astype(np.float64))
        _close(gx.cpu().numpy(), x_ref, 1e-4, "chol_solve x (n=%d)" % nn)
        _close(np.tril(gH.cpu().numpy()), L_ref, 1e-4, "chol_solve factor (n=%d)" % nn)
    # a non-positive pivot is reported as k + 1
    S = np.eye(8, dtype=np.float32)
    S[3, 3] = -1.0
    st = K.chol_solve(_dev(S, np.float32), _dev(np.ones(8), np.float32), z(8), 8)
    assert int(st.item()) == 4
    dxp = rng.standard_normal(n).astype(np.float32) * 1e-2
    dxl = z(nl, 3)
    K.backsub(Hpl, Hlli, bl, _dev(dxp, np.float32), g_okf, _dev(offs, np.int32), dxl, nl, d)
    _close(dxl.cpu().numpy(), LO.k_backsub(Hpl_h, Hi_h, bl_h, dxp, okf, offs), 1e-4, "backsub")
    with pytest.raises(TypeError):
        K.inv3_damped(Hll.double(), Hlli, nl, lam)


def test_stage_kernels_inverse_depth(G):
    import torch
    from xclean_b200.backend import kernels as K
    from xclean_b200.backend.local_ba import build_pairs
    fx, cx, cy = G["rig"][:3]
    order = np.argsort(G["i_olm"], kind="stable")
    okf, olm, ouv = G["i_okf"][order].astype(np.int32), G["i_olm"][order].astype(np.int32), G["i_ouv"][order]
    nk, nl, N = len(G["i_poses0"]), len(G["i_rho0"]), len(okf)
    d, n = 6, 6 * nk
    Tcw = LO.se3_inv(G["i_poses0"])[:, :3, :].reshape(nk, 12)
    z = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")
    g_okf, g_olm = _dev(okf, np.int32), _dev(olm, np.int32)
    Jp, resw, kslot, Hll, bl, Hpl = (z(N, 2, 2, 6), z(N, 2), torch.zeros(N, 2, dtype=torch.int32, device="cuda"),
                                     z(nl, 9), z(nl, 3), z(N, 2, 6, 3))
    K.build_blocks_id(_dev(Tcw, np.float32), _dev(G["i_hpose"], np.float32), _dev(G["i_hidx"], np.int32),
                      _dev(G["i_mbear0"], np.float32), _dev(G["i_rho0"], np.float32), g_okf, g_olm,
                      _dev(ouv, np.float32), Jp, resw, kslot, Hll, bl, Hpl, N, fx, cx, cy, LO.HUBER_K)
    ref = LO.k_build_blocks_id(Tcw.astype(np.float32), G["i_hpose"].astype(np.float32), G["i_hidx"],
                               G["i_mbear0"].astype(np.float32), G["i_rho0"].astype(np.float32), okf, olm,
                               ouv.astype(np.float32), fx, cx, cy, LO.HUBER_K, nl)
    assert np.array_equal(kslot.cpu().numpy(), ref["kslot"])
    for name, t in (("Jp", Jp), ("resw", resw), ("Hll", Hll), ("bl", bl), ("Hpl", Hpl)):
        _close(t.cpu().numpy(), ref[name], 2e-4, name)
    Hll2, bl2 = z(nl, 9), z(nl, 3)
    valid = (np.arange(nl) % 5 != 0).astype(np.float32)
    K.landmark_prior_id(_dev(G["i_mbear0"], np.float32), _dev(G["i_rho0"], np.float32), _dev(G["i_m0"], np.float32),
                        _dev(G["i_prho0"], np.float32), _dev(G["i_invsig"], np.float32),
                        _dev(G["i_wbear"], np.float32), _dev(valid, np.float32), Hll2, bl2, nl, LO.HUBER_K)
    f32 = lambda k: G[k].astype(np.float32).astype(np.float64)       # the device's inputs exactly
    hp, bp_ = LO.k_landmark_prior_id(f32("i_mbear0"), f32("i_rho0"), f32("i_m0"), f32("i_prho0"), f32("i_invsig"),
                                     f32("i_wbear"), valid, LO.HUBER_K)
    _close(Hll2.cpu().numpy(), hp, 1e-4, "landmark_prior_id Hll")
    _close(bl2.cpu().numpy(), bp_, 1e-4, "landmark_prior_id bl")
    Hlli = z(nl, 9)
    K.inv3_damped(Hll, Hlli, nl, 1e-4)
    ks = kslot.cpu().numpy()
    Hpl_h, Hi_h, bl_h = Hpl.cpu().numpy(), Hlli.cpu().numpy(), bl.cpu().numpy()
    Hred, grad = z(n, n), z(n)
    K.pose_blocks_id(Jp, resw, kslot, Hred, grad, N, d, n)
    Hr, gr = LO.k_pose_blocks_id(Jp.cpu().numpy(), resw.cpu().numpy(), ks, n)
    _close(Hred.cpu().numpy(), Hr, 1e-4, "pose_blocks_id H")
    _close(grad.cpu().numpy(), gr, 1e-4, "pose_blocks_id g")
    offs, pa, pb = build_pairs(olm, nl)
    Hs, gs = z(n, n), z(n)
    K.schur_pairs_id(Hpl, Hlli, kslot, g_olm, _dev(pa, np.int32), _dev(pb, np.int32), Hs, len(pa), d, n)
    K.schur_grad_id(Hpl, Hlli, bl, kslot, g_olm, gs, N, d)
    _close(Hs.cpu().numpy(), LO.k_schur_pairs_id(Hpl_h, Hi_h, ks, olm, pa, pb, n), 1e-4, "schur_pairs_id")
    _close(gs.cpu().numpy(), LO.k_schur_grad_id(Hpl_h, Hi_h, bl_h, ks, olm, n), 1e-4, "schur_grad_id")
    dxp = np.random.default_rng(1).standard_normal(n).astype(np.float32) * 1e-2
    dxl = z(nl, 3)
    K.backsub_id(Hpl, Hlli, bl, _dev(dxp, np.float32), kslot, _dev(offs, np.int32), dxl, nl, d)
    _close(dxl.cpu().numpy(), LO.k_backsub_id(Hpl_h, Hi_h, bl_h, dxp, ks, offs), 1e-4, "backsub_id")
