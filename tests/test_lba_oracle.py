"""The local-BA oracle (float64 restatement of src/xclean/backend/ba.py's CPU solvers and helpers) against outputs of
the reference itself (tests/golden/lba_golden.npz, made by tests/golden/make_golden_lba.py).  CPU only."""
import os

import numpy as np
import pytest

from oracle import lba_oracle as LO

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lba_golden.npz")


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLD))


def _rig(G):
    fx, cx, cy = G["rig"][:3]
    return fx, cx, cy


def test_lie_helpers_match_the_reference(G):
    np.testing.assert_allclose(LO.se3_exp(G["lie_xi"]), G["lie_exp"], rtol=0, atol=1e-12)
    phi = G["lie_xi"][:, 3:]
    np.testing.assert_allclose(LO.so3_log(G["lie_R"]), G["lie_log"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(LO.so3_project(G["lie_Rn"]), G["lie_proj"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(LO.so3_jr_inv(phi), G["lie_jrinv"], rtol=0, atol=1e-9)


def test_build_pairs_matches_the_reference(G):
    offs, pa, pb = LO.build_pairs(G["bp_olm"], 9)
    assert np.array_equal(offs, G["bp_offs"])
    assert np.array_equal(pa, G["bp_pa"]) and np.array_equal(pb, G["bp_pb"])


def test_rotation_factor_blocks_match_the_reference(G):
    rotf = [(int(a), int(b), M, float(s)) for a, b, M, s in zip(G["p_rot_a"], G["p_rot_b"], G["p_rot_M"],
                                                                 G["p_rot_sig"])]
    H, g, chi = LO.rot_factor_blocks(LO.se3_inv(G["e_poses0"]), rotf, 6, 6 * len(G["e_poses0"]))
    np.testing.assert_allclose(H, G["r_H"], rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(g, G["r_g"], rtol=1e-9, atol=1e-8)
    assert abs(chi - G["r_chi"][0]) <= 1e-9 * max(1.0, abs(chi))


def test_euclidean_solver_matches_the_reference(G):
    fx, cx, cy = _rig(G)
    p, q, st = LO.solve_np(G["e_poses0"], G["e_pts0"], G["e_okf"], G["e_olm"], G["e_ouv"], fx, cx, cy, 0, 5)
    np.testing.assert_allclose(p, G["e_poses"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(q, G["e_pts"], rtol=0, atol=1e-9)
    np.testing.assert_allclose([st["chi2_0"], st["chi2_n"], st["rms_0"], st["rms_n"]], G["e_stats"], rtol=1e-9)


def test_euclidean_solver_with_prior_rotf_and_held_keyframes_matches_the_reference(G):
    fx, cx, cy = _rig(G)
    rotf = [(int(a), int(b), M, float(s)) for a, b, M, s in zip(G["p_rot_a"], G["p_rot_b"], G["p_rot_M"],
                                                                 G["p_rot_sig"])]
    p, q, st = LO.solve_np(G["e_poses0"], G["e_pts0"], G["e_okf"], G["e_olm"], G["e_ouv"], fx, cx, cy, G["p_free"],
                           5, prior=(G["p_c"], G["p_rho0"], G["p_invsig"], G["p_valid"]), rotf=rotf)
    np.testing.assert_allclose(p, G["p_poses"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(q, G["p_pts"], rtol=0, atol=1e-9)
    np.testing.assert_allclose([st["chi2_0"], st["chi2_n"], st["rms_0"], st["rms_n"]], G["p_stats"], rtol=1e-9)


def test_inverse_depth_blocks_match_the_reference(G):
    fx, cx, cy = _rig(G)
    Jo, Jh, Jl, r = LO.analytic_blocks_id(G["i_poses0"], LO.se3_inv(G["i_poses0"]), G["i_rho0"], G["i_mbear0"],
                                          G["i_hidx"], G["i_hpose"], G["i_okf"], G["i_olm"], G["i_ouv"], fx, cx, cy)
    for a, b in ((Jo, "a_Jobs"), (Jh, "a_Jhost"), (Jl, "a_Jlm"), (r, "a_r")):
        np.testing.assert_allclose(a, G[b], rtol=1e-12, atol=1e-9)


def test_inverse_depth_solver_matches_the_reference(G):
    fx, cx, cy = _rig(G)
    prior = (G["i_m0"], G["i_prho0"], G["i_wbear"], G["i_invsig"], G["i_valid"])
    p, rho, m, st = LO.solve_np_id(G["i_poses0"], G["i_rho0"], G["i_mbear0"], G["i_hidx"], G["i_hpose"], G["i_okf"],
                                   G["i_olm"], G["i_ouv"], fx, cx, cy, 0, 5, prior=prior)
    np.testing.assert_allclose(p, G["i_poses"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(rho, G["i_rho"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(m, G["i_mbear"], rtol=0, atol=1e-12)
    np.testing.assert_allclose([st["chi2_0"], st["chi2_n"], st["rms_0"], st["rms_n"]], G["i_stats"], rtol=1e-9)


def test_reference_solvers_move_poses_toward_the_truth(G):
    """The reference's own acceptance bar (tests/test_ba_solver.py): pose error < 0.6x the initial, rms decreases."""
    err = lambda a, b: float(np.sqrt(np.mean(np.sum((a[:, :3, 3] - b[:, :3, 3]) ** 2, 1))))
    assert err(G["e_poses"], G["e_poses_true"]) < 0.6 * err(G["e_poses0"], G["e_poses_true"])
    assert G["e_stats"][3] < G["e_stats"][2]
    assert G["i_stats"][3] < G["i_stats"][2]


def test_device_loop_restatement_converges_like_the_cpu_solver(G):
    """The float64 restatement of the reference's device LM loop (another accept rule, no per-step projection) lands
    within the reference's own GPU-vs-numpy tolerance of _solve_np (src/xclean/tests/test_ba.py: pose 5e-3 m,
    rms 0.05 px)."""
    fx, cx, cy = _rig(G)
    p, q, _r, st = LO.solve_gpu_loop("euclid", G["e_poses0"], G["e_pts0"], G["e_okf"], G["e_olm"], G["e_ouv"], fx, cx,
                                     cy, 0, 5)
    assert np.abs(p[:, :3, 3] - G["e_poses"][:, :3, 3]).max() < 5e-3
    assert abs(st["rms_n"] - G["e_stats"][3]) < 0.05
    prior = (G["i_m0"], G["i_prho0"], G["i_wbear"], G["i_invsig"], G["i_valid"])
    p, m, rho, st = LO.solve_gpu_loop("id", G["i_poses0"], G["i_mbear0"], G["i_okf"], G["i_olm"], G["i_ouv"], fx, cx,
                                      cy, 0, 5, prior=prior, rho=G["i_rho0"], hidx=G["i_hidx"],
                                      hpose_ext=G["i_hpose"])
    assert np.abs(p[:, :3, 3] - G["i_poses"][:, :3, 3]).max() < 5e-3
    assert abs(st["rms_n"] - G["i_stats"][3]) < 0.05
