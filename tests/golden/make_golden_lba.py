"""Generate tests/golden/lba_golden.npz from the reference's own local-BA code (run once, where the reference is).

    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_lba.py <reference>/src

Records, from src/xclean/backend/ba.py, ba_synth.py and core/lie.py of the reference:
  * e_*   the synthetic Euclidean problem make_problem() (15 keyframes, 600 points, seed 5) and _solve_np's result
          (keyframe 0 held, 5 iterations);
  * p_*   the same problem with a depth prior, gyro rotation factors and two held keyframes, and _solve_np's result;
  * i_*   an inverse-depth problem built from it (hosts: the first observer; landmarks hosted by keyframes 0-2 keep
          those hosts as out-of-window constants; the host's own rows dropped; bearing + depth prior) and
          _solve_np_id's result; _analytic_blocks_id at the start state;
  * r_*   _rot_factor_blocks on the gyro factors at the start state;
  * bp_*  build_pairs on a small sorted landmark list;
  * lie_* se3_exp, so3_log, so3_project and so3_jr_inv on random, small-angle and near-pi inputs.
"""
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lba_golden.npz")


def main(src):
    sys.path.insert(0, src)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    from xclean.backend import ba as B
    from xclean.backend.ba_synth import make_problem
    from xclean.core import lie
    out = {}
    pb = make_problem()
    rig = pb["rig"]
    out.update(e_poses0=pb["poses0"], e_pts0=pb["pts0"], e_okf=pb["okf"], e_olm=pb["olm"], e_ouv=pb["ouv"],
               e_poses_true=pb["poses_true"], e_pts_true=pb["pts_true"],
               rig=np.array([rig.fx_rect, rig.cx, rig.cy, rig.width, rig.height], np.float64))
    p, q, st = B._solve_np(pb["poses0"].copy(), pb["pts0"].copy(), pb["okf"], pb["olm"], pb["ouv"], rig, 0, 5)
    out.update(e_poses=p, e_pts=q, e_stats=np.array([st["chi2_0"], st["chi2_n"], st["rms_0"], st["rms_n"]]))

    # prior, rotation factors, two held keyframes
    rng = np.random.RandomState(11)
    nk, nl = len(pb["poses0"]), len(pb["pts0"])
    first = np.full(nl, -1)
    for o in range(len(pb["okf"])):
        if first[pb["olm"][o]] < 0:
            first[pb["olm"][o]] = pb["okf"][o]
    c = pb["poses_true"][first, :3, 3]
    dist = np.linalg.norm(pb["pts_true"] - c, axis=1)
    rho0 = 1.0 / dist * (1.0 + 0.01 * rng.randn(nl))
    invsig = np.full(nl, 1.0 / 0.01)
    # every prior valid: _solve_np indexes the full invsig array with the valid subset (ba.py:788)
    valid = np.ones(nl)
    Tcw_true = lie.se3_inv(pb["poses_true"])
    rotf = []
    for i in range(nk - 1):
        M = Tcw_true[i, :3, :3] @ Tcw_true[i + 1, :3, :3].T @ lie.so3_exp(rng.randn(3) * 0.002)
        rotf.append((i, i + 1, M, 0.01))
    free = np.ones(nk, bool)
    free[[0, 4]] = False
    p2, q2, st2 = B._solve_np(pb["poses0"].copy(), pb["pts0"].copy(), pb["okf"], pb["olm"], pb["ouv"], rig, free, 5,
                              prior=(c, rho0, invsig, valid), rotf=rotf)
    out.update(p_c=c, p_rho0=rho0, p_invsig=invsig, p_valid=valid, p_free=free,
               p_rot_a=np.array([f[0] for f in rotf]), p_rot_b=np.array([f[1] for f in rotf]),
               p_rot_M=np.stack([f[2] for f in rotf]), p_rot_sig=np.array([f[3] for f in rotf]),
               p_poses=p2, p_pts=q2, p_stats=np.array([st2["chi2_0"], st2["chi2_n"], st2["rms_0"], st2["rms_n"]]))
    Hr, gr, chir = B._rot_factor_blocks(lie.se3_inv(pb["poses0"]), rotf, 6, 6 * nk)
    out.update(r_H=Hr, r_g=gr, r_chi=np.array([chir]))

    # inverse-depth problem
    okf, olm, ouv = pb["okf"].astype(np.int64), pb["olm"].astype(np.int64), pb["ouv"]
    host = first.copy()
    out_host = host <= 2                          # hosted outside the window (keyframes 0-2 leave it)
    keep_kf = np.arange(3, nk)
    remap = np.full(nk, -1)
    remap[keep_kf] = np.arange(len(keep_kf))
    Tcw0 = lie.se3_inv(pb["poses0"])
    # bearing and inverse depth at the host, from the host's (noisy) pixel and the perturbed point
    hobs = np.full(nl, -1)
    for o in range(len(okf)):
        if okf[o] == host[olm[o]] and hobs[olm[o]] < 0:
            hobs[olm[o]] = o
    uvh = ouv[hobs]
    mbear = np.stack([(uvh[:, 0] - rig.cx) / rig.fx_rect, (uvh[:, 1] - rig.cy) / rig.fx_rect, np.ones(nl)], 1)
    Ph = np.einsum("nij,nj->ni", Tcw0[host, :3, :3], pb["pts0"]) + Tcw0[host, :3, 3]
    rho = 1.0 / np.maximum(Ph[:, 2], 0.3)
    hidx = np.where(out_host, -1, remap[host])
    hpose = np.zeros((nl, 12))
    hpose[out_host] = pb["poses_true"][host[out_host], :3, :].reshape(-1, 12)
    sel = (okf != host[olm]) & (remap[okf] >= 0)
    i_okf, i_olm, i_ouv = remap[okf[sel]].astype(np.int32), olm[sel].astype(np.int32), ouv[sel]
    i_poses0 = pb["poses0"][keep_kf].copy()
    i_poses0[0] = pb["poses_true"][keep_kf[0]]     # the held keyframe agrees with the out-of-window hosts
    Pt = np.einsum("nij,nj->ni", Tcw_true[host, :3, :3], pb["pts_true"]) + Tcw_true[host, :3, 3]
    prior_id = (mbear[:, :2].copy(), 1.0 / Pt[:, 2] * (1.0 + 0.01 * rng.randn(nl)), np.full(nl, 1.0 / 1e-3),
                np.full(nl, 1.0 / 0.02), np.ones(nl))
    pi, ri, mi, sti = B._solve_np_id(i_poses0.copy(), rho.copy(), mbear.copy(), hidx, hpose, i_okf, i_olm, i_ouv, rig,
                                     0, 5, prior=prior_id)
    out.update(i_poses0=i_poses0, i_rho0=rho, i_mbear0=mbear, i_hidx=hidx, i_hpose=hpose, i_okf=i_okf, i_olm=i_olm,
               i_ouv=i_ouv, i_m0=prior_id[0], i_prho0=prior_id[1], i_wbear=prior_id[2], i_invsig=prior_id[3],
               i_valid=prior_id[4], i_poses=pi, i_rho=ri, i_mbear=mi,
               i_stats=np.array([sti["chi2_0"], sti["chi2_n"], sti["rms_0"], sti["rms_n"]]),
               i_poses_true=pb["poses_true"][keep_kf])
    Jo, Jh, Jl, r = B._analytic_blocks_id(i_poses0, lie.se3_inv(i_poses0), rho, mbear, hidx, hpose, i_okf, i_olm,
                                          i_ouv, rig)
    out.update(a_Jobs=Jo, a_Jhost=Jh, a_Jlm=Jl, a_r=r)

    olm_s = np.sort(rng.randint(0, 7, 25)).astype(np.int32)
    offs, pa, pb_ = B.build_pairs(olm_s, 9)
    out.update(bp_olm=olm_s, bp_offs=offs, bp_pa=pa, bp_pb=pb_)

    phi = np.concatenate([rng.randn(20, 3) * 0.5, rng.randn(10, 3) * 1e-3, rng.randn(5, 3) * 1e-9])
    ax = rng.randn(5, 3)
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    phi = np.concatenate([phi, ax * (np.pi - 1e-6)])
    xi = np.concatenate([rng.randn(len(phi), 3), phi], 1)
    Rn = lie.so3_exp(phi) + rng.randn(len(phi), 3, 3) * 1e-4
    out.update(lie_xi=xi, lie_exp=lie.se3_exp(xi), lie_R=lie.so3_exp(phi), lie_log=lie.so3_log(lie.so3_exp(phi)),
               lie_Rn=Rn, lie_proj=lie.so3_project(Rn), lie_jrinv=lie.so3_jr_inv(phi))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    main(sys.argv[1])
