"""Synthetic local-BA problems with a known ground truth (the shape of src/xclean/backend/ba_synth.py).

make_problem(nk, nl, obs_per, seed, ...) -> dict(rig, poses_true, pts_true, poses0, pts0, okf, olm, ouv): keyframes on
a smooth arc (0.09 m, 0.01 m and 0.02 rad of yaw per keyframe), points uniform in x [-1.9, 3.1], y [-1.5, 1.5],
z [1.5, 8] m, each seen by `obs_per` random keyframes when in front of the camera (z >= 0.5 m) and inside the
752 x 480 image, 0.5 px pixel noise; keyframe 0 exact, the others perturbed by exp(N(0, 0.02)) on the right, points
by N(0, 0.05) m.  make_problem_id converts one into the host-anchored inverse-depth form of _solve_gpu_id.
"""
from __future__ import annotations

import numpy as np


class Rig:
    fx_rect = 458.654
    cx, cy = 367.215, 248.375
    width, height = 752, 480


def _se3_exp(xi):
    xi = np.asarray(xi, np.float64)
    rho, phi = xi[:3], xi[3:]
    t2 = float(phi @ phi)
    t = np.sqrt(t2)
    if t < 1e-8:
        a, b, c = 1.0 - t2 / 6.0, 0.5 - t2 / 24.0, 1.0 / 6.0 - t2 / 120.0
    else:
        a, b, c = np.sin(t) / t, (1.0 - np.cos(t)) / t2, (t - np.sin(t)) / (t2 * t)
    K = np.array([[0.0, -phi[2], phi[1]], [phi[2], 0.0, -phi[0]], [-phi[1], phi[0], 0.0]])
    T = np.eye(4)
    T[:3, :3] = np.eye(3) + a * K + b * K @ K
    T[:3, 3] = (np.eye(3) + b * K + c * K @ K) @ rho
    return T


def _se3_inv(T):
    out = np.eye(4)
    out[:3, :3] = T[:3, :3].T
    out[:3, 3] = -T[:3, :3].T @ T[:3, 3]
    return out


def make_problem(nk=15, nl=600, obs_per=4, seed=5, pose_noise=0.02, pt_noise=0.05, px_noise=0.5):
    rng = np.random.RandomState(seed)
    rig = Rig()
    poses_true = np.stack([_se3_exp([0.09 * i, 0.01 * i, 0.0, 0.0, 0.02 * i, 0.0]) for i in range(nk)])
    pts = np.stack([rng.uniform(-2.5, 2.5, nl) + 0.6, rng.uniform(-1.5, 1.5, nl), rng.uniform(1.5, 8.0, nl)], 1)
    Tcw = np.stack([_se3_inv(T) for T in poses_true])
    okf, olm, ouv = [], [], []
    for j in range(nl):
        for k in rng.choice(nk, size=min(obs_per, nk), replace=False):
            Pc = Tcw[k, :3, :3] @ pts[j] + Tcw[k, :3, 3]
            if Pc[2] < 0.5:
                continue
            u = rig.fx_rect * Pc[0] / Pc[2] + rig.cx
            v = rig.fx_rect * Pc[1] / Pc[2] + rig.cy
            if not (0 <= u < rig.width and 0 <= v < rig.height):
                continue
            okf.append(k)
            olm.append(j)
            ouv.append((u + rng.randn() * px_noise, v + rng.randn() * px_noise))
    okf = np.array(okf, np.int32)
    uniq, olm = np.unique(np.array(olm, np.int64), return_inverse=True)
    pts = pts[uniq]
    poses0 = poses_true.copy()
    for i in range(1, nk):
        poses0[i] = poses_true[i] @ _se3_exp(rng.randn(6) * pose_noise)
    pts0 = pts + rng.randn(*pts.shape) * pt_noise
    return dict(rig=rig, poses_true=poses_true, pts_true=pts, poses0=poses0, pts0=pts0, okf=okf,
                olm=olm.astype(np.int32), ouv=np.array(ouv, np.float64).reshape(-1, 2))


def make_problem_id(pb, leave=3, seed=11):
    """Inverse-depth form of a make_problem dict: host = a landmark's first observer; keyframes 0..leave-1 leave the
    window (their landmarks keep them as constant hosts, hpose_ext = the true T_wc); the host's own rows are dropped;
    bearing from the host pixel, inverse depth from the perturbed point; the held window keyframe is exact.
    -> dict(poses0, rho0, mbear0, hidx, hpose_ext, okf, olm, ouv, prior, poses_true, rig)."""
    rng = np.random.RandomState(seed)
    rig = pb["rig"]
    nk, nl = len(pb["poses0"]), len(pb["pts0"])
    okf, olm, ouv = pb["okf"].astype(np.int64), pb["olm"].astype(np.int64), pb["ouv"]
    first = np.full(nl, -1)
    hobs = np.full(nl, -1)
    for o in range(len(okf)):
        if first[olm[o]] < 0:
            first[olm[o]] = okf[o]
            hobs[olm[o]] = o
    keep_kf = np.arange(leave, nk)
    remap = np.full(nk, -1)
    remap[keep_kf] = np.arange(len(keep_kf))
    Tcw0 = np.stack([_se3_inv(T) for T in pb["poses0"]])
    Tcw_t = np.stack([_se3_inv(T) for T in pb["poses_true"]])
    uvh = ouv[hobs]
    mbear = np.stack([(uvh[:, 0] - rig.cx) / rig.fx_rect, (uvh[:, 1] - rig.cy) / rig.fx_rect, np.ones(nl)], 1)
    Ph = np.einsum("nij,nj->ni", Tcw0[first, :3, :3], pb["pts0"]) + Tcw0[first, :3, 3]
    rho = 1.0 / np.maximum(Ph[:, 2], 0.3)
    out_host = first < leave
    hidx = np.where(out_host, -1, remap[first])
    hpose = np.zeros((nl, 12))
    hpose[out_host] = pb["poses_true"][first[out_host], :3, :].reshape(-1, 12)
    sel = (okf != first[olm]) & (remap[okf] >= 0)
    poses0 = pb["poses0"][keep_kf].copy()
    poses0[0] = pb["poses_true"][keep_kf[0]]
    Pt = np.einsum("nij,nj->ni", Tcw_t[first, :3, :3], pb["pts_true"]) + Tcw_t[first, :3, 3]
    prior = (mbear[:, :2].copy(), 1.0 / Pt[:, 2] * (1.0 + 0.01 * rng.randn(nl)), np.full(nl, 1e3), np.full(nl, 50.0),
             np.ones(nl))
    return dict(poses0=poses0, rho0=rho, mbear0=mbear, hidx=hidx, hpose_ext=hpose, okf=remap[okf[sel]].astype(np.int32),
                olm=olm[sel].astype(np.int32), ouv=ouv[sel], prior=prior, poses_true=pb["poses_true"][keep_kf],
                rig=rig)
