"""Seeded synthetic sliding-window BA problems in the reference's window form (vio/window.Problem, stereo).

A window: K keyframes on a smooth random SE(3) path (step `step_m` metres and `step_deg` degrees between keyframes),
L landmarks uniform in the first keyframe's frustum at depths [z0, z1], each seen by a geometric-ish number of
keyframes as stereo observations: a left (u, v) row and a right u_R row per observing keyframe, with Gaussian pixel
noise and a fraction of uniform outliers.  Landmarks are hosted by their first observing keyframe in the reference's
inverse-depth chart (a, b, rho): m = (a, b, 1) the host's normalised left ray, rho the inverse depth.  The initial
state perturbs keyframes 1.. by (pose_m, pose_deg) and landmarks by depth_frac of their depth; keyframe 0 stays at
the truth (the held gauge slot).

The window arrays use the field names of window.Problem (src/xclean/vio/window.py:768-792):
    Rwb (K,3,3) pwb (K,3) Rbc pbc lmp (L,3) lm_host (L,) lm_mask rho_meas rho_isig ob_start (L+1,)
    ob_pose ob_cam ob_z (M,2) ob_isig ob_valid fx fy cx cy B huber_k
"""
from __future__ import annotations

import math

import numpy as np

HUBER_K = 1.345


def so3_exp(w):
    w = np.asarray(w, np.float64)
    th2 = float(w @ w)
    th = math.sqrt(th2)
    K = np.array([[0.0, -w[2], w[1]], [w[2], 0.0, -w[0]], [-w[1], w[0], 0.0]])
    if th < 1e-8:
        a, b = 1.0 - th2 / 6.0, 0.5 - th2 / 24.0
    else:
        a, b = math.sin(th) / th, (1.0 - math.cos(th)) / th2
    return np.eye(3) + a * K + b * (K @ K)


class Window:
    """One window's arrays (the fields of window.Problem) plus its ground truth."""

    FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
              "ob_cam", "ob_z", "ob_isig", "ob_valid", "fx", "fy", "cx", "cy", "B", "huber_k")

    def __init__(self, **kw):
        for k, v in kw.items():
            setattr(self, k, v)

    def copy(self):
        return Window(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})

    @property
    def P(self):
        return self.Rwb.shape[0]

    @property
    def L(self):
        return self.lmp.shape[0]

    @property
    def M(self):
        return self.ob_pose.shape[0]


def make_window(seed, K=10, L=1500, obs_min=2, obs_max=6, z0=2.0, z1=20.0, step_m=0.2, step_deg=5.0, px_noise=1.0,
                outlier_frac=0.05, pose_m=0.05, pose_deg=1.0, depth_frac=0.05, fx=458.0, fy=458.0, cx=367.0,
                cy=248.0, W=752, H=480, B=0.11, geometric=False, rng=None, Rbc=None, pbc=None, depth_prior=0.0):
    """-> Window (initial state in Rwb / pwb / lmp; truth in Rwb_true / pwb_true / lmp_true).  Rbc / pbc: the
    body-to-camera extrinsic (identity by default); depth_prior > 0: an inverse-depth prior on every landmark with
    that relative noise (none by default).  The defaults draw the same random sequence as without these options."""
    rng = np.random.default_rng(seed) if rng is None else rng
    # camera = body (identity extrinsic), smooth path: each step a random direction of norm step_m and a random axis
    Rbc = np.eye(3) if Rbc is None else np.asarray(Rbc, np.float64)
    pbc = np.zeros(3) if pbc is None else np.asarray(pbc, np.float64)
    Rs = [np.eye(3)]
    ps = [np.zeros(3)]
    v = np.array([0.3, 0.0, 1.0])
    v /= np.linalg.norm(v)
    for _k in range(1, K):
        v = v + rng.normal(0.0, 0.3, 3)
        v /= np.linalg.norm(v)
        ax = rng.normal(0.0, 1.0, 3)
        ax /= np.linalg.norm(ax)
        Rs.append(Rs[-1] @ so3_exp(ax * math.radians(step_deg)))
        ps.append(ps[-1] + step_m * v)
    Rwc_t = np.stack(Rs)                      # camera poses; the body poses follow from the extrinsic
    pwc_t = np.stack(ps)
    # landmarks in keyframe 0's frustum
    zs = rng.uniform(z0, z1, L)
    us = rng.uniform(0.05 * W, 0.95 * W, L)
    vs = rng.uniform(0.05 * H, 0.95 * H, L)
    Pc0 = np.stack([(us - cx) / fx * zs, (vs - cy) / fy * zs, zs], 1)
    Pw = Pc0 @ Rwc_t[0].T + pwc_t[0]
    # every (keyframe, landmark) projection at once
    Pc = np.einsum("kji,klj->kli", Rwc_t, Pw[None, :, :] - pwc_t[:, None, :])        # (K, L, 3)
    z = Pc[:, :, 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        ul = fx * Pc[:, :, 0] / z + cx
        vl = fy * Pc[:, :, 1] / z + cy
        ur = fx * (Pc[:, :, 0] - B) / z + cx
    vis = (z >= 0.5) & (ul >= 0) & (ul < W) & (vl >= 0) & (vl < H) & (ur >= 0) & (ur < W)
    nvis = vis.sum(0)
    if geometric:
        n = np.minimum(obs_max, obs_min + rng.geometric(0.35, L) - 1)
    else:
        n = rng.integers(obs_min, obs_max + 1, L)
    n = np.minimum(n, nvis)
    keep = nvis >= obs_min
    keys = rng.random((K, L))
    keys[~vis] = np.inf
    rank = np.argsort(np.argsort(keys, axis=0), axis=0)                                  # rank of each keyframe
    sel = (rank < n[None, :]) & vis & keep[None, :]                                       # (K, L)
    lidx = np.nonzero(keep)[0]
    Lk = len(lidx)
    selT = sel[:, lidx].T                                                                 # (Lk, K), keyframe order
    cnt = selT.sum(1)
    ob_start = np.zeros(Lk + 1, np.int64)
    ob_start[1:] = np.cumsum(2 * cnt)
    li, ki = np.nonzero(selT)                                                             # landmark-major, k ascending
    lg = lidx[li]
    nr = len(li)
    zl = np.stack([ul[ki, lg], vl[ki, lg]], 1) + rng.normal(0.0, px_noise, (nr, 2))
    zr = ur[ki, lg] + rng.normal(0.0, px_noise, nr)
    ol = rng.random(nr) < outlier_frac
    zl[ol] = np.stack([rng.uniform(0, W, int(ol.sum())), rng.uniform(0, H, int(ol.sum()))], 1)
    orr = rng.random(nr) < outlier_frac
    zr[orr] = rng.uniform(0, W, int(orr.sum()))
    ob_pose = np.repeat(ki, 2).astype(np.int64)
    ob_cam = np.tile(np.array([0, 1], np.int64), nr)
    ob_z = np.zeros((2 * nr, 2))
    ob_z[0::2] = zl
    ob_z[1::2, 0] = zr
    first = ob_start[:-1] // 2                                                            # each landmark's first row
    host = ki[first] if Lk else np.zeros(0, np.int64)
    Ph = np.einsum("lji,lj->li", Rwc_t[host], Pw[lidx] - pwc_t[host])
    lmp_true = np.stack([Ph[:, 0] / Ph[:, 2], Ph[:, 1] / Ph[:, 2], 1.0 / Ph[:, 2]], 1) if Lk else np.zeros((0, 3))
    zh = zl[first] if Lk else np.zeros((0, 2))
    rho0 = lmp_true[:, 2] / (1.0 + rng.normal(0.0, depth_frac, Lk))
    lmp0 = np.stack([(zh[:, 0] - cx) / fx, (zh[:, 1] - cy) / fy, rho0], 1) if Lk else np.zeros((0, 3))
    lm_host = host.astype(np.int64)
    flat_n = 2 * nr
    Rwb_t = Rwc_t @ Rbc.T
    pwb_t = pwc_t - Rwb_t @ pbc
    # initial poses: keyframe 0 at the truth (held), the others perturbed
    Rwb0 = Rwb_t.copy()
    pwb0 = pwb_t.copy()
    for k in range(1, K):
        ax = rng.normal(0.0, 1.0, 3)
        ax /= np.linalg.norm(ax)
        Rwb0[k] = Rwb_t[k] @ so3_exp(ax * math.radians(pose_deg))
        d = rng.normal(0.0, 1.0, 3)
        pwb0[k] = pwb_t[k] + pose_m * d / np.linalg.norm(d)
    rho_meas, rho_isig = np.zeros(Lk), np.zeros(Lk)
    if depth_prior > 0 and Lk:
        rho_meas = lmp_true[:, 2] * (1.0 + depth_prior * rng.normal(0.0, 1.0, Lk))
        rho_isig = 1.0 / (depth_prior * lmp_true[:, 2])
    return Window(Rwb=np.ascontiguousarray(Rwb0), pwb=np.ascontiguousarray(pwb0), Rbc=Rbc, pbc=pbc,
                  lmp=np.ascontiguousarray(lmp0.reshape(-1, 3)), lm_host=lm_host, lm_mask=np.ones(Lk, np.bool_),
                  rho_meas=rho_meas, rho_isig=rho_isig, ob_start=ob_start, ob_pose=ob_pose, ob_cam=ob_cam,
                  ob_z=np.ascontiguousarray(ob_z), ob_isig=np.full(flat_n, 1.0 / px_noise),
                  ob_valid=np.ones(flat_n, np.bool_), fx=float(fx), fy=float(fy), cx=float(cx), cy=float(cy),
                  B=float(B), huber_k=HUBER_K, Rwb_true=Rwb_t, pwb_true=pwb_t,
                  lmp_true=np.ascontiguousarray(lmp_true.reshape(-1, 3)))


def config0_window(seed=0):
    """One window: 10 keyframes, 1,500 landmarks at 2-20 m seen by 2-6 keyframes, 1 px noise, 5 % outliers."""
    return make_window(seed, K=10, L=1500, obs_min=2, obs_max=6)


def config2_windows(n=256, seed=1):
    """Uneven windows: K ~ U{5..20}, L ~ U{300..3000}, 2-12 observing keyframes per landmark (geometric)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        K = int(rng.integers(5, 21))
        L = int(rng.integers(300, 3001))
        out.append(make_window(None, K=K, L=L, obs_min=2, obs_max=12, geometric=True, rng=np.random.default_rng(
            [seed, i])))
    return out


def config3_windows(n=64, seed=3):
    """Differentiable-BA batch: 10 keyframes, 2,000 landmarks seen by 2-6 keyframes, 1 px noise, 5 % outliers."""
    return [make_window(None, K=10, L=2000, obs_min=2, obs_max=6, rng=np.random.default_rng([seed, i]))
            for i in range(n)]


def config4_windows(n=32, seed=4):
    """Large windows: 20 keyframes, 6,000 landmarks seen by 3-15 keyframes, 10 % outliers."""
    return [make_window(None, K=20, L=6000, obs_min=3, obs_max=15, outlier_frac=0.10, step_m=0.15,
                        rng=np.random.default_rng([seed, i])) for i in range(n)]
