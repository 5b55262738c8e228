"""Oracle (test infrastructure only): float64 numpy restatement of the reference's local bundle adjustment.

Covers src/xclean/backend/ba.py's CPU solvers (_solve_np, ba.py:713-874; _solve_np_id, ba.py:1212-1342; the
analytic inverse-depth blocks, ba.py:1153-1209; the gyro rotation factors, ba.py:644-697; _free_mask, ba.py:700-710;
build_pairs, ba.py:902-927) and, stage by stage, the arithmetic of the CUDA kernels in src/xclean/backend/kernels.py
(build_blocks :45-114, depth_prior :135-166, inv3_damped :169-191, schur_pairs :203-232, schur_grad :235-258,
pose_blocks :261-285, chol_solve :291-346, backsub :349-374, build_blocks_id :417-580, landmark_prior_id :599-643,
pose_blocks_id :646-680, schur_pairs_id :683-717, schur_grad_id :720-745, backsub_id :748-775) in float64.

The Lie-group helpers restate src/xclean/core/lie.py (Rodrigues with Taylor series below 0.126 rad, the left Jacobian
V, quaternion logarithm, SVD projection).  Pinned against outputs of the reference itself in
tests/golden/lba_golden.npz (tests/golden/make_golden_lba.py).  Only tests and the benchmark's CPU leg use this file.
"""
from __future__ import annotations

import numpy as np

HUBER_K = 1.345
D_POSE = 6
_TAYLOR = 0.126


# ------------------------------------------------------------------------------------------------------ Lie group
def hat(v):
    v = np.asarray(v, np.float64)
    K = np.zeros(v.shape[:-1] + (3, 3))
    K[..., 0, 1], K[..., 0, 2] = -v[..., 2], v[..., 1]
    K[..., 1, 0], K[..., 1, 2] = v[..., 2], -v[..., 0]
    K[..., 2, 0], K[..., 2, 1] = -v[..., 1], v[..., 0]
    return K


def _coeffs(t2):
    """sin t / t, (1 - cos t) / t^2, (t - sin t) / t^3, with their series below 0.126 rad."""
    t2 = np.asarray(t2, np.float64)
    t = np.sqrt(t2)
    small = t < _TAYLOR
    ts = np.where(small, 1.0, t)
    a = np.where(small, 1 - t2 / 6 + t2 ** 2 / 120 - t2 ** 3 / 5040, np.sin(ts) / ts)
    b = np.where(small, 0.5 - t2 / 24 + t2 ** 2 / 720 - t2 ** 3 / 40320, (1 - np.cos(ts)) / np.where(small, 1.0, t2))
    c = np.where(small, 1 / 6 - t2 / 120 + t2 ** 2 / 5040 - t2 ** 3 / 362880,
                 (ts - np.sin(ts)) / np.where(small, 1.0, t2 * ts))
    return a, b, c


def so3_exp(phi):
    phi = np.asarray(phi, np.float64)
    a, b, _c = _coeffs(np.sum(phi * phi, -1))
    K = hat(phi)
    return np.eye(3) + a[..., None, None] * K + b[..., None, None] * (K @ K)


def se3_exp(xi):
    """[rho (translation), phi (rotation)] -> 4x4."""
    xi = np.asarray(xi, np.float64)
    rho, phi = xi[..., :3], xi[..., 3:]
    a, b, c = _coeffs(np.sum(phi * phi, -1))
    K = hat(phi)
    KK = K @ K
    R = np.eye(3) + a[..., None, None] * K + b[..., None, None] * KK
    V = np.eye(3) + b[..., None, None] * K + c[..., None, None] * KK
    T = np.zeros(xi.shape[:-1] + (4, 4))
    T[..., :3, :3] = R
    T[..., :3, 3] = np.einsum("...ij,...j->...i", V, rho)
    T[..., 3, 3] = 1.0
    return T


def se3_inv(T):
    T = np.asarray(T, np.float64)
    out = np.zeros_like(T)
    Rt = np.swapaxes(T[..., :3, :3], -1, -2)
    out[..., :3, :3] = Rt
    out[..., :3, 3] = -np.einsum("...ij,...j->...i", Rt, T[..., :3, 3])
    out[..., 3, 3] = 1.0
    return out


def so3_project(R):
    R = np.asarray(R, np.float64)
    U, _s, Vt = np.linalg.svd(R)
    D = np.eye(3) * np.ones(R.shape[:-2] + (1, 1))
    D[..., 2, 2] = np.sign(np.linalg.det(U @ Vt))
    return U @ D @ Vt


def _quat(R):
    """Unit quaternion [w, x, y, z] by the branch of the largest of (trace, R00, R11, R22); w >= 0."""
    R = np.asarray(R, np.float64)
    tr = R[..., 0, 0] + R[..., 1, 1] + R[..., 2, 2]
    q = np.zeros(R.shape[:-2] + (4,))
    which = np.argmax(np.stack([tr, R[..., 0, 0], R[..., 1, 1], R[..., 2, 2]], -1), -1)
    which = np.where(tr > 0, 0, np.maximum(which, 1))
    b = which == 0
    if b.any():
        t = 2.0 * np.sqrt(np.maximum(tr[b] + 1.0, 0.0))
        q[b, 0] = 0.25 * t
        q[b, 1] = (R[b, 2, 1] - R[b, 1, 2]) / t
        q[b, 2] = (R[b, 0, 2] - R[b, 2, 0]) / t
        q[b, 3] = (R[b, 1, 0] - R[b, 0, 1]) / t
    for k, (a, c, d) in enumerate(((0, 1, 2), (1, 2, 0), (2, 0, 1)), start=1):
        b = which == k
        if not b.any():
            continue
        t = 2.0 * np.sqrt(np.maximum(1.0 + R[b, a, a] - R[b, c, c] - R[b, d, d], 0.0))
        q[b, 0] = (R[b, d, c] - R[b, c, d]) / t
        q[b, 1 + a] = 0.25 * t
        q[b, 1 + c] = (R[b, c, a] + R[b, a, c]) / t
        q[b, 1 + d] = (R[b, d, a] + R[b, a, d]) / t
    q[q[..., 0] < 0] *= -1.0
    return q


def so3_log(R):
    q = _quat(R)
    v = q[..., 1:]
    nv = np.linalg.norm(v, axis=-1)
    th = 2.0 * np.arctan2(nv, q[..., 0])
    s = np.where(nv < 3.65e-8, 2.0, th / np.where(nv < 3.65e-8, 1.0, nv))
    return v * s[..., None]


def so3_jr_inv(phi):
    """I + 1/2 hat(phi) + k hat(phi)^2 (the inverse left Jacobian at -phi)."""
    phi = np.atleast_2d(np.asarray(phi, np.float64))
    t2 = np.sum(phi * phi, -1)
    t = np.sqrt(t2)
    small = t < _TAYLOR
    ts = np.where(small, 1.0, t)
    k = np.where(small, 1 / 12 + t2 / 720 + t2 ** 2 / 30240 + t2 ** 3 / 1209600,
                 (1 - ts * np.sin(ts) / (2 * (1 - np.cos(ts)))) / np.where(small, 1.0, t2))
    K = hat(phi)
    return np.eye(3) + 0.5 * K + k[..., None, None] * (K @ K)


# --------------------------------------------------------------------------------------------------- solver helpers
def free_mask(free, nk):
    """ba.py:700-710: a boolean mask, or the index of the one held keyframe."""
    if np.ndim(free) == 0:
        m = np.ones(nk, bool)
        m[int(free)] = False
        return m
    return np.asarray(free, bool)


def huber_w(e, k=HUBER_K):
    return np.where(e <= k, 1.0, k / np.maximum(e, 1e-9))


def build_pairs(olm_sorted, nl):
    """ba.py:902-927: CSR starts and every ordered observation pair inside each landmark's segment."""
    counts = np.bincount(olm_sorted, minlength=nl).astype(np.int64)
    offs = np.zeros(nl + 1, np.int64)
    offs[1:] = np.cumsum(counts)
    pa, pb = [], []
    for l in range(nl):
        idx = np.arange(offs[l], offs[l + 1])
        pa.append(np.repeat(idx, len(idx)))
        pb.append(np.tile(idx, len(idx)))
    cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
    return offs.astype(np.int32), cat(pa), cat(pb)


def rot_factor_blocks(T_cw, factors, d, n):
    """ba.py:644-697: e = log(M^T R_a R_b^T), J_a = Jr^-1(e) (R_a R_b^T)^T / sigma, J_b = -Jr^-1(e) / sigma."""
    H = np.zeros((n, n))
    g = np.zeros(n)
    if not factors:
        return H, g, 0.0
    chi = 0.0
    for a, b, M, sig in factors:
        w = 1.0 / max(float(sig), 1e-9)
        A = T_cw[a, :3, :3] @ T_cw[b, :3, :3].T
        e = so3_log(np.asarray(M).T @ A)
        Jr = so3_jr_inv(e)[0]
        Ja = w * Jr @ A.T
        Jb = -w * Jr
        r = w * e
        chi += float(r @ r)
        ia, ib = a * d + 3, b * d + 3
        H[ia:ia + 3, ia:ia + 3] += Ja.T @ Ja
        H[ia:ia + 3, ib:ib + 3] += Ja.T @ Jb
        H[ib:ib + 3, ia:ia + 3] += Jb.T @ Ja
        H[ib:ib + 3, ib:ib + 3] += Jb.T @ Jb
        g[ia:ia + 3] -= Ja.T @ r
        g[ib:ib + 3] -= Jb.T @ r
    return H, g, chi


def _hold(Hred, bp, free, d):
    for i in np.nonzero(~free)[0]:
        f0 = i * d
        Hred[f0:f0 + d, :] = 0.0
        Hred[:, f0:f0 + d] = 0.0
        Hred[f0:f0 + d, f0:f0 + d] = np.eye(d)
        bp[f0:f0 + d] = 0.0


# ------------------------------------------------------------------------------------------- Euclidean CPU solver
def solve_np(poses, pts, okf, olm, ouv, fx, cx, cy, free, iters, lam0=1e-4, prior=None, rotf=None):
    """ba.py:713-874 (_solve_np): Euclidean points, left pose perturbation T_cw <- exp(xi) T_cw, Huber IRLS,
    landmark blocks damped by lam * max(tr / 3, 1e-9), dense reduced system damped by lam * max(diag, 1e-9),
    accept if the plain chi does not grow (lam / 2, floor 1e-7) else lam x 4 (cap 1e2)."""
    okf = np.asarray(okf, np.int64)
    olm = np.asarray(olm, np.int64)
    ouv = np.asarray(ouv, np.float64)
    nk, nl = len(poses), len(pts)
    d, n = D_POSE, D_POSE * nk
    free = free_mask(free, nk)
    lam = lam0
    T_cw = se3_inv(np.asarray(poses, np.float64))
    pts = np.array(pts, np.float64)

    def resid(T_cw, pts):
        Pc = np.einsum("nij,nj->ni", T_cw[okf, :3, :3], pts[olm]) + T_cw[okf, :3, 3]
        z = np.maximum(Pc[:, 2], 1e-6)
        return np.stack([fx * Pc[:, 0] / z + cx, fx * Pc[:, 1] / z + cy], 1) - ouv, Pc

    r0, _ = resid(T_cw, pts)
    rms0 = float(np.sqrt(np.mean(np.sum(r0 ** 2, 1))))
    chi0 = float(np.sum(r0 ** 2))
    for _ in range(iters):
        r, Pc = resid(T_cw, pts)
        sw = np.sqrt(huber_w(np.linalg.norm(r, axis=1)))[:, None]
        x, y, z = Pc[:, 0], Pc[:, 1], np.maximum(Pc[:, 2], 1e-6)
        iz = 1.0 / z
        A = np.zeros((len(r), 2, 3))
        A[:, 0, 0] = A[:, 1, 1] = fx * iz
        A[:, 0, 2] = -fx * x * iz * iz
        A[:, 1, 2] = -fx * y * iz * iz
        dP = np.zeros((len(r), 3, 6))
        dP[:, 0, 0] = dP[:, 1, 1] = dP[:, 2, 2] = 1.0
        dP[:, :, 3:] = -hat(np.stack([x, y, z], 1))
        Jp = np.einsum("nij,njk->nik", A, dP) * sw[:, :, None]
        Jl = np.einsum("nij,njk->nik", A, T_cw[okf, :3, :3]) * sw[:, :, None]
        rw = r * sw
        Hll = np.zeros((nl, 3, 3))
        bl = np.zeros((nl, 3))
        np.add.at(Hll, olm, np.einsum("nri,nrj->nij", Jl, Jl))
        np.add.at(bl, olm, -np.einsum("nri,nr->ni", Jl, rw))
        Hpl = np.einsum("nri,nrj->nij", Jp, Jl)
        Hpp = np.zeros((n, n))
        bp = np.zeros(n)
        blk = np.einsum("nri,nrj->nij", Jp, Jp)
        gp = -np.einsum("nri,nr->ni", Jp, rw)
        for o in range(len(r)):
            k0 = okf[o] * d
            Hpp[k0:k0 + d, k0:k0 + d] += blk[o]
            bp[k0:k0 + d] += gp[o]
        if prior is not None:
            c, rho0, invsig, valid = prior
            dPp = pts - c
            dist = np.linalg.norm(dPp, axis=1)
            ok = (np.asarray(valid) > 0.5) & (dist > 1e-6)
            rho = np.where(ok, 1.0 / np.where(ok, dist, 1.0), 0.0)
            rp = (rho - rho0) * invsig
            swp = np.sqrt(huber_w(np.abs(rp)))
            gg = np.where(ok, -rho ** 2 / np.where(ok, dist, 1.0) * invsig, 0.0)
            Jpr = dPp * (gg * swp)[:, None]
            Jpr[~ok] = 0.0
            rpw = np.where(ok, rp * swp, 0.0)
            Hll += np.einsum("ni,nj->nij", Jpr, Jpr)
            bl -= Jpr * rpw[:, None]
        Hll += lam * np.maximum(np.trace(Hll, axis1=1, axis2=2) / 3.0, 1e-9)[:, None, None] * np.eye(3)
        Hlli = np.linalg.inv(Hll)
        T3 = np.einsum("nij,njk->nik", Hpl, Hlli[olm])
        Hred = Hpp.copy()
        for l in range(nl):
            obs = np.nonzero(olm == l)[0]
            for i in obs:
                ki = okf[i] * d
                bp[ki:ki + d] -= T3[i] @ bl[l]
                for j in obs:
                    kj = okf[j] * d
                    Hred[ki:ki + d, kj:kj + d] -= T3[i] @ Hpl[j].T
        if rotf:
            Hr, gr, _ = rot_factor_blocks(T_cw, rotf, d, n)
            Hpp += Hr      # ba.py adds the rotation factors to Hpp after Hred was copied from it
            bp += gr
        _hold(Hred, bp, free, d)
        Hred[np.arange(n), np.arange(n)] += lam * np.maximum(np.diag(Hred), 1e-9)
        try:
            dxp = np.linalg.solve(Hred, bp)
        except np.linalg.LinAlgError:
            break
        rhs = bl.copy()
        np.add.at(rhs, olm, -np.einsum("nij,ni->nj", Hpl, dxp.reshape(nk, d)[okf]))
        dxl = np.einsum("nij,nj->ni", Hlli, rhs)
        T_new = T_cw.copy()
        for i in np.nonzero(free)[0]:
            T_new[i] = se3_exp(dxp[i * d:(i + 1) * d]) @ T_cw[i]
            T_new[i][:3, :3] = so3_project(T_new[i][:3, :3])
        pts_new = pts + dxl
        r2, _ = resid(T_new, pts_new)
        if np.sum(r2 ** 2) <= np.sum(r ** 2):
            T_cw, pts = T_new, pts_new
            lam = max(lam * 0.5, 1e-7)
        else:
            lam = min(lam * 4.0, 1e2)
    rn, _ = resid(T_cw, pts)
    return se3_inv(T_cw), pts, {"chi2_0": chi0, "chi2_n": float(np.sum(rn ** 2)), "rms_0": rms0,
                                "rms_n": float(np.sqrt(np.mean(np.sum(rn ** 2, 1))))}


# --------------------------------------------------------------------------------------- inverse-depth CPU solver
def host_frames(poses, hidx, hpose_ext):
    """ba.py:1116-1136: host T_wc per landmark, from the window (hidx >= 0) or the carried constant."""
    hidx = np.asarray(hidx, np.int64)
    nl = len(hidx)
    ext = np.asarray(hpose_ext, np.float64).reshape(nl, 3, 4)
    R = ext[:, :, :3].copy()
    t = ext[:, :, 3].copy()
    inw = hidx >= 0
    R[inw] = poses[hidx[inw], :3, :3]
    t[inw] = poses[hidx[inw], :3, 3]
    return R, t


def analytic_blocks_id(poses, T_cw, rho, mbear, hidx, hpose_ext, okf, olm, ouv, fx, cx, cy, sw=None):
    """ba.py:1153-1209: observer block A [I | -hat(Pc)], host block A R_ch [-I | hat(Ph)] (zero for an
    out-of-window host), landmark block for (x_n, y_n, rho), residual."""
    okf = np.asarray(okf, np.int64)
    olm = np.asarray(olm, np.int64)
    hidx = np.asarray(hidx, np.int64)
    N = len(okf)
    Rh, th = host_frames(poses, hidx, hpose_ext)
    Ph = mbear / np.maximum(rho, 1e-12)[:, None]
    Pw = np.einsum("nij,nj->ni", Rh, Ph) + th
    Pc = np.einsum("nij,nj->ni", T_cw[okf, :3, :3], Pw[olm]) + T_cw[okf, :3, 3]
    z = np.maximum(Pc[:, 2], 1e-6)
    r = np.stack([fx * Pc[:, 0] / z + cx, fx * Pc[:, 1] / z + cy], 1) - ouv
    iz = 1.0 / z
    A = np.zeros((N, 2, 3))
    A[:, 0, 0] = A[:, 1, 1] = fx * iz
    A[:, 0, 2] = -fx * Pc[:, 0] * iz * iz
    A[:, 1, 2] = -fx * Pc[:, 1] * iz * iz
    dPo = np.zeros((N, 3, 6))
    dPo[:, 0, 0] = dPo[:, 1, 1] = dPo[:, 2, 2] = 1.0
    dPo[:, :, 3:] = -hat(np.stack([Pc[:, 0], Pc[:, 1], z], 1))
    Jobs = np.einsum("nij,njk->nik", A, dPo)
    ARch = np.einsum("nij,njk->nik", A, np.einsum("nij,njk->nik", T_cw[okf, :3, :3], Rh[olm]))
    Pho = Ph[olm]
    dPh = np.zeros((N, 3, 6))
    dPh[:, 0, 0] = dPh[:, 1, 1] = dPh[:, 2, 2] = -1.0
    dPh[:, :, 3:] = hat(Pho)
    Jhost = np.einsum("nij,njk->nik", ARch, dPh)
    Jhost[hidx[olm] < 0] = 0.0
    irho = 1.0 / np.maximum(rho[olm], 1e-12)
    Jlm = np.empty((N, 2, 3))
    Jlm[:, :, 0] = ARch[:, :, 0] * irho[:, None]
    Jlm[:, :, 1] = ARch[:, :, 1] * irho[:, None]
    Jlm[:, :, 2] = -np.einsum("nqk,nk->nq", ARch, Pho) * irho[:, None]
    if sw is not None:
        Jobs, Jhost, Jlm = Jobs * sw[:, :, None], Jhost * sw[:, :, None], Jlm * sw[:, :, None]
    return Jobs, Jhost, Jlm, r


def solve_np_id(poses, rho, mbear, hidx, hpose_ext, okf, olm, ouv, fx, cx, cy, free, iters, lam0=1e-4,
                prior=None, rotf=None, rho_floor=1e-4):
    """ba.py:1212-1342 (_solve_np_id): host-anchored inverse depth, two pose blocks per observation."""
    okf = np.asarray(okf, np.int64)
    olm = np.asarray(olm, np.int64)
    ouv = np.asarray(ouv, np.float64)
    nk, nl = len(poses), len(rho)
    d, n = D_POSE, D_POSE * nk
    free = free_mask(free, nk)
    lam = lam0
    poses = np.array(poses, np.float64)
    rho = np.array(rho, np.float64)
    mbear = np.array(mbear, np.float64)
    hidx = np.asarray(hidx, np.int64)
    T_cw = se3_inv(poses)
    kslot = np.stack([okf, hidx[olm]], 1)

    def resid(poses, T_cw, rho, mbear):
        Rh, th = host_frames(poses, hidx, hpose_ext)
        Pw = np.einsum("nij,nj->ni", Rh, mbear / np.maximum(rho, 1e-12)[:, None]) + th
        Pc = np.einsum("nij,nj->ni", T_cw[okf, :3, :3], Pw[olm]) + T_cw[okf, :3, 3]
        z = np.maximum(Pc[:, 2], 1e-6)
        return np.stack([fx * Pc[:, 0] / z + cx, fx * Pc[:, 1] / z + cy], 1) - ouv

    r0 = resid(poses, T_cw, rho, mbear)
    rms0 = float(np.sqrt(np.mean(np.sum(r0 ** 2, 1))))
    chi0 = float(np.sum(r0 ** 2))
    for _ in range(iters):
        r = resid(poses, T_cw, rho, mbear)
        sw = np.sqrt(huber_w(np.linalg.norm(r, axis=1)))[:, None]
        Jobs, Jhost, Jlm, _r = analytic_blocks_id(poses, T_cw, rho, mbear, hidx, hpose_ext, okf, olm, ouv, fx, cx,
                                                  cy, sw=sw)
        rw = r * sw
        Jp = np.stack([Jobs, Jhost], 1)
        Hll = np.zeros((nl, 3, 3))
        bl = np.zeros((nl, 3))
        np.add.at(Hll, olm, np.einsum("nqa,nqb->nab", Jlm, Jlm))
        np.add.at(bl, olm, -np.einsum("nqa,nq->na", Jlm, rw))
        Hpl = np.einsum("nsqa,nqc->nsac", Jp, Jlm)
        if prior is not None:
            m0, rho0, wbear, invsig, valid = prior
            ok = np.asarray(valid) > 0.5
            rp = np.stack([(mbear[:, 0] - m0[:, 0]) * wbear, (mbear[:, 1] - m0[:, 1]) * wbear,
                           (rho - rho0) * invsig], 1)
            J0 = np.stack([wbear, wbear, invsig], 1)
            swp = np.sqrt(huber_w(np.abs(rp)))
            swp[:, :2] = 1.0
            Jpr = J0 * swp
            for c in range(3):
                Hll[ok, c, c] += (Jpr[:, c] ** 2)[ok]
            bl[ok] -= (Jpr * rp * swp)[ok]
        Hpp = np.zeros((n, n))
        grad = np.zeros(n)
        U = np.zeros((n, nl, 3))
        for o in range(len(r)):
            for sa in range(2):
                ka = kslot[o, sa]
                if ka < 0:
                    continue
                grad[ka * d:(ka + 1) * d] -= Jp[o, sa].T @ rw[o]
                U[ka * d:(ka + 1) * d, olm[o]] += Hpl[o, sa]
                for sb in range(2):
                    kb = kslot[o, sb]
                    if kb >= 0:
                        Hpp[ka * d:(ka + 1) * d, kb * d:(kb + 1) * d] += Jp[o, sa].T @ Jp[o, sb]
        if rotf:
            Hr, gr, _ = rot_factor_blocks(T_cw, rotf, d, n)
            Hpp += Hr
            grad += gr
        Hd = Hll + lam * np.maximum(np.trace(Hll, axis1=1, axis2=2) / 3.0, 1e-9)[:, None, None] * np.eye(3)
        Hlli = np.linalg.inv(Hd)
        T3 = np.einsum("alc,lcd->ald", U, Hlli)
        Hred = Hpp - np.einsum("ald,bld->ab", T3, U)
        bp = grad - np.einsum("ald,ld->a", T3, bl)
        _hold(Hred, bp, free, d)
        Hred[np.arange(n), np.arange(n)] += lam * np.maximum(np.diag(Hred), 1e-9)
        try:
            dxp = np.linalg.solve(Hred, bp)
        except np.linalg.LinAlgError:
            break
        dxl = np.einsum("lcd,ld->lc", Hlli, bl - np.einsum("alc,a->lc", U, dxp))
        T_new = T_cw.copy()
        if free.any():
            T_new[free] = se3_exp(dxp.reshape(nk, d)[free]) @ T_cw[free]
            T_new[free, :3, :3] = so3_project(T_new[free, :3, :3])
        m_new = mbear.copy()
        m_new[:, :2] += dxl[:, :2]
        rho_new = np.maximum(rho + dxl[:, 2], rho_floor)
        p_new = se3_inv(T_new)
        r2 = resid(p_new, T_new, rho_new, m_new)
        if np.sum(r2 ** 2) <= np.sum(r ** 2):
            T_cw, poses, rho, mbear = T_new, p_new, rho_new, m_new
            lam = max(lam * 0.5, 1e-7)
        else:
            lam = min(lam * 4.0, 1e2)
    rn = resid(poses, T_cw, rho, mbear)
    return poses, rho, mbear, {"chi2_0": chi0, "chi2_n": float(np.sum(rn ** 2)), "rms_0": rms0,
                               "rms_n": float(np.sqrt(np.mean(np.sum(rn ** 2, 1))))}


# ------------------------------------------------------------------------------- stage kernels, float64 numpy
def k_build_blocks(Tcw, pts, okf, olm, ouv, fx, cx, cy, huber, nl):
    """kernels.py:45-114 -> Jpose (N,2,6), Jlm (N,2,3), resw (N,2), Hll (nl,9), bl (nl,3), Hpl (N,6,3)."""
    T = np.asarray(Tcw, np.float64).reshape(-1, 3, 4)
    okf, olm = np.asarray(okf, np.int64), np.asarray(olm, np.int64)
    Pc = np.einsum("nij,nj->ni", T[okf, :, :3], np.asarray(pts, np.float64)[olm]) + T[okf, :, 3]
    z = np.maximum(Pc[:, 2], 1e-6)
    r = np.stack([fx * Pc[:, 0] / z + cx, fx * Pc[:, 1] / z + cy], 1) - ouv
    sw = np.sqrt(huber_w(np.linalg.norm(r, axis=1), huber))
    A = np.zeros((len(okf), 2, 3))
    A[:, 0, 0] = A[:, 1, 1] = fx / z
    A[:, 0, 2] = -fx * Pc[:, 0] / z ** 2
    A[:, 1, 2] = -fx * Pc[:, 1] / z ** 2
    dP = np.zeros((len(okf), 3, 6))
    dP[:, 0, 0] = dP[:, 1, 1] = dP[:, 2, 2] = 1.0
    dP[:, :, 3:] = -hat(np.stack([Pc[:, 0], Pc[:, 1], z], 1))
    Jp = np.einsum("nij,njk->nik", A, dP) * sw[:, None, None]
    Jl = np.einsum("nij,njk->nik", A, T[okf, :, :3]) * sw[:, None, None]
    rw = r * sw[:, None]
    Hll = np.zeros((nl, 3, 3))
    bl = np.zeros((nl, 3))
    np.add.at(Hll, olm, np.einsum("nqa,nqb->nab", Jl, Jl))
    np.add.at(bl, olm, -np.einsum("nqa,nq->na", Jl, rw))
    return dict(Jpose=Jp, Jlm=Jl, resw=rw, Hll=Hll.reshape(nl, 9), bl=bl,
                Hpl=np.einsum("nqa,nqb->nab", Jp, Jl))


def k_depth_prior(pts, chost, rho0, invsig, valid, huber):
    """kernels.py:135-166 -> Hll (nl,9), bl (nl,3) contributions."""
    nl = len(pts)
    dP = np.asarray(pts, np.float64) - chost
    d2 = np.sum(dP * dP, 1)
    ok = (np.asarray(valid) >= 0.5) & (d2 >= 1e-12)
    dist = np.sqrt(np.where(ok, d2, 1.0))
    rho = 1.0 / dist
    r = (rho - rho0) * invsig
    sw = np.sqrt(huber_w(np.abs(r), huber))
    J = (-rho * rho / dist * invsig * sw)[:, None] * dP
    J[~ok] = 0.0
    rw = np.where(ok, r * sw, 0.0)
    return np.einsum("na,nb->nab", J, J).reshape(nl, 9), -J * rw[:, None]


def k_inv3_damped(Hll, lam):
    """kernels.py:169-191."""
    H = np.asarray(Hll, np.float64).reshape(-1, 3, 3)
    dmp = lam * np.maximum(np.trace(H, axis1=1, axis2=2) / 3.0, 1e-9)
    return np.linalg.inv(H + dmp[:, None, None] * np.eye(3)).reshape(-1, 9)


def k_schur_pairs(Hpl, Hlli, okf, olm, pa, pb, n, d=6):
    """kernels.py:203-232 -> the contribution to Hred."""
    H = np.zeros((n, n))
    Hpl = np.asarray(Hpl, np.float64).reshape(-1, d, 3)
    Hi = np.asarray(Hlli, np.float64).reshape(-1, 3, 3)
    for oi, oj in zip(pa, pb):
        ki, kj = okf[oi] * d, okf[oj] * d
        H[ki:ki + d, kj:kj + d] -= Hpl[oi] @ Hi[olm[oi]] @ Hpl[oj].T
    return H


def k_schur_grad(Hpl, Hlli, bl, okf, olm, n, d=6):
    """kernels.py:235-258."""
    g = np.zeros(n)
    Hpl = np.asarray(Hpl, np.float64).reshape(-1, d, 3)
    Hi = np.asarray(Hlli, np.float64).reshape(-1, 3, 3)
    for o in range(len(okf)):
        g[okf[o] * d:(okf[o] + 1) * d] -= Hpl[o] @ Hi[olm[o]] @ bl[olm[o]]
    return g


def k_pose_blocks(Jp, res, kf, n, r=2, d=6):
    """kernels.py:261-285."""
    H = np.zeros((n, n))
    g = np.zeros(n)
    J = np.asarray(Jp, np.float64).reshape(-1, r, d)
    res = np.asarray(res, np.float64).reshape(-1, r)
    for o in range(len(kf)):
        k = kf[o]
        if k < 0:
            continue
        H[k * d:(k + 1) * d, k * d:(k + 1) * d] += J[o].T @ J[o]
        g[k * d:(k + 1) * d] -= J[o].T @ res[o]
    return H, g


def k_chol_solve(H, b):
    """kernels.py:291-346 for a positive definite H -> (lower factor, solution)."""
    L = np.linalg.cholesky(np.asarray(H, np.float64))
    return L, np.linalg.solve(L.T, np.linalg.solve(L, b))


def k_backsub(Hpl, Hlli, bl, dxp, okf, offs, d=6):
    """kernels.py:349-374."""
    nl = len(offs) - 1
    Hpl = np.asarray(Hpl, np.float64).reshape(-1, d, 3)
    Hi = np.asarray(Hlli, np.float64).reshape(-1, 3, 3)
    out = np.zeros((nl, 3))
    for l in range(nl):
        rhs = np.array(bl[l], np.float64)
        for s in range(offs[l], offs[l + 1]):
            rhs -= Hpl[s].T @ dxp[okf[s] * d:(okf[s] + 1) * d]
        out[l] = Hi[l] @ rhs
    return out


def k_build_blocks_id(Tcw, hpose, hidx, mbear, rhov, okf, olm, ouv, fx, cx, cy, huber, nl):
    """kernels.py:417-580 -> Jp (N,2,2,6), resw, kslot (N,2), Hll (nl,9), bl (nl,3), Hpl (N,2,6,3)."""
    T = np.zeros((len(np.asarray(Tcw).reshape(-1, 12)), 4, 4))
    T[:, :3, :] = np.asarray(Tcw, np.float64).reshape(-1, 3, 4)
    T[:, 3, 3] = 1.0
    poses = se3_inv(T)
    okf, olm = np.asarray(okf, np.int64), np.asarray(olm, np.int64)
    rho = np.asarray(rhov, np.float64)
    mb = np.asarray(mbear, np.float64)
    Jobs, Jhost, Jlm, r = analytic_blocks_id(poses, T, rho, mb, hidx, hpose, okf, olm, ouv, fx, cx, cy)
    sw = np.sqrt(huber_w(np.linalg.norm(r, axis=1), huber))[:, None]
    Jobs, Jhost, Jlm, rw = Jobs * sw[:, :, None], Jhost * sw[:, :, None], Jlm * sw[:, :, None], r * sw
    Jp = np.stack([Jobs, Jhost], 1)
    Hll = np.zeros((nl, 3, 3))
    bl = np.zeros((nl, 3))
    np.add.at(Hll, olm, np.einsum("nqa,nqb->nab", Jlm, Jlm))
    np.add.at(bl, olm, -np.einsum("nqa,nq->na", Jlm, rw))
    kslot = np.stack([okf, np.asarray(hidx, np.int64)[olm]], 1)
    return dict(Jp=Jp, resw=rw, kslot=kslot, Hll=Hll.reshape(nl, 9), bl=bl,
                Hpl=np.einsum("nsqa,nqc->nsac", Jp, Jlm))


def k_landmark_prior_id(mb, rhov, m0, rho0, invsig, wbear, valid, huber):
    """kernels.py:599-643 -> Hll (nl,9), bl (nl,3) contributions (bearing rows not robustified)."""
    nl = len(rhov)
    ok = np.asarray(valid) >= 0.5
    r = np.stack([(mb[:, 0] - m0[:, 0]) * wbear, (mb[:, 1] - m0[:, 1]) * wbear, (rhov - rho0) * invsig], 1)
    sw = np.ones_like(r)
    sw[:, 2] = np.sqrt(huber_w(np.abs(r[:, 2]), huber))
    J = np.stack([wbear, wbear, invsig], 1) * sw
    H = np.zeros((nl, 3, 3))
    for a in range(3):
        H[:, a, a] = J[:, a] ** 2
    b = -J * r * sw
    H[~ok] = 0.0
    b[~ok] = 0.0
    return H.reshape(nl, 9), b


def k_pose_blocks_id(Jp, res, kslot, n, d=6):
    """kernels.py:646-680."""
    H = np.zeros((n, n))
    g = np.zeros(n)
    Jp = np.asarray(Jp, np.float64).reshape(-1, 2, 2, d)
    res = np.asarray(res, np.float64).reshape(-1, 2)
    for o in range(len(Jp)):
        for sa in range(2):
            ka = kslot[o][sa]
            if ka < 0:
                continue
            for sb in range(2):
                kb = kslot[o][sb]
                if kb >= 0:
                    H[ka * d:(ka + 1) * d, kb * d:(kb + 1) * d] += Jp[o, sa].T @ Jp[o, sb]
            g[ka * d:(ka + 1) * d] -= Jp[o, sa].T @ res[o]
    return H, g


def k_schur_pairs_id(Hpl, Hlli, kslot, olm, pa, pb, n, d=6):
    """kernels.py:683-717."""
    H = np.zeros((n, n))
    Hpl = np.asarray(Hpl, np.float64).reshape(-1, 2, d, 3)
    Hi = np.asarray(Hlli, np.float64).reshape(-1, 3, 3)
    for oi, oj in zip(pa, pb):
        for si in range(2):
            ki = kslot[oi][si]
            if ki < 0:
                continue
            for sj in range(2):
                kj = kslot[oj][sj]
                if kj >= 0:
                    H[ki * d:(ki + 1) * d, kj * d:(kj + 1) * d] -= Hpl[oi, si] @ Hi[olm[oi]] @ Hpl[oj, sj].T
    return H


def k_schur_grad_id(Hpl, Hlli, bl, kslot, olm, n, d=6):
    """kernels.py:720-745."""
    g = np.zeros(n)
    Hpl = np.asarray(Hpl, np.float64).reshape(-1, 2, d, 3)
    Hi = np.asarray(Hlli, np.float64).reshape(-1, 3, 3)
    for o in range(len(Hpl)):
        for s in range(2):
            k = kslot[o][s]
            if k >= 0:
                g[k * d:(k + 1) * d] -= Hpl[o, s] @ Hi[olm[o]] @ bl[olm[o]]
    return g


def k_backsub_id(Hpl, Hlli, bl, dxp, kslot, offs, d=6):
    """kernels.py:748-775."""
    nl = len(offs) - 1
    Hpl = np.asarray(Hpl, np.float64).reshape(-1, 2, d, 3)
    Hi = np.asarray(Hlli, np.float64).reshape(-1, 3, 3)
    out = np.zeros((nl, 3))
    for l in range(nl):
        rhs = np.array(bl[l], np.float64)
        for s in range(offs[l], offs[l + 1]):
            for sl in range(2):
                k = kslot[s][sl]
                if k >= 0:
                    rhs -= Hpl[s, sl].T @ dxp[k * d:(k + 1) * d]
        out[l] = Hi[l] @ rhs
    return out


# ------------------------------------------------------------------ the reference's device LM loop, in float64
def solve_gpu_loop(model, poses, lm, okf, olm, ouv, fx, cx, cy, free, iters, lam0=1e-4, prior=None, rotf=None,
                   rho=None, hidx=None, hpose_ext=None, rho_floor=1e-4):
    """The LM schedule of _solve_gpu (ba.py:930-1089, model "euclid") and _solve_gpu_id (ba.py:1345-1497, model
    "id"), restated in float64: chi = sum resw^2 at the head of each iteration; above the previous accepted chi ->
    restore the best state, lam x 4 (cap 1e2), next iteration; otherwise save the state, build the reduced system
    (landmark blocks damped by lam max(tr/3, 1e-9); rotation factors into both the Hessian and the gradient; held
    keyframes -> identity rows; diagonal += lam max(diag, 1e-9)), Cholesky solve, back-substitution; a non-finite
    step -> lam x 10 (cap 1e3); else T_cw <- exp(xi) T_cw for free keyframes, landmarks += step, lam / 2 (floor 1e-7).
    One SO(3) projection at the end, then the final chi.  -> (poses, lm, rho, stats)."""
    okf = np.asarray(okf, np.int64)
    olm = np.asarray(olm, np.int64)
    ouv = np.asarray(ouv, np.float64)
    nk = len(poses)
    nl = len(lm)
    N = len(okf)
    d, n = D_POSE, D_POSE * nk
    freem = free_mask(free, nk)
    T_cw = se3_inv(np.asarray(poses, np.float64))
    lm = np.array(lm, np.float64)
    rho = None if rho is None else np.array(rho, np.float64)
    idm = model == "id"
    lam = lam0
    chi_prev = None
    best = (T_cw.copy(), lm.copy(), None if rho is None else rho.copy(), None)
    rms0 = None

    def build(T_cw, lm, rho, with_prior):
        if idm:
            B = k_build_blocks_id(T_cw[:, :3, :].reshape(nk, 12), hpose_ext, hidx, lm, rho, okf, olm, ouv, fx, cx,
                                  cy, HUBER_K, nl)
            if with_prior and prior is not None:
                m0, rho0, wbear, invsig, valid = prior
                h, b = k_landmark_prior_id(lm, rho, m0, rho0, invsig, wbear, valid, HUBER_K)
                B["Hll"] = B["Hll"] + h
                B["bl"] = B["bl"] + b
        else:
            B = k_build_blocks(T_cw[:, :3, :].reshape(nk, 12), lm, okf, olm, ouv, fx, cx, cy, HUBER_K, nl)
            if with_prior and prior is not None:
                c, rho0, invsig, valid = prior
                h, b = k_depth_prior(lm, c, rho0, invsig, valid, HUBER_K)
                B["Hll"] = B["Hll"] + h
                B["bl"] = B["bl"] + b
        return B

    for _ in range(iters):
        B = build(T_cw, lm, rho, True)
        chi = float(np.sum(B["resw"] ** 2))
        if rms0 is None:
            rms0 = float(np.sqrt(chi / max(N, 1)))
        if chi_prev is not None and chi > chi_prev:
            T_cw, lm = best[0].copy(), best[1].copy()
            rho = None if best[2] is None else best[2].copy()
            lam = min(lam * 4.0, 1e2)
            continue
        chi_prev = chi
        best = (T_cw.copy(), lm.copy(), None if rho is None else rho.copy(), chi)
        Hlli = k_inv3_damped(B["Hll"], lam).reshape(nl, 3, 3)
        Hred = np.zeros((n, n))
        grad = np.zeros(n)
        U = np.zeros((n, nl, 3))
        if idm:
            Jp, Hpl, kslot = B["Jp"], B["Hpl"], B["kslot"]
            entries = [(o, s, kslot[o, s]) for o in range(N) for s in range(2) if kslot[o, s] >= 0]
            for o in range(N):
                for sa in range(2):
                    ka = kslot[o, sa]
                    if ka < 0:
                        continue
                    for sb in range(2):
                        kb = kslot[o, sb]
                        if kb >= 0:
                            Hred[ka * d:(ka + 1) * d, kb * d:(kb + 1) * d] += Jp[o, sa].T @ Jp[o, sb]
                    grad[ka * d:(ka + 1) * d] -= Jp[o, sa].T @ B["resw"][o]
            for o, s, k in entries:
                U[k * d:(k + 1) * d, olm[o]] += Hpl[o, s]
        else:
            Jp, Hpl = B["Jpose"], B["Hpl"]
            for o in range(N):
                k = okf[o]
                Hred[k * d:(k + 1) * d, k * d:(k + 1) * d] += Jp[o].T @ Jp[o]
                grad[k * d:(k + 1) * d] -= Jp[o].T @ B["resw"][o]
                U[k * d:(k + 1) * d, olm[o]] += Hpl[o]
        T3 = np.einsum("alc,lcd->ald", U, Hlli)
        Hred -= np.einsum("ald,bld->ab", T3, U)
        grad -= np.einsum("ald,ld->a", T3, B["bl"])
        if rotf:
            Hr, gr, _ = rot_factor_blocks(T_cw, rotf, d, n)
            Hred += Hr
            grad += gr
        _hold(Hred, grad, freem, d)
        Hred[np.arange(n), np.arange(n)] += lam * np.maximum(np.diag(Hred), 1e-9)
        try:
            L = np.linalg.cholesky(Hred)
            dxp = np.linalg.solve(L.T, np.linalg.solve(L, grad))
        except np.linalg.LinAlgError:
            dxp = np.full(n, np.nan)
        dxl = np.einsum("lcd,ld->lc", Hlli, B["bl"] - np.einsum("alc,a->lc", U, dxp))
        if not (np.isfinite(dxp).all() and np.isfinite(dxl).all()):
            lam = min(lam * 10.0, 1e3)
            continue
        if freem.any():
            T_cw[freem] = se3_exp(dxp.reshape(nk, d)[freem]) @ T_cw[freem]
        if idm:
            lm[:, :2] += dxl[:, :2]
            rho = np.maximum(rho + dxl[:, 2], rho_floor)
        else:
            lm = lm + dxl
        lam = max(lam * 0.5, 1e-7)
    T_cw[:, :3, :3] = so3_project(T_cw[:, :3, :3])
    B = build(T_cw, lm, rho, False)
    chi_n = float(np.sum(B["resw"] ** 2))
    return se3_inv(T_cw), lm, rho, {"chi2_0": best[3] if best[3] else chi_n, "chi2_n": chi_n, "rms_0": rms0,
                                    "rms_n": float(np.sqrt(chi_n / max(N, 1))), "lam": lam}
