"""FP64 autodiff reference for the implicit adjoint of the window solve (test infrastructure only).

The reference has no adjoint; this restates its window cost (src/xclean/vio/window.py: stereo residuals, whitening,
Huber with k = 1.345, inverse-depth prior; the same cost as oracle/ba_oracle.c's visual cost, which is pinned to the
reference) as a torch float64 function of the state x = (per-slot body-pose perturbations [dphi, dp], landmark
(a, b, rho)) and of the parameters theta = (fx, fy, cx, cy, baseline B, the 6-DoF left-to-right extrinsic [omega, t]
at the rectified rig), the per-observation weights 1/sigma and the observed pixels.  The right camera sees
q_r = Exp(omega) q + rho (t - B e_x) (the rectified model is omega = t = 0).  It provides:
  * solve(win, ...)        Newton with the exact Hessian to a gradient of ~1e-13 (the converged state x*), from a
                           start inside the basin of the minimum (e.g. the state window.solve converged to);
  * implicit_grad(...)     dL/dtheta = -(d2C/dtheta dx)^T (d2C/dx2)^-1 dL/dx* by autograd (the FP64 autodiff reference);
  * implicit_grad_schur(...) the same through the Schur complement on the poses, for windows of thousands of
                           landmarks (Hessian-vector products, no dense Hessian), with the gradient's max-norm;
  * fd_grad(...)           central finite differences of L(x*(theta)) with step 1e-6.
The held slot is not a variable; landmarks outside lm_mask or without a valid observation are constants.
"""
from __future__ import annotations

import copy

import numpy as np
import torch

HUBER_K = 1.345
NW_THETA = 11          # fx, fy, cx, cy, B, omega (3), t (3)
f64 = torch.float64


def _hat(v):
    z = torch.zeros_like(v[..., 0])
    return torch.stack([torch.stack([z, -v[..., 2], v[..., 1]], -1), torch.stack([v[..., 2], z, -v[..., 0]], -1),
                        torch.stack([-v[..., 1], v[..., 0], z], -1)], -2)


def _exp(w):
    """Rodrigues for (..., 3), twice differentiable at 0 (series below 1e-4 rad, no sqrt there)."""
    t2 = (w * w).sum(-1)
    small = t2 < 1e-8
    t2s = torch.where(small, torch.ones_like(t2), t2)
    t = torch.sqrt(t2s)
    a = torch.where(small, 1 - t2 / 6 + t2 * t2 / 120, torch.sin(t) / t)
    b = torch.where(small, 0.5 - t2 / 24 + t2 * t2 / 720, (1 - torch.cos(t)) / t2s)
    K = _hat(w)
    return torch.eye(3, dtype=w.dtype) + a[..., None, None] * K + b[..., None, None] * (K @ K)


def _huber(en):
    return torch.where(en <= HUBER_K, 0.5 * en * en, HUBER_K * (en - 0.5 * HUBER_K))


class Window:
    """A window's arrays as float64 torch tensors (a synth_ba.Window or anything with its fields).  const (optional,
    bool per landmark): landmarks held constant (not variables) whose rows stay in the cost."""

    def __init__(self, w, hold=0, const=None):
        g = lambda k: torch.as_tensor(np.array(getattr(w, k), np.float64))
        self.R0, self.p0 = g("Rwb"), g("pwb")
        self.Rbc, self.pbc = g("Rbc"), g("pbc")
        self.l0 = g("lmp")
        self.P, self.L = self.R0.shape[0], self.l0.shape[0]
        self.rho_meas, self.rho_isig = g("rho_meas"), g("rho_isig")
        ob_start = np.asarray(w.ob_start, np.int64)
        lm_of = np.repeat(np.arange(self.L), np.diff(ob_start))
        mask = np.asarray(w.lm_mask, bool)
        valid = np.asarray(w.ob_valid, bool) & mask[lm_of]
        self.sel = torch.as_tensor(np.nonzero(valid)[0])
        self.lm = torch.as_tensor(lm_of[valid])
        self.host = torch.as_tensor(np.asarray(w.lm_host, np.int64)[lm_of[valid]])
        self.tgt = torch.as_tensor(np.asarray(w.ob_pose, np.int64)[valid])
        self.right = torch.as_tensor(np.asarray(w.ob_cam, np.int64)[valid] == 1)
        self.prior = torch.as_tensor(mask & (np.asarray(w.rho_isig) > 0))
        has = np.zeros(self.L, bool)
        has[lm_of[valid]] = True
        self.lvar = torch.as_tensor(mask & has & (~np.asarray(const, bool) if const is not None else True))
        self.pvar = torch.as_tensor(np.array([s != hold for s in range(self.P)]))
        self.theta0 = torch.tensor([w.fx, w.fy, w.cx, w.cy, w.B, 0, 0, 0, 0, 0, 0], dtype=f64)
        self.isig0 = g("ob_isig")
        self.z0 = g("ob_z")

    def n_x(self):
        return 6 * int(self.pvar.sum()) + 3 * int(self.lvar.sum())

    def unpack(self, x):
        npv = int(self.pvar.sum())
        dpose = torch.zeros(self.P, 6, dtype=f64)
        dpose = dpose.index_put((torch.nonzero(self.pvar)[:, 0],), x[:6 * npv].reshape(npv, 6))
        dl = torch.zeros(self.L, 3, dtype=f64)
        dl = dl.index_put((torch.nonzero(self.lvar)[:, 0],), x[6 * npv:].reshape(-1, 3))
        return self.R0 @ _exp(dpose[:, :3]), self.p0 + dpose[:, 3:], self.l0 + dl

    def cost(self, x, theta, isig, z):
        fx, fy, cx, cy, B = theta[0], theta[1], theta[2], theta[3], theta[4]
        R, p, lm = self.unpack(x)
        Rwc = R @ self.Rbc
        pwc = p + R @ self.pbc
        L = lm[self.lm]
        m = torch.stack([L[:, 0], L[:, 1], torch.ones_like(L[:, 0])], 1)
        rho = L[:, 2]
        Rh, Rt = Rwc[self.host], Rwc[self.tgt]
        Y = torch.einsum("nij,nj->ni", Rh, m) + rho[:, None] * (pwc[self.host] - pwc[self.tgt])
        q = torch.einsum("nji,nj->ni", Rt, Y)
        tlr = theta[8:11] - torch.stack([B, torch.zeros_like(B), torch.zeros_like(B)])
        qr = q @ _exp(theta[5:8]).T + rho[:, None] * tlr
        qq = torch.where(self.right[:, None], qr, q)
        s = isig[self.sel]
        zz = z[self.sel]
        e0 = (fx * qq[:, 0] / qq[:, 2] + cx - zz[:, 0]) * s
        e1 = torch.where(self.right, torch.zeros_like(e0), (fy * q[:, 1] / q[:, 2] + cy - zz[:, 1]) * s)
        en2 = e0 * e0 + e1 * e1
        en = torch.sqrt(torch.where(en2 > 0, en2, torch.ones_like(en2)))
        c = torch.where(en2 > 0, _huber(en), torch.zeros_like(en)).sum()
        r = (lm[:, 2] - self.rho_meas) * self.rho_isig
        ra = torch.sqrt(torch.where(r * r > 0, r * r, torch.ones_like(r)))
        return c + torch.where(self.prior & (r * r > 0), _huber(ra), torch.zeros_like(ra)).sum()

    def recentre(self, x):
        with torch.no_grad():
            self.R0, self.p0, self.l0 = self.unpack(x)


def _grad_hess(win, theta, isig, z):
    x = torch.zeros(win.n_x(), dtype=f64)
    f = lambda xx: win.cost(xx, theta, isig, z)
    g = torch.func.grad(f)(x)
    H = torch.func.hessian(f)(x)
    return g, H


def solve(win, theta, isig, z, iters=40, tol=1e-13):
    """Newton with the exact Hessian (Levenberg safeguard) until |grad|_max <= tol * (1 + |grad_0|_max)."""
    lam = 1e-8
    g0 = None
    for _ in range(iters):
        g, H = _grad_hess(win, theta, isig, z)
        gm = float(g.abs().max())
        g0 = gm if g0 is None else g0
        if gm <= tol * (1 + g0):
            break
        c = float(win.cost(torch.zeros_like(g), theta, isig, z))
        while True:
            dx = -torch.linalg.solve(H + lam * torch.diag(torch.diag(H).abs() + 1e-12), g)
            if float(win.cost(dx, theta, isig, z)) <= c + 1e-12 * abs(c):
                win.recentre(dx)
                lam = max(lam / 10, 1e-14)
                break
            lam *= 10
            if lam > 1e6:
                return win
    return win


def implicit_grad(win, theta, isig, z, dLdp):
    """dL/d(theta, isig, z) for L with dL/dp = dLdp (P,3) at the converged state."""
    g, H = _grad_hess(win, theta, isig, z)
    n = win.n_x()
    v = torch.zeros(n, dtype=f64)
    piv = torch.nonzero(win.pvar)[:, 0]
    for j, s in enumerate(piv.tolist()):
        v[6 * j + 3:6 * j + 6] = torch.as_tensor(np.asarray(dLdp[s], np.float64))
    lam_ = torch.linalg.solve(H, v)
    x = torch.zeros(n, dtype=f64)
    gx = lambda th, si, zz: torch.func.grad(lambda xx: win.cost(xx, th, si, zz))(x)
    _, vjp = torch.func.vjp(gx, theta, isig, z)
    gt, gs, gz = vjp(lam_)
    return (-gt).numpy(), (-gs).numpy(), (-gz).numpy()


def implicit_grad_schur(win, theta, isig, z, dLdp):
    """implicit_grad for windows too large for a dense Hessian (thousands of landmarks).  The Hessian's pose columns
    come from one Hessian-vector product per pose variable; its landmark blocks are 3x3 and independent, so the
    product along component i of every landmark at once gives column i of all of them.  H lam = v (v on the poses
    only) is solved through the Schur complement on the poses: lam_p = S^-1 v_p with S = Hpp - Hpl Hll^-1 Hlp, then
    lam_l = -Hll^-1 Hlp lam_p.  -> as implicit_grad, and the largest |gradient| over the variables at the state."""
    n = win.n_x()
    npv = 6 * int(win.pvar.sum())
    nl = (n - npv) // 3
    x = torch.zeros(n, dtype=f64)
    gfun = torch.func.grad(lambda xx: win.cost(xx, theta, isig, z))
    g = gfun(x)
    hvp = lambda v: torch.func.jvp(gfun, (x,), (v,))[1]
    Hp = torch.func.vmap(hvp)(torch.eye(n, dtype=f64)[:npv])          # row j = H e_j (pose variable j)
    Hpp = Hp[:, :npv]
    Hlp = Hp[:, npv:].T.reshape(nl, 3, npv)                          # landmark rows, pose columns
    Hll = torch.zeros(nl, 3, 3, dtype=f64)
    for i in range(3):
        v = torch.zeros(n, dtype=f64)
        v[npv + i::3] = 1.0
        Hll[:, :, i] = hvp(v)[npv:].reshape(nl, 3)
    Hll = 0.5 * (Hll + Hll.transpose(1, 2))
    T = torch.linalg.solve(Hll, Hlp)                                 # Hll^-1 Hlp per landmark
    S = Hpp - torch.einsum("lip,liq->pq", Hlp, T)
    S = 0.5 * (S + S.T)
    vp = torch.zeros(npv, dtype=f64)
    piv = torch.nonzero(win.pvar)[:, 0]
    for j, s in enumerate(piv.tolist()):
        vp[6 * j + 3:6 * j + 6] = torch.as_tensor(np.asarray(dLdp[s], np.float64))
    lam_p = torch.linalg.solve(S, vp)
    lam_l = -torch.einsum("lip,p->li", T, lam_p).reshape(-1)
    lam = torch.cat([lam_p, lam_l])
    gx = lambda th, si, zz: torch.func.grad(lambda xx: win.cost(xx, th, si, zz))(x)
    _, vjp = torch.func.vjp(gx, theta, isig, z)
    gt, gs, gz = vjp(lam)
    return (-gt).numpy(), (-gs).numpy(), (-gz).numpy(), float(g.abs().max())


def fd_grad(start, theta, isig, z, loss, step=1e-6, idx=None):
    """Central differences of loss(p*) over theta (all 11) and the isig / z entries in idx (dict of index lists);
    each solve starts from a copy of `start` (a converged Window)."""
    def L(th, si, zz):
        w = solve(copy.deepcopy(start), th, si, zz)
        return float(loss(w.p0))

    out = {}
    for grp, base in (("theta", theta), ("isig", isig), ("z", z)):
        flat = base.reshape(-1)
        sel = range(flat.numel()) if grp == "theta" else (idx or {}).get(grp, [])
        g = np.full(flat.numel(), np.nan)
        for j in sel:
            args = {"theta": theta, "isig": isig, "z": z}
            vals = []
            for sgn in (1.0, -1.0):
                pert = flat.clone()
                pert[j] += sgn * step
                args[grp] = pert.reshape(base.shape)
                vals.append(L(args["theta"], args["isig"], args["z"]))
            g[j] = (vals[0] - vals[1]) / (2 * step)
        out[grp] = g.reshape(tuple(base.shape))
    return out
