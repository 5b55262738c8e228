"""FP64 autodiff reference for the implicit adjoint of the window solve (test infrastructure only).

The reference has no adjoint; this restates its window cost (src/xclean/vio/window.py: stereo residuals, whitening,
Huber with k = 1.345, inverse-depth prior; the same cost as oracle/ba_oracle.c's visual cost) as a torch float64
function of the state x = (per-slot body-pose perturbations [dphi, dp], landmark (a, b, rho)) and of the parameters
theta = (fx, fy, cx, cy, baseline B, the 6-DoF left-to-right extrinsic [omega, t] at the rectified rig, per-observation
weights 1/sigma, observed pixels).  The right camera sees q_r = Exp(omega) q + rho (t - B e_x) (the rectified model is
omega = t = 0).  It provides:
  * solve(...)            Newton with the exact Hessian to a gradient of ~1e-13 (the converged state x*);
  * implicit_grad(...)    dL/dtheta = -(d2C/dtheta dx)^T (d2C/dx2)^-1 dL/dx* by autograd (the FP64 autodiff reference);
  * fd_grad(...)          central finite differences of L(x*(theta)) with step 1e-6.
A slot may be held (not a variable); landmarks outside lm_mask or without a valid observation are constants.
"""
from __future__ import annotations

import numpy as np
import torch

HUBER_K = 1.345
NW_THETA = 11          # fx, fy, cx, cy, B, omega (3), t (3)


def _hat(v):
    z = torch.zeros((), dtype=v.dtype)
    return torch.stack([torch.stack([z, -v[2], v[1]]), torch.stack([v[2], z, -v[0]]),
                        torch.stack([-v[1], v[0], z])])


def _exp(w):
    """Rodrigues, smooth at 0 (series below 1e-4 rad), differentiable twice."""
    t2 = (w * w).sum()
    K = _hat(w)
    if float(t2) < 1e-8:
        a = 1 - t2 / 6 + t2 * t2 / 120
        b = 0.5 - t2 / 24 + t2 * t2 / 720
    else:
        t = torch.sqrt(t2)
        a = torch.sin(t) / t
        b = (1 - torch.cos(t)) / t2
    return torch.eye(3, dtype=w.dtype) + a * K + b * (K @ K)


def _huber(en):
    return torch.where(en <= HUBER_K, 0.5 * en * en, HUBER_K * (en - 0.5 * HUBER_K))


class Window:
    """A window's arrays as float64 torch tensors (a synth_ba.Window or anything with its fields)."""

    def __init__(self, w, hold=0):
        g = lambda k: torch.as_tensor(np.asarray(getattr(w, k), np.float64))
        self.R0, self.p0 = g("Rwb").clone(), g("pwb").clone()
        self.Rbc, self.pbc = g("Rbc"), g("pbc")
        self.l0 = g("lmp").clone()
        self.host = np.asarray(w.lm_host, np.int64)
        self.mask = np.asarray(w.lm_mask, bool)
        self.rho_meas, self.rho_isig = g("rho_meas"), g("rho_isig")
        self.ob_start = np.asarray(w.ob_start, np.int64)
        self.pose = np.asarray(w.ob_pose, np.int64)
        self.cam = np.asarray(w.ob_cam, np.int64)
        self.valid = np.asarray(w.ob_valid, bool)
        self.theta0 = torch.tensor([w.fx, w.fy, w.cx, w.cy, w.B, 0, 0, 0, 0, 0, 0], dtype=torch.float64)
        self.isig0 = g("ob_isig").clone()
        self.z0 = g("ob_z").clone()
        self.P, self.L = self.R0.shape[0], self.l0.shape[0]
        self.hold = hold
        lm_of = np.repeat(np.arange(self.L), np.diff(self.ob_start))
        self.lm_of = lm_of
        has = np.zeros(self.L, bool)
        has[lm_of[self.valid]] = True
        self.lvar = self.mask & has                       # landmarks that are variables
        self.pvar = np.array([s != hold for s in range(self.P)])

    def n_x(self):
        return 6 * int(self.pvar.sum()) + 3 * int(self.lvar.sum())

    def unpack(self, x):
        """x -> (R (P,3,3), p (P,3), lm (L,3)) around the stored linearisation point."""
        Rs, ps, i = [], [], 0
        for s in range(self.P):
            if self.pvar[s]:
                Rs.append(self.R0[s] @ _exp(x[i:i + 3]))
                ps.append(self.p0[s] + x[i + 3:i + 6])
                i += 6
            else:
                Rs.append(self.R0[s])
                ps.append(self.p0[s])
        lms = []
        for l in range(self.L):
            if self.lvar[l]:
                lms.append(self.l0[l] + x[i:i + 3])
                i += 3
            else:
                lms.append(self.l0[l])
        return torch.stack(Rs), torch.stack(ps), torch.stack(lms)

    def cost(self, x, theta, isig, z):
        fx, fy, cx, cy, B = theta[0], theta[1], theta[2], theta[3], theta[4]
        Rlr = _exp(theta[5:8])
        tlr = theta[8:11]
        R, p, lm = self.unpack(x)
        Rwc = R @ self.Rbc
        pwc = p + R @ self.pbc
        c = torch.zeros((), dtype=torch.float64)
        for l in range(self.L):
            if not self.mask[l]:
                continue
            h = self.host[l]
            a, b, rho = lm[l, 0], lm[l, 1], lm[l, 2]
            m = torch.stack([a, b, torch.ones((), dtype=torch.float64)])
            for k in range(self.ob_start[l], self.ob_start[l + 1]):
                if not self.valid[k]:
                    continue
                t = self.pose[k]
                q = Rwc[t].T @ (Rwc[h] @ m + rho * (pwc[h] - pwc[t]))
                if self.cam[k] == 0:
                    e = torch.stack([(fx * q[0] / q[2] + cx - z[k, 0]) * isig[k],
                                     (fy * q[1] / q[2] + cy - z[k, 1]) * isig[k]])
                else:
                    qr = Rlr @ q + rho * (tlr - torch.stack([B, torch.zeros_like(B), torch.zeros_like(B)]))
                    e = ((fx * qr[0] / qr[2] + cx - z[k, 0]) * isig[k]).reshape(1)
                c = c + _huber(torch.sqrt((e * e).sum()))
            if float(self.rho_isig[l]) > 0:
                r = (rho - self.rho_meas[l]) * self.rho_isig[l]
                c = c + _huber(torch.abs(r))
        return c

    def recentre(self, x):
        """Absorb x into the linearisation point."""
        with torch.no_grad():
            R, p, lm = self.unpack(x)
            self.R0, self.p0, self.l0 = R.clone(), p.clone(), lm.clone()


def solve(win, theta, isig, z, iters=30, tol=1e-13):
    """Newton with the exact Hessian (and a Levenberg safeguard) to |grad| <= tol (1 + |grad_0|)."""
    n = win.n_x()
    lam = 1e-6
    g0 = None
    for _ in range(iters):
        x = torch.zeros(n, dtype=torch.float64, requires_grad=True)
        c = win.cost(x, theta, isig, z)
        g, = torch.autograd.grad(c, x, create_graph=True)
        if g0 is None:
            g0 = float(g.abs().max())
        if float(g.abs().max()) <= tol * (1 + g0):
            break
        H = torch.stack([torch.autograd.grad(g[i], x, retain_graph=True)[0] for i in range(n)]).detach()
        while True:
            dx = -torch.linalg.solve(H + lam * torch.diag(torch.diag(H)), g.detach())
            c2 = win.cost(dx, theta, isig, z)
            if float(c2) <= float(c) + 1e-15 * abs(float(c)):
                win.recentre(dx)
                lam = max(lam / 10, 1e-12)
                break
            lam *= 10
            if lam > 1e8:
                return win
    return win


def poses(win):
    return win.p0.clone()


def implicit_grad(win, theta, isig, z, dLdp):
    """dL/d(theta, isig, z) for L with dL/dp = dLdp (P,3) at the converged state (autograd, float64)."""
    n = win.n_x()
    x = torch.zeros(n, dtype=torch.float64, requires_grad=True)
    th = theta.clone().requires_grad_(True)
    si = isig.clone().requires_grad_(True)
    zz = z.clone().requires_grad_(True)
    c = win.cost(x, th, si, zz)
    g, = torch.autograd.grad(c, x, create_graph=True)
    H = torch.stack([torch.autograd.grad(g[i], x, retain_graph=True)[0] for i in range(n)]).detach()
    v = torch.zeros(n, dtype=torch.float64)
    i = 0
    for s in range(win.P):
        if win.pvar[s]:
            v[i + 3:i + 6] = torch.as_tensor(dLdp[s])
            i += 6
    lam_ = torch.linalg.solve(H, v)
    mixed = torch.autograd.grad(g, (th, si, zz), grad_outputs=lam_, allow_unused=True)
    out = [(-m if m is not None else torch.zeros_like(t)) for m, t in zip(mixed, (th, si, zz))]
    return out[0].detach().numpy(), out[1].detach().numpy(), out[2].detach().numpy()


def fd_grad(make_window, theta, isig, z, loss, step=1e-6, which=("theta", "isig", "z"), idx=None):
    """Central differences of loss(p*(theta, isig, z)); make_window() gives a fresh Window at the start state.
    idx: optional dict of index lists per group (default: every entry)."""
    def L(th, si, zz):
        w = solve(make_window(), th, si, zz)
        return float(loss(poses(w)))

    out = {}
    for grp, base in (("theta", theta), ("isig", isig), ("z", z)):
        if grp not in which:
            continue
        flat = base.reshape(-1)
        sel = range(flat.numel()) if idx is None or grp not in idx else idx[grp]
        g = np.zeros(flat.numel())
        for j in sel:
            args = {"theta": theta, "isig": isig, "z": z}
            plus = flat.clone()
            minus = flat.clone()
            plus[j] += step
            minus[j] -= step
            args[grp] = plus.reshape(base.shape)
            lp = L(args["theta"], args["isig"], args["z"])
            args[grp] = minus.reshape(base.shape)
            lm = L(args["theta"], args["isig"], args["z"])
            g[j] = (lp - lm) / (2 * step)
        out[grp] = g.reshape(tuple(base.shape))
    return out
