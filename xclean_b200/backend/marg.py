"""The marginal prior of the window solve: the drop-in for xclean.vio.marg (src/xclean/vio/marg.py), pose blocks.

A prior is the cost 1/2 |S d + r|^2 over blocks, one per window slot.  d stacks, per block, the box-minus of the
slot's current pose against the block's first linearisation point x0 (FEJ: S and x0 never change once formed):
[Log(R0^T R), p - p0] (marg.py:43-53).  It is kept in square-root form, made from an information form (H, b) by an
eigen-decomposition with the numerical-rank floor EIG_FLOOR (eigenvalues below EIG_FLOOR x the largest are dropped,
not inverted: marg.py:81-91).  The Schur marginalisation (marg.py:164-175) inverts its eliminated block the same
way; `combine` (marg.py:178-205) keeps the x0 of blocks already in the old prior and re-expresses b there.

This module is host-side float64 algebra on matrices of at most a few hundred rows, as the reference's is; the prior
enters the device window solve (backend.ba.solve_batch / BatchSolver with `priors=`) as S, r and x0, where its terms
are added to the reduced camera system, the gradient and the cost of every LM iteration on the GPU.

Blocks here are 6-dim pose blocks.  The 15-dim visual-inertial blocks of the reference (velocity and IMU biases)
belong to the IMU factors, which this path does not carry: a 15-dim block raises NotImplementedError.
"""
from __future__ import annotations

import math

import numpy as np

EIG_FLOOR = 1e-12


def so3_log(R):
    """window.so3_log_nb (src/xclean/vio/window.py:65-105): the rotation vector of R, with the near-zero and near-pi
    branches of the reference."""
    R = np.asarray(R, np.float64)
    c = min(max((R[0, 0] + R[1, 1] + R[2, 2] - 1.0) * 0.5, -1.0), 1.0)
    th = math.acos(c)
    v = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]])
    if th < 1e-6:
        return 0.5 * v
    if th > math.pi - 1e-4:
        B = 0.5 * (R + R.T)
        i = 0                              # the largest diagonal entry, the first on ties
        for j in (1, 2):
            if B[j, j] > B[i, i]:
                i = j
        den = math.sqrt(max((B[i, i] - c) / (1.0 - c), 0.0))
        ax = np.array([(B[j, i] - (c if j == i else 0.0)) / max(den * (1.0 - c), 1e-12) for j in range(3)])
        ax[i] = den
        nrm = math.sqrt(ax[0] ** 2 + ax[1] ** 2 + ax[2] ** 2)
        sgn = -1.0 if ax[0] * v[0] + ax[1] * v[1] + ax[2] * v[2] < 0 else 1.0
        return sgn * th * ax / nrm
    return (th / (2.0 * math.sin(th))) * v


def _pose0(st):
    """(R, p) float64 copies of a state-like tuple (R, p, v, bg, ba): the x0 a pose block keeps."""
    R, p = st[0], st[1]
    z = np.zeros(3)
    return (np.array(R, np.float64), np.array(p, np.float64), z.copy(), z.copy(), z.copy())


def _check_dims(dims):
    for d in dims:
        if int(d) != 6:
            raise NotImplementedError("marg: only 6-dim pose blocks (the 15-dim visual-inertial blocks need the IMU "
                                      "factors, which this path does not carry)")


def _box_minus(R, p, x0):
    out = np.empty(6)
    out[:3] = so3_log(np.ascontiguousarray(x0[0].T @ R))
    out[3:] = p - x0[1]
    return out


def _eig_floor(H):
    """Eigen-decomposition of the symmetric part of H with the rank floor: -> (eigenvalues kept, their vectors)."""
    lam, V = np.linalg.eigh(0.5 * (H + H.T))
    top = float(lam.max()) if lam.size else 0.0
    keep = lam > EIG_FLOOR * max(top, 1e-300)
    return lam[keep], V[:, keep]


class Prior:
    """1/2 |S d + r|^2 over pose blocks (marg.Prior): sids (slot ids in block order), dims (6 each), x0 per block
    ((R0, p0, v0, bg0, ba0); v / bg / ba unused by pose blocks), S (m, 6 nb), r (m,)."""

    def __init__(self, sids, dims, x0, S, r):
        _check_dims(dims)
        self.sids = [s for s in sids]
        self.dims = [int(d) for d in dims]
        self.x0 = [_pose0(x) for x in x0]
        self.S = np.array(S, np.float64)
        self.r = np.array(r, np.float64)
        self.cols = None
        self._idx = None

    @property
    def n(self):
        return 6 * len(self.dims)

    def info(self):
        """(H, b) = (S^T S, S^T r) at x0."""
        return self.S.T @ self.S, self.S.T @ self.r

    @classmethod
    def from_info(cls, sids, dims, x0, H, b):
        lam, V = _eig_floor(np.asarray(H, np.float64))
        root = np.sqrt(lam)
        return cls(sids, dims, x0, root[:, None] * V.T, (V.T @ np.asarray(b, np.float64)) / root)

    def bind(self, index_of_sid, off=None, slot_dims=None):
        """Attach the prior to a window: index_of_sid maps each block's slot id to its slot index; off (P + 1) the
        window's block offsets (6 per slot by default)."""
        cols, idx = [], []
        for s, dim in zip(self.sids, self.dims):
            i = index_of_sid[s]
            if slot_dims is not None and dim > int(slot_dims[i]):
                raise RuntimeError("prior block of slot %d has %d dims, the slot has %d" % (s, dim, slot_dims[i]))
            o = 6 * i if off is None else int(off[i])
            cols.append(np.arange(o, o + dim))
            idx.append(i)
        self.cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
        self._idx = idx

    def slots(self):
        """The window slot of each block (after bind)."""
        if self._idx is None:
            raise RuntimeError("Prior.bind() first")
        return list(self._idx)

    def delta(self, Rwb, pwb):
        d = np.zeros(self.n)
        for k, i in enumerate(self.slots()):
            d[6 * k:6 * k + 6] = _box_minus(np.asarray(Rwb[i], np.float64), np.asarray(pwb[i], np.float64),
                                            self.x0[k])
        return d

    def terms(self, state, n):
        """(H (n, n), b (n,), cost) of the prior at `state` (R, p, ...) in a system of n columns."""
        res = self.S @ self.delta(state[0], state[1]) + self.r
        H = np.zeros((n, n))
        b = np.zeros(n)
        H[np.ix_(self.cols, self.cols)] = self.S.T @ self.S
        b[self.cols] = self.S.T @ res
        return H, b, 0.5 * float(res @ res)

    def cost(self, state):
        res = self.S @ self.delta(state[0], state[1]) + self.r
        return 0.5 * float(res @ res)

    def drop_slot(self, sid):
        """Marginalise one slot's block out of the prior (exact Schur on the information form at x0); None when it
        was the last block."""
        if sid not in self.sids:
            return self
        k = self.sids.index(sid)
        H, b = self.info()
        marg = np.arange(6 * k, 6 * k + 6)
        keep = np.setdiff1d(np.arange(self.n), marg)
        H2, b2 = schur(H, b, keep, marg)
        rest = [i for i in range(len(self.sids)) if i != k]
        if not rest:
            return None
        return Prior.from_info([self.sids[i] for i in rest], [self.dims[i] for i in rest],
                               [self.x0[i] for i in rest], H2, b2)

    def shrink_slot(self, sid):
        """A pose block has no velocity / bias dims to marginalise: unchanged."""
        return self


def schur(H, b, keep, marg):
    """Eliminate `marg` from (H, b): H' = H_kk - H_km H_mm^+ H_mk, b' = b_k - H_km H_mm^+ b_m, with H_mm^+ the
    floored eigen-inverse (a rank-deficient block gives up its unobservable part).  -> (H' symmetrised, b')."""
    H = np.asarray(H, np.float64)
    b = np.asarray(b, np.float64)
    keep = np.asarray(keep, np.int64)
    marg = np.asarray(marg, np.int64)
    lam, V = _eig_floor(H[np.ix_(marg, marg)])
    Hmm_inv = (V / lam) @ V.T
    Hkm = H[np.ix_(keep, marg)]
    Hk = H[np.ix_(keep, keep)] - Hkm @ Hmm_inv @ Hkm.T
    bk = b[keep] - Hkm @ Hmm_inv @ b[marg]
    return 0.5 * (Hk + Hk.T), bk


def combine(prior_old, sids_new, dims_new, states_cur, H_cur, b_cur):
    """The new prior over blocks (sids_new, dims_new) from (H_cur, b_cur) linearised at the current states (one
    (R, p, ...) per block): a block the old prior holds keeps its x0 and b is moved there (b_x0 = b_cur - H_cur d);
    a new block starts at its current estimate."""
    _check_dims(dims_new)
    x0, d = [], np.zeros(6 * len(sids_new))
    for k, (s, st) in enumerate(zip(sids_new, states_cur)):
        cur = _pose0(st)
        if prior_old is not None and s in prior_old.sids:
            keep = prior_old.x0[prior_old.sids.index(s)]
            x0.append(keep)
            d[6 * k:6 * k + 6] = _box_minus(cur[0], cur[1], keep)
        else:
            x0.append(cur)
    H_cur = np.asarray(H_cur, np.float64)
    return Prior.from_info(sids_new, dims_new, x0, H_cur, np.asarray(b_cur, np.float64) - H_cur @ d)


def gauge_prior(sid, R, p, info=1e10):
    """The visual-odometry gauge: a 6-DoF prior of information `info` on one keyframe (marg.py:208-213)."""
    return Prior([sid], [6], [(R, p, None, None, None)], math.sqrt(info) * np.eye(6), np.zeros(6))
