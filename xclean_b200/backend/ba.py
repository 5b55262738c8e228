"""Bundle adjustment on the device: the batched sliding-window solve (the reference's window.solve model) and, in
backend/local_ba.py, the drop-in _solve_gpu / _solve_gpu_id of src/xclean/backend/ba.py (with backend/kernels.py,
the drop-in of its stage kernels).

    res = solve_batch(windows, iters=5, lam0=1e-4, precision="mixed", hold=0)
    # windows: synth_ba.Window objects (the fields of vio/window.Problem, `pf` = PoseFree or None); solved in place
    # res: dict(cost0, cost, accepted, lam, status (per window), dx0 (the first pose step per window))

    bs = BatchSolver(windows, device)       # pack once, keep resident on the device
    bs.solve(iters, lam0, precision)        # one persistent launch for every window; results stay on the device

    bs.linearise()                          # final_linearisation's reduced visual system per window
    posefree_cost(...), posefree_step(...)  # window.py's pose-free block functions, bit-identical
    posefree_marginals(w)                   # final_linearisation's pose-free marginals into w.pf.Hinv / w.pf.ok
    systems, costs = final_linearisation_batch(windows);  H, b, off = marg_system_batch(windows, masks)[i]

    # window.py's own single-window signatures (visual windows, with a marginal prior over pose slots (w.prior, a
    # bound backend.marg.Prior or the reference's marg.Prior); IMU terms raise NotImplementedError)
    st = solve(pb, iters=5, lam0=1e-4);  final_linearisation(pb);  marg_system(pb, lm_mask)

Every call goes through libxcb200.so's C ABI (xcb_ba_solve_windows_dev); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib

PRECISIONS = {"fp64": _lib.XCB_BA_FP64, "mixed": _lib.XCB_BA_MIXED}
MAX_SLOTS = 20
MAX_ROWS_PER_LANDMARK = 32
MAX_TOUCHED_SLOTS = 16      # host + observing keyframes per landmark (the kernel's per-warp scratch)


class PoseFree:
    """window.PoseFree (src/xclean/vio/window.py:795-810): landmarks kept out of the Schur system, seen only in their
    host's left image.  host (n,) slot indices, z (n,2) the host left pixels, isg their whitening, rmeas / ris (n,)
    the inverse-depth prior, lmp (n,3) the state (updated by the solve), Hinv (n,3,3) / ok (n,) the marginals
    (posefree_marginals)."""

    def __init__(self, host, z, isg, rmeas, ris, lmp):
        self.host = np.ascontiguousarray(host, np.int64)
        self.z = np.ascontiguousarray(np.asarray(z, np.float64).reshape(-1, 2))
        self.isg = float(isg)
        self.rmeas = np.ascontiguousarray(rmeas, np.float64)
        self.ris = np.ascontiguousarray(ris, np.float64)
        self.lmp = np.ascontiguousarray(np.asarray(lmp, np.float64).reshape(-1, 3)).copy()
        n = len(self.host)
        self.Hinv = np.zeros((n, 3, 3))
        self.ok = np.zeros(n, np.bool_)


def _pf_of(w):
    pf = getattr(w, "pf", None)
    return pf if (pf is not None and len(pf.host) > 0) else None


class _Merged:
    """A window with its pose-free landmarks appended as ordinary landmarks, each with its one observation (host
    slot, left camera, its pixel and whitening) and its inverse-depth prior.  window.solve treats the pose-free block
    exactly as build_system treats such a landmark (_pf_block_fast is build_system's landmark block with t == h,
    window.py:550-680): the observation has no pose coupling, the block is damped and guarded the same way, its
    cost joins the window's and its step is accepted with the poses' (window.py:934-975)."""

    def __init__(self, w, pf):
        n = len(pf.host)
        for k in ("Rwb", "pwb", "Rbc", "pbc", "fx", "fy", "cx", "cy", "B", "huber_k"):
            setattr(self, k, getattr(w, k))
        self.prior = getattr(w, "prior", None)
        M = int(np.asarray(w.ob_start)[-1])
        self.lmp = np.concatenate([np.asarray(w.lmp, np.float64).reshape(-1, 3), pf.lmp])
        self.lm_host = np.concatenate([np.asarray(w.lm_host, np.int64), pf.host])
        self.lm_mask = np.concatenate([np.asarray(w.lm_mask, np.bool_), np.ones(n, np.bool_)])
        self.rho_meas = np.concatenate([np.asarray(w.rho_meas, np.float64), pf.rmeas])
        self.rho_isig = np.concatenate([np.asarray(w.rho_isig, np.float64), pf.ris])
        self.ob_start = np.concatenate([np.asarray(w.ob_start, np.int64), M + 1 + np.arange(n, dtype=np.int64)])
        self.ob_pose = np.concatenate([np.asarray(w.ob_pose, np.int64), pf.host])
        self.ob_cam = np.concatenate([np.asarray(w.ob_cam, np.int64), np.zeros(n, np.int64)])
        self.ob_z = np.concatenate([np.asarray(w.ob_z, np.float64).reshape(-1, 2), pf.z])
        self.ob_isig = np.concatenate([np.asarray(w.ob_isig, np.float64), np.full(n, pf.isg)])
        self.ob_valid = np.concatenate([np.asarray(w.ob_valid, np.bool_), np.ones(n, np.bool_)])


def merge_posefree(w):
    """The window as the batched solve sees it: `w` itself, or, with a pose-free block, a view with the block's
    landmarks appended after w's own (their states follow w.lmp's rows in the packed batch)."""
    pf = _pf_of(w)
    if pf is None:
        return w
    if (pf.host < 0).any() or (pf.host >= w.Rwb.shape[0]).any():
        raise ValueError("solve_batch: a pose-free landmark's host slot is outside the window")
    return _Merged(w, pf)


def pack_windows(windows, hold=0):
    """Concatenate windows into the batch layout of xcb_ba_windows (host numpy arrays); pose-free blocks are
    appended to their windows' landmarks (merge_posefree)."""
    windows = [merge_posefree(w) for w in windows]
    nw = len(windows)
    P = np.array([w.Rwb.shape[0] for w in windows], np.int32)
    L = np.array([w.lmp.shape[0] for w in windows], np.int32)
    M = np.array([w.ob_pose.shape[0] for w in windows], np.int64)
    if P.max(initial=0) > MAX_SLOTS:
        raise ValueError("solve_batch: a window has %d slots (at most %d)" % (P.max(), MAX_SLOTS))
    slot_off = np.zeros(nw, np.int32)
    lm_off = np.zeros(nw, np.int32)
    if nw:
        slot_off[1:] = np.cumsum(P)[:-1]
        lm_off[1:] = np.cumsum(L)[:-1]
    ob_base = np.zeros(nw + 1, np.int64)
    ob_base[1:] = np.cumsum(M)
    lm_ob = np.concatenate([w.ob_start[:-1].astype(np.int64) + ob_base[i] for i, w in enumerate(windows)]
                           + [np.array([ob_base[-1]], np.int64)])
    rows = np.diff(lm_ob)
    if len(rows) and rows.max() > MAX_ROWS_PER_LANDMARK:
        raise ValueError("solve_batch: a landmark has %d observation rows (at most %d)" % (rows.max(),
                                                                                       MAX_ROWS_PER_LANDMARK))
    for i, w in enumerate(windows):
        host, pose = np.asarray(w.lm_host, np.int64), np.asarray(w.ob_pose, np.int64)
        if (host < 0).any() or (host >= P[i]).any() or (pose < 0).any() or (pose >= P[i]).any():
            raise ValueError("solve_batch: window %d has a host or observing slot outside 0..%d" % (i, P[i] - 1))
        if len(pose):
            # distinct slots a landmark touches: its observing keyframes and its host
            lm_of = np.repeat(np.arange(len(host)), np.diff(np.asarray(w.ob_start, np.int64)))
            keys = np.unique(np.concatenate([lm_of * MAX_SLOTS + pose, np.arange(len(host)) * MAX_SLOTS + host]))
            touched = np.bincount(keys // MAX_SLOTS, minlength=len(host))
            if touched.max() > MAX_TOUCHED_SLOTS:
                raise ValueError("solve_batch: a landmark of window %d touches %d keyframes (at most %d)"
                                 % (i, touched.max(), MAX_TOUCHED_SLOTS))
    cat = lambda name, dt: np.ascontiguousarray(np.concatenate([np.asarray(getattr(w, name)).reshape(
        len(getattr(w, name)), -1) for w in windows]).astype(dt)) if nw else np.zeros(0, dt)
    hold_a = np.full(nw, -1 if hold is None else int(hold), np.int32)
    cam = np.array([[w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k] for w in windows], np.float64).reshape(nw, 6)
    ext = np.array([np.concatenate([np.asarray(w.Rbc, np.float64).ravel(), np.asarray(w.pbc, np.float64).ravel()])
                    for w in windows], np.float64).reshape(nw, 12)
    work = P.astype(np.int64) ** 2 * 36 + M.astype(np.int64) * 64
    order = np.argsort(-work, kind="stable").astype(np.int32)
    pr = _pack_priors(windows, P)
    return dict(**pr, P=P, L=L, slot_off=slot_off, lm_off=lm_off, hold=hold_a, order=order, cam=cam, ext=ext,
                Rwb=cat("Rwb", np.float64).reshape(-1, 9), pwb=cat("pwb", np.float64).reshape(-1, 3),
                lmp=cat("lmp", np.float64).reshape(-1, 3), lm_host=cat("lm_host", np.int32).ravel(),
                lm_mask=cat("lm_mask", np.uint8).ravel(), rho_meas=cat("rho_meas", np.float64).ravel(),
                rho_isig=cat("rho_isig", np.float64).ravel(), lm_ob=lm_ob.astype(np.int32),
                ob_pose=cat("ob_pose", np.int32).ravel(), ob_cam=cat("ob_cam", np.uint8).ravel(),
                ob_z=cat("ob_z", np.float64).reshape(-1, 2), ob_isig=cat("ob_isig", np.float64).ravel(),
                ob_valid=cat("ob_valid", np.uint8).ravel(), max_slots=int(P.max(initial=1)), nw=nw)


PRIOR_FIELDS = ("pr_m", "pr_nb", "pr_boff", "pr_soff", "pr_roff", "pr_blk", "pr_x0", "pr_S", "pr_r")


def _prior_slots(pr, P):
    """The window slot of each block of a bound prior (window.Problem.prior: marg.Prior after bind(), 6-dim pose
    blocks with the default 6-per-slot offsets)."""
    if not hasattr(pr, "dims"):
        raise ValueError("solve_batch: the window's prior is not a marginal prior (marg.Prior)")
    cols = getattr(pr, "cols", None)
    dims = [int(x) for x in pr.dims]
    if cols is None:
        raise ValueError("solve_batch: the window's prior is not bound to its slots (Prior.bind)")
    if any(x != 6 for x in dims):
        raise NotImplementedError("solve_batch: prior blocks of 15 dims (visual-inertial) are not on this path")
    cols = np.asarray(cols, np.int64)
    slots = cols[0::6] // 6
    if len(cols) != 6 * len(dims) or (cols != (6 * np.repeat(slots, 6) + np.tile(np.arange(6), len(dims)))).any():
        raise ValueError("solve_batch: a prior block does not cover one whole pose slot")
    if (slots < 0).any() or (slots >= P).any() or len(np.unique(slots)) != len(slots):
        raise ValueError("solve_batch: prior blocks must be distinct slots of the window")
    return slots


def _pack_priors(windows, P):
    """The marginal priors of the windows (w.prior: None or a bound marg.Prior) in the pr_* layout of xcb_ba_windows;
    {} when no window has one."""
    prs = [getattr(w, "prior", None) for w in windows]
    if all(p is None for p in prs):
        return {}
    nw = len(windows)
    m = np.zeros(nw, np.int32)
    nb = np.zeros(nw, np.int32)
    boff = np.zeros(nw, np.int32)
    soff = np.zeros(nw, np.int32)
    roff = np.zeros(nw, np.int32)
    blk, x0, S, r = [], [], [], []
    nblk = ns = nr = 0
    for i, pr in enumerate(prs):
        boff[i], soff[i], roff[i] = nblk, ns, nr
        if pr is None:
            continue
        slots = _prior_slots(pr, int(P[i]))
        Sw = np.ascontiguousarray(pr.S, np.float64).reshape(-1, 6 * len(slots))
        rw = np.ascontiguousarray(pr.r, np.float64).reshape(Sw.shape[0])
        if Sw.shape[0] > 6 * len(slots):
            raise ValueError("solve_batch: a prior has more rows than columns")
        m[i], nb[i] = Sw.shape[0], len(slots)
        blk.append(slots.astype(np.int32))
        x0.append(np.stack([np.concatenate([np.asarray(x[0], np.float64).ravel(), np.asarray(x[1], np.float64).ravel()])
                            for x in pr.x0]))
        S.append(Sw.ravel())
        r.append(rw)
        nblk += len(slots)
        ns += Sw.size
        nr += len(rw)
    cat = lambda parts, dt, shape: (np.ascontiguousarray(np.concatenate(parts).astype(dt)).reshape(shape) if parts
                                    else np.zeros(shape, dt))
    return dict(pr_m=m, pr_nb=nb, pr_boff=boff, pr_soff=soff, pr_roff=roff, pr_blk=cat(blk, np.int32, (-1,)),
                pr_x0=cat(x0, np.float64, (-1, 12)), pr_S=cat(S, np.float64, (-1,)), pr_r=cat(r, np.float64, (-1,)))


class BatchSolver:
    """A packed batch resident on the device (torch tensors for the memory; the kernels are libxcb200's)."""

    FIELDS = ("P", "L", "slot_off", "lm_off", "hold", "order", "cam", "ext", "Rwb", "pwb", "lmp", "lm_host",
              "lm_mask", "rho_meas", "rho_isig", "lm_ob", "ob_pose", "ob_cam", "ob_z", "ob_isig", "ob_valid")

    def __init__(self, windows, device="cuda", hold=0, packed=None):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.host = packed if packed is not None else pack_windows(windows, hold)
        self.nw = self.host["nw"]
        self.max_slots = self.host["max_slots"]
        self.t = {k: torch.from_numpy(np.ascontiguousarray(self.host[k])).to(self.dev) for k in self.FIELDS}
        for k in PRIOR_FIELDS:
            if k in self.host:
                a = np.ascontiguousarray(self.host[k])
                self.t[k] = torch.from_numpy(a if a.size else np.zeros(1, a.dtype)).to(self.dev)
        self.init = {k: self.t[k].clone() for k in ("Rwb", "pwb", "lmp")}
        self.generation = 0         # bumped by every call that changes the state or the constant-landmark flags
        self.stats = torch.zeros((max(self.nw, 1), 8), dtype=torch.float64, device=self.dev)
        self.dx0 = torch.zeros((max(self.nw, 1), 6 * MAX_SLOTS), dtype=torch.float64, device=self.dev)
        Lt = int(self.host["lmp"].shape[0])
        L = _lib.lib()
        nb = int(L.xcb_ba_scratch_bytes(self.nw, Lt))
        self.scratch = torch.zeros(nb, dtype=torch.uint8, device=self.dev)
        self.desc = _lib.BaWindows()
        self.desc.nw = self.nw
        for k in self.FIELDS + PRIOR_FIELDS:
            if k in self.t:
                setattr(self.desc, k, self.t[k].data_ptr())

    def reset(self):
        self.generation += 1
        for k in ("Rwb", "pwb", "lmp"):
            self.t[k].copy_(self.init[k])
        self.clear_frozen()

    def clear_frozen(self):
        """Forget the constant-landmark flags of the Newton calls (they belong to the state they were found at)."""
        self.generation += 1
        if hasattr(self, "nscratch"):
            self.nscratch.zero_()

    def frozen(self):
        """-> bool tensor [Lt]: the landmarks flagged constant by newton() calls (all False before any)."""
        Lt = int(self.host["lmp"].shape[0])
        if not hasattr(self, "nscratch"):
            return self.torch.zeros(Lt, dtype=self.torch.bool, device=self.dev)
        lsc = self.nscratch[256:256 + 8 * 19 * Lt].view(self.torch.float64).view(Lt, 19)
        return lsc[:, 18] != 0.0

    def _nscratch(self):
        if not hasattr(self, "nscratch"):
            nb = int(_lib.lib().xcb_ba_newton_scratch_bytes(self.nw, int(self.host["lmp"].shape[0])))
            self.nscratch = self.torch.zeros(nb, dtype=self.torch.uint8, device=self.dev)
        return self.nscratch

    def solve_free(self, iters=20, lam0=1e-4, stream=None, grid=0, path="window"):
        """window.solve (float64) with the landmarks that earlier newton() calls found frozen held constant, so that
        the LM converges to a stationary point of the cost in the other variables.  path: "window" (one CTA per
        window), "large" (the large-window path) or "auto" (use_large decides).  -> stats [nw, 8] (cost0, cost,
        accepted, lam, status, iters, -, -)."""
        torch = self.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.dev)
        sc = self._nscratch()
        self.generation += 1
        stats = torch.zeros((max(self.nw, 1), 8), dtype=torch.float64, device=self.dev)
        if path == "large" or (path == "auto" and self.use_large()):
            self._large_setup()
            rc = _lib.lib().xcb_ba_solve_windows_large_free_dev(
                ctypes.byref(self.desc), int(self.host["Rwb"].shape[0]), int(self.host["lmp"].shape[0]),
                self.lchunks.data_ptr(), self.nchunks, self.max_slots, int(iters), float(lam0), stats.data_ptr(),
                self.lscratch.data_ptr(), self.lscratch.numel(), sc.data_ptr(), sc.numel(),
                ctypes.c_void_p(s.cuda_stream or None))
            _lib.check(rc, None, "xcb_ba_solve_windows_large_free_dev")
            return stats[:self.nw]
        rc = _lib.lib().xcb_ba_solve_windows_free_dev(ctypes.byref(self.desc), int(self.host["lmp"].shape[0]),
                                                      self.max_slots, int(iters), float(lam0), stats.data_ptr(),
                                                      sc.data_ptr(), sc.numel(), int(grid),
                                                      ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_solve_windows_free_dev")
        return stats[:self.nw]

    LARGE_CHUNK = 256           # landmarks per chunk of the large-window path (LW_CHUNK in ba_window.cu)

    def use_large(self):
        """The large-window path pays when the batch has fewer windows than half the SMs and they are large (the
        persistent kernel gives each window one SM); windows with a marginal prior always take the persistent one."""
        if "pr_m" in self.host or self.nw == 0:
            return False
        sms = self.torch.cuda.get_device_properties(self.dev).multi_processor_count
        return self.nw * 2 <= sms and int(self.host["L"].mean()) >= 4 * self.LARGE_CHUNK

    def _large_setup(self):
        if hasattr(self, "lchunks"):
            return
        ch = [(w, l0, min(l0 + self.LARGE_CHUNK, int(L))) for w, L in enumerate(self.host["L"])
              for l0 in range(0, int(L), self.LARGE_CHUNK)]
        ch.sort(key=lambda c: -(int(self.host["P"][c[0]]) ** 2))     # the windows with the largest systems first
        self.lchunks = self.torch.tensor(ch if ch else [(0, 0, 0)], dtype=self.torch.int32, device=self.dev)
        self.nchunks = len(ch)
        nb = int(_lib.lib().xcb_ba_large_scratch_bytes(self.nw, int(self.host["Rwb"].shape[0]),
                                                       int(self.host["lmp"].shape[0])))
        self.lscratch = self.torch.zeros(nb, dtype=self.torch.uint8, device=self.dev)

    def solve_large(self, iters=5, lam0=1e-4, precision="mixed", stream=None):
        """window.solve for every window with the large-window path (xcb_ba_solve_windows_large_dev): the landmark
        passes of all windows on all SMs, the per-window steps one CTA per window; asynchronous on `stream`."""
        torch = self.torch
        self._large_setup()
        s = stream if stream is not None else torch.cuda.current_stream(self.dev)
        self.generation += 1
        rc = _lib.lib().xcb_ba_solve_windows_large_dev(
            ctypes.byref(self.desc), int(self.host["Rwb"].shape[0]), int(self.host["lmp"].shape[0]),
            self.lchunks.data_ptr(), self.nchunks, self.max_slots, int(iters), float(lam0), PRECISIONS[precision],
            self.stats.data_ptr(), self.dx0.data_ptr(), 6 * MAX_SLOTS, self.lscratch.data_ptr(),
            self.lscratch.numel(), ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_solve_windows_large_dev")

    def solve(self, iters=5, lam0=1e-4, precision="mixed", stream=None, grid=0, path="window"):
        """One persistent launch over every window (asynchronous on `stream`, torch's current stream by default).
        path: "window" (one CTA per window), "large" (solve_large) or "auto" (use_large decides)."""
        torch = self.torch
        if path == "large" or (path == "auto" and self.use_large()):
            return self.solve_large(iters, lam0, precision, stream)
        s = stream if stream is not None else torch.cuda.current_stream(self.dev)
        self.generation += 1
        rc = _lib.lib().xcb_ba_solve_windows_dev(ctypes.byref(self.desc), self.max_slots, int(iters), float(lam0),
                                                 PRECISIONS[precision], self.stats.data_ptr(), self.dx0.data_ptr(),
                                                 6 * MAX_SLOTS, self.scratch.data_ptr(), self.scratch.numel(),
                                                 int(grid), ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_solve_windows_dev")

    def linearise(self, stream=None, grid=0):
        """final_linearisation's visual outputs (window.py:985-1008, build_system at lam = 0) of every window at the
        state on the device: -> (list of dict(H (6P,6P), b (6P), lm_ok (L), Hll_inv (L,3,3), ob_chi2 (M)) float64
        host arrays over the packed window (pose-free landmarks and their observations after the window's own),
        robust cost per window).  No hold, no damping; the state is unchanged."""
        torch = self.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.dev)
        nm = 6 * self.max_slots
        Lw = self.host["L"].astype(np.int64)
        lm_ob = self.host["lm_ob"].astype(np.int64)
        lo = self.host["lm_off"].astype(np.int64)
        Mw = lm_ob[lo + Lw] - lm_ob[lo]
        stride = int(nm * nm + nm + 10 * Lw.max(initial=0) + Mw.max(initial=0))
        out = torch.zeros(max(self.nw, 1) * stride, dtype=torch.float64, device=self.dev)
        rc = _lib.lib().xcb_ba_linearise_windows_dev(ctypes.byref(self.desc), self.max_slots, out.data_ptr(), stride,
                                                     self.stats.data_ptr(), self.scratch.data_ptr(),
                                                     self.scratch.numel(), int(grid),
                                                     ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_linearise_windows_dev")
        s.synchronize()
        o = out.cpu().numpy()
        systems = []
        for i in range(self.nw):
            n, L, M = 6 * int(self.host["P"][i]), int(Lw[i]), int(Mw[i])
            blk = o[i * stride:i * stride + n * n + n + 10 * L + M]
            rec = blk[n * n + n:n * n + n + 10 * L].reshape(L, 10)
            systems.append(dict(H=blk[:n * n].reshape(n, n).copy(), b=blk[n * n:n * n + n].copy(),
                                lm_ok=rec[:, 0] != 0, Hll_inv=rec[:, 1:].reshape(L, 3, 3).copy(),
                                ob_chi2=blk[n * n + n + 10 * L:].copy()))
        return systems, self.stats.cpu().numpy()[:self.nw, 0].copy()

    def newton(self, steps=3, maxit=60, tol=1e-12, stream=None, grid=0, flag=True):
        """Exact-Hessian Newton steps on every window (in place): the converged state the adjoint differentiates.
        flag: landmarks whose decoupled Gauss-Newton step would take the inverse depth to <= 1e-9 at an evaluated
        state are flagged constant (flags persist until clear_frozen / reset); False keeps the flags as they are.
        -> per-window stats tensor [nw, 4] (CG iterations, relative residual, final gradient max-norm, status)."""
        mode = _lib.XCB_BA_NEWTON_POLISH if flag else _lib.XCB_BA_NEWTON_POLISH_FIXED
        return self._newton(mode, steps, maxit, tol, None, stream, grid)[0]

    def adjoint(self, gpose, maxit=60, tol=1e-12, stream=None, grid=0):
        """dL/dtheta at the current (converged) state for dL/d(dphi, dp) = gpose [slots, 6] (float64 CUDA tensor)
        -> (stats [nw, 4], gtheta [nw, 11], gisig [M], gz [M, 2])."""
        return self._newton(_lib.XCB_BA_NEWTON_ADJOINT, 0, maxit, tol, gpose, stream, grid)

    def _newton(self, mode, steps, maxit, tol, gpose, stream, grid):
        torch = self.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.dev)
        M = int(self.host["ob_isig"].shape[0])
        self._nscratch()
        stats = torch.zeros((max(self.nw, 1), 4), dtype=torch.float64, device=self.dev)
        gtheta = torch.zeros((max(self.nw, 1), 11), dtype=torch.float64, device=self.dev)
        gisig = torch.zeros(max(M, 1), dtype=torch.float64, device=self.dev)
        gz = torch.zeros((max(M, 1), 2), dtype=torch.float64, device=self.dev)
        gp = None
        if gpose is not None:
            gp = gpose.to(self.dev, torch.float64).contiguous()
            if tuple(gp.shape) != (int(self.host["Rwb"].shape[0]), 6):
                raise ValueError("adjoint: gpose must be [slots, 6]")
        if mode != _lib.XCB_BA_NEWTON_ADJOINT:
            self.generation += 1
        rc = _lib.lib().xcb_ba_newton_windows_dev(
            ctypes.byref(self.desc), self.max_slots, int(mode), int(steps), int(maxit), float(tol),
            ctypes.c_void_p(gp.data_ptr() if gp is not None else None), ctypes.c_void_p(gtheta.data_ptr()),
            ctypes.c_void_p(gisig.data_ptr()), ctypes.c_void_p(gz.data_ptr()), ctypes.c_void_p(stats.data_ptr()),
            ctypes.c_void_p(self.nscratch.data_ptr()), self.nscratch.numel(), int(grid),
            ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_newton_windows_dev")
        return stats[:self.nw], gtheta[:self.nw], gisig[:M], gz[:M]

    def results(self):
        st = self.stats.cpu().numpy()[:self.nw]
        return {"cost0": st[:, 0], "cost": st[:, 1], "accepted": st[:, 2].astype(np.int64), "lam": st[:, 3],
                "status": st[:, 4].astype(np.int64), "dx0": self.dx0.cpu().numpy()[:self.nw]}

    def unpack_into(self, windows):
        Rwb = self.t["Rwb"].cpu().numpy()
        pwb = self.t["pwb"].cpu().numpy()
        lmp = self.t["lmp"].cpu().numpy()
        so, lo = self.host["slot_off"], self.host["lm_off"]
        for i, w in enumerate(windows):
            P, L = w.Rwb.shape[0], w.lmp.shape[0]
            w.Rwb[:] = Rwb[so[i]:so[i] + P].reshape(P, 3, 3)
            w.pwb[:] = pwb[so[i]:so[i] + P]
            w.lmp[:] = lmp[lo[i]:lo[i] + L]
            pf = _pf_of(w)
            if pf is not None:
                pf.lmp[:] = lmp[lo[i] + L:lo[i] + L + len(pf.host)]


def solve_batch(windows, iters=5, lam0=1e-4, precision="mixed", hold=0, device="cuda", path="auto"):
    """window.solve for every window on the device (one persistent launch, or the large-window path for a few large
    windows: BatchSolver.solve's `path`); windows are updated in place."""
    bs = BatchSolver(windows, device, hold)
    bs.solve(iters, lam0, precision, path=path)
    bs.torch.cuda.synchronize(bs.dev)
    bs.unpack_into(windows)
    res = bs.results()
    for i, w in enumerate(windows):
        res.setdefault("dx0_list", []).append(res["dx0"][i][:6 * w.Rwb.shape[0]])
    return res


def _pf_arrays(Rwb, pwb, Rbc, pbc, lmp, host, rmeas, ris, z):
    f = lambda a, shape: np.ascontiguousarray(a, np.float64).reshape(shape)
    Rwb = f(Rwb, (-1, 3, 3))
    lmp = f(lmp, (-1, 3))
    n = len(lmp)
    return [Rwb, f(pwb, (len(Rwb), 3)), f(Rbc, (3, 3)), f(pbc, (3,)), lmp,
            np.ascontiguousarray(host, np.int64).reshape(n), f(rmeas, (n,)), f(ris, (n,)), f(z, (n, 2))]


def _pf_call(a, isg, fx, fy, cx, cy, huber_k, behind, lam, cost, lmp_out, Hinv_out, ok_out):
    L = _lib.lib()
    p = _lib.ptr
    rc = L.xcb_ba_posefree_host(len(a[0]), p(a[0]), p(a[1]), p(a[2]), p(a[3]), len(a[4]), *[p(x) for x in a[4:]],
                                float(isg), float(fx), float(fy), float(cx), float(cy), float(huber_k), int(bool(behind)),
                                float(lam), p(cost), p(lmp_out), p(Hinv_out),
                                None if ok_out is None else p(ok_out.view(np.uint8)), None)
    if rc != _lib.XCB_OK:
        msg = (L.xcb_last_error() or b"").decode(errors="replace")
        raise (ValueError if rc == _lib.XCB_ERR_ARG else RuntimeError)("posefree: %s" % msg)


def posefree_cost(Rwb, pwb, Rbc, pbc, lmp, host, rmeas, ris, z, isg, fx, fy, cx, cy, B, huber_k, behind):
    """window.posefree_cost on the device (src/xclean/vio/window.py:683-710): the robust cost of the pose-free
    landmarks (host observation + inverse-depth prior; behind=True adds 1e6 per point behind its host), the
    reference's float64 value bit for bit.  B is unused, as in the reference (left observations only)."""
    a = _pf_arrays(Rwb, pwb, Rbc, pbc, lmp, host, rmeas, ris, z)
    cost = np.zeros(1)
    _pf_call(a, isg, fx, fy, cx, cy, huber_k, behind, 0.0, cost, None, None, None)
    return float(cost[0])


def posefree_step(Rwb, pwb, Rbc, pbc, lmp_in, host, rmeas, ris, z, isg, fx, fy, cx, cy, huber_k, lam, lmp_out,
                  Hinv_out, ok_out):
    """window.posefree_step on the device (window.py:713-765): lmp_out = the trial state, Hinv_out (written where
    ok) / ok_out = the damped 3x3 inverses and lm_ok (lam = 0: final_linearisation's marginals); in place, the
    reference's bits.  Returns 0."""
    a = _pf_arrays(Rwb, pwb, Rbc, pbc, lmp_in, host, rmeas, ris, z)
    n = len(a[4])
    for o, dt, shape in ((lmp_out, np.float64, (n, 3)), (Hinv_out, np.float64, (n, 3, 3)), (ok_out, np.bool_, (n,))):
        if not (isinstance(o, np.ndarray) and o.dtype == dt and o.flags.c_contiguous and o.shape == shape):
            raise ValueError("posefree_step: outputs must be C-contiguous arrays of the reference's shapes")
    _pf_call(a, isg, fx, fy, cx, cy, huber_k, False, lam, None, lmp_out, Hinv_out, ok_out)
    return 0


def posefree_marginals(w):
    """final_linearisation's pose-free part (window.py:1003-1006): the block's 3x3 marginals at lam = 0 at the
    window's current state, into w.pf.Hinv / w.pf.ok (nothing when the window has no block)."""
    pf = _pf_of(w)
    if pf is None:
        return
    posefree_step(w.Rwb, w.pwb, w.Rbc, w.pbc, pf.lmp, pf.host, pf.rmeas, pf.ris, pf.z, pf.isg, w.fx, w.fy, w.cx, w.cy,
                  w.huber_k, 0.0, np.zeros_like(pf.lmp), pf.Hinv, pf.ok)


def final_linearisation_batch(windows, device="cuda"):
    """window.final_linearisation for a batch of visual windows (no IMU; a window's marginal prior, w.prior, is added
    to its system): per window a dict of the reference's outputs - H, b (the Schur-reduced system at lam = 0), ob_chi2 (M), lm_ok (L),
    Hll_inv (L,3,3) of the window's own landmarks and observations - and the pose-free block's marginals into
    w.pf.Hinv / w.pf.ok.  -> (list of dicts, robust costs (the block's cost included))."""
    bs = BatchSolver(windows, device, hold=None)
    systems, cost = bs.linearise()
    for w, sy in zip(windows, systems):
        L, M = w.lmp.shape[0], int(np.asarray(w.ob_start)[-1])
        sy["lm_ok"], sy["Hll_inv"], sy["ob_chi2"] = sy["lm_ok"][:L], sy["Hll_inv"][:L], sy["ob_chi2"][:M]
        posefree_marginals(w)
    return systems, cost


def marg_system_batch(windows, lm_masks, device="cuda"):
    """window.marg_system (window.py:1011-1031) for a batch of purely visual windows: for each window and its
    landmark mask, the linear system (H, b) of the masked landmarks' visual observations, Schur'd out, at the current
    state (lam = 0; a window's marginal prior is added, as the reference adds it; no IMU terms), and the state offsets.
    The pose-free block never enters (the reference's marg_system does not see it).  -> list of (H, b, off)."""
    views = []
    for w, m in zip(windows, lm_masks):
        v = _Masked(w, np.ascontiguousarray(m, np.bool_).reshape(w.lmp.shape[0]))
        views.append(v)
    systems, _cost = BatchSolver(views, device, hold=None).linearise()
    return [(s["H"], s["b"], np.arange(w.Rwb.shape[0] + 1, dtype=np.int64) * 6) for s, w in zip(systems, windows)]


class _Masked:
    """A window's arrays with another landmark mask and no pose-free block."""

    def __init__(self, w, mask):
        for k in ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "rho_meas", "rho_isig", "ob_start", "ob_pose", "ob_cam",
                  "ob_z", "ob_isig", "ob_valid", "fx", "fy", "cx", "cy", "B", "huber_k"):
            setattr(self, k, getattr(w, k))
        self.prior = getattr(w, "prior", None)
        self.lm_mask = mask


# --------------------------------------------------------------------- window.py's single-window signatures
def _visual_only(pb, what):
    if getattr(pb, "imu", None):
        raise NotImplementedError("%s: the IMU terms are not on this path (visual windows, with or without a marginal "
                                  "prior over pose slots)" % what)
    if getattr(pb, "dims", None) is not None and (np.asarray(pb.dims) != 6).any():
        raise NotImplementedError("%s: full-state slots (dims 15) are not on this path" % what)


def solve(pb, iters=5, lam0=1e-4, device="cuda"):
    """window.solve (src/xclean/vio/window.py:889-982) for one visual window, pose-free block included, in float64 on
    the device; pb is updated in place.  -> dict(cost0, cost, accepted, iters, lam) as the reference returns."""
    _visual_only(pb, "solve")
    res = solve_batch([pb], iters=iters, lam0=lam0, precision="fp64", hold=None, device=device)
    if int(res["status"][0]) != 0:
        raise RuntimeError("solve: the window exceeds the device solver's limits (status %d)" % int(res["status"][0]))
    return {"cost0": float(res["cost0"][0]), "cost": float(res["cost"][0]), "accepted": int(res["accepted"][0]),
            "iters": int(iters), "lam": float(res["lam"][0])}


def final_linearisation(pb, device="cuda"):
    """window.final_linearisation (window.py:985-1008) for one visual window: -> (H, bvec, ob_chi2, lm_ok, Hll_inv,
    imu_chi2 ([]: no IMU), off), the pose-free block's marginals into pb.pf.Hinv / pb.pf.ok."""
    _visual_only(pb, "final_linearisation")
    (sy,), _cost = final_linearisation_batch([pb], device=device)
    P = pb.Rwb.shape[0]
    return sy["H"], sy["b"], sy["ob_chi2"], sy["lm_ok"], sy["Hll_inv"], [], np.arange(P + 1, dtype=np.int64) * 6


def marg_system(pb, lm_mask, device="cuda"):
    """window.marg_system (window.py:1011-1031) for one visual window: -> (H, b, off)."""
    _visual_only(pb, "marg_system")
    return marg_system_batch([pb], [lm_mask], device=device)[0]
