"""CPU ORACLE of the sliding-window BA (test infrastructure and CPU baseline; never the product path).

numpy wrappers over oracle/ba_oracle.c, the float64 restatement of the reference's stereo window solve
(src/xclean/vio/window.py: build_system, visual_cost, back_substitute, apply_update, solve).  Windows are
xclean_b200.backend.synth_ba.Window objects (the fields of window.Problem)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import front_oracle as _fo

c_double, c_int, P = ctypes.c_double, ctypes.c_int, ctypes.c_void_p


class XoWindow(ctypes.Structure):
    _fields_ = [("P", c_int), ("L", c_int), ("M", c_int), ("Rwb", P), ("pwb", P), ("Rbc", P), ("pbc", P),
                ("lmp", P), ("lm_host", P), ("lm_mask", P), ("rho_meas", P), ("rho_isig", P), ("ob_start", P),
                ("ob_pose", P), ("ob_cam", P), ("ob_z", P), ("ob_isig", P), ("ob_valid", P), ("fx", c_double),
                ("fy", c_double), ("cx", c_double), ("cy", c_double), ("B", c_double), ("huber_k", c_double),
                ("hold", c_int)]


def _lib():
    L = _fo.lib()
    W = ctypes.POINTER(XoWindow)
    L.xo_ba_build_system.restype = c_double
    L.xo_ba_build_system.argtypes = [W, P, P, P, c_double, P, P, P, P, P, P, P]
    L.xo_ba_visual_cost.restype = c_double
    L.xo_ba_visual_cost.argtypes = [W, P, P, P]
    L.xo_ba_step.restype = c_double
    L.xo_ba_step.argtypes = [W, c_double, P, P, P, P, P, ctypes.POINTER(c_int)]
    L.xo_ba_solve.restype = None
    L.xo_ba_solve.argtypes = [W, c_int, c_double, P, P]
    L.xo_ba_solve_batch.restype = None
    L.xo_ba_solve_batch.argtypes = [W, c_int, c_int, c_double, c_int, P]
    return L


def _arr(w, name, dt):
    a = np.ascontiguousarray(getattr(w, name), dt)
    setattr(w, name, a)
    return a


def as_struct(w, hold=0):
    """A ctypes view of a Window (its arrays are made contiguous in place; Rwb / pwb / lmp are updated in place)."""
    keep = []
    s = XoWindow()
    s.P, s.L, s.M = int(w.Rwb.shape[0]), int(w.lmp.shape[0]), int(w.ob_pose.shape[0])
    for name, dt in (("Rwb", np.float64), ("pwb", np.float64), ("Rbc", np.float64), ("pbc", np.float64),
                     ("lmp", np.float64), ("lm_host", np.int64), ("lm_mask", np.uint8), ("rho_meas", np.float64),
                     ("rho_isig", np.float64), ("ob_start", np.int64), ("ob_pose", np.int64), ("ob_cam", np.int64),
                     ("ob_z", np.float64), ("ob_isig", np.float64), ("ob_valid", np.uint8)):
        a = _arr(w, name, dt)
        keep.append(a)
        setattr(s, name, a.ctypes.data)
    s.fx, s.fy, s.cx, s.cy, s.B, s.huber_k = w.fx, w.fy, w.cx, w.cy, w.B, w.huber_k
    s.hold = -1 if hold is None else int(hold)
    s._keep = keep
    return s


def build_system(w, lam, want_chi2=False):
    """-> (H (6P,6P), b (6P,), cost, Hll_inv (L,3,3), bl (L,3), Hlp (L,P,3,6), lm_ok (L,)[, ob_chi2 (M,)])"""
    s = as_struct(w, None)
    Pn, L, M = s.P, s.L, s.M
    H = np.zeros((6 * Pn, 6 * Pn))
    b = np.zeros(6 * Pn)
    Hi = np.zeros((max(L, 1), 3, 3))
    bl = np.zeros((max(L, 1), 3))
    Hlp = np.zeros((max(L, 1), Pn, 3, 6))
    ok = np.zeros(max(L, 1), np.uint8)
    chi = np.zeros(max(M, 1))
    c = _lib().xo_ba_build_system(ctypes.byref(s), s.Rwb, s.pwb, s.lmp, c_double(lam), H.ctypes.data, b.ctypes.data,
                                  Hi.ctypes.data, bl.ctypes.data, Hlp.ctypes.data, ok.ctypes.data, chi.ctypes.data)
    if want_chi2:
        return H, b, c, Hi[:L], bl[:L], Hlp[:L], ok[:L].astype(bool), chi[:M]
    return H, b, c, Hi[:L], bl[:L], Hlp[:L], ok[:L].astype(bool)


def visual_cost(w):
    s = as_struct(w, None)
    return _lib().xo_ba_visual_cost(ctypes.byref(s), s.Rwb, s.pwb, s.lmp)


def step(w, lam, hold=0):
    """The first reduced pose step of a linearisation: -> (dx (6P,), cost, ok)."""
    s = as_struct(w, hold)
    Pn, L = s.P, s.L
    dx = np.zeros(6 * Pn)
    Hi = np.zeros((max(L, 1), 9))
    bl = np.zeros((max(L, 1), 3))
    Hlp = np.zeros((max(L, 1), Pn, 18))
    ok_l = np.zeros(max(L, 1), np.uint8)
    ok = c_int(0)
    c = _lib().xo_ba_step(ctypes.byref(s), c_double(lam), dx.ctypes.data, Hi.ctypes.data, bl.ctypes.data,
                          Hlp.ctypes.data, ok_l.ctypes.data, ctypes.byref(ok))
    return dx, c, bool(ok.value)


def solve(w, iters=5, lam0=1e-4, hold=0):
    """window.solve (purely visual) in place.  -> dict(cost0, cost, accepted, lam, dx0 = the first pose step)."""
    s = as_struct(w, hold)
    out = np.zeros(4)
    dx0 = np.zeros(6 * s.P)
    _lib().xo_ba_solve(ctypes.byref(s), int(iters), c_double(lam0), out.ctypes.data, dx0.ctypes.data)
    return {"cost0": out[0], "cost": out[1], "accepted": int(out[2]), "lam": out[3], "dx0": dx0}


def solve_batch(windows, iters=5, lam0=1e-4, hold=0, nthreads=None):
    """All windows in place, OpenMP over windows.  -> (n, 4) [cost0, cost, accepted, lam]."""
    import os
    structs = [as_struct(w, hold) for w in windows]
    arr = (XoWindow * len(structs))(*structs)
    arr_p = ctypes.cast(arr, ctypes.POINTER(XoWindow))
    out = np.zeros((len(structs), 4))
    _lib().xo_ba_solve_batch(arr_p, len(structs), int(iters), c_double(lam0), int(nthreads or os.cpu_count() or 1),
                             out.ctypes.data)
    return out


def _pf_common(Rwb, pwb, Rbc, pbc, lmp, host, rmeas, ris, z):
    f = lambda a: np.ascontiguousarray(a, np.float64)
    Rwb, pwb, Rbc, pbc = f(Rwb).reshape(-1, 3, 3), f(pwb).reshape(-1, 3), f(Rbc).reshape(3, 3), f(pbc).reshape(3)
    lmp = f(lmp).reshape(-1, 3)
    host = np.ascontiguousarray(host, np.int64).reshape(-1)
    return Rwb, pwb, Rbc, pbc, lmp, host, f(rmeas).reshape(-1), f(ris).reshape(-1), f(z).reshape(-1, 2)


def posefree_cost(Rwb, pwb, Rbc, pbc, lmp, host, rmeas, ris, z, isg, fx, fy, cx, cy, B, huber_k, behind):
    """window.posefree_cost (window.py:683-710)."""
    L = _fo.lib()
    L.xo_ba_posefree_cost.restype = c_double
    a = _pf_common(Rwb, pwb, Rbc, pbc, lmp, host, rmeas, ris, z)
    return L.xo_ba_posefree_cost(len(a[0]), *[ctypes.c_void_p(x.ctypes.data) for x in a[:4]], len(a[4]),
                                 *[ctypes.c_void_p(x.ctypes.data) for x in a[4:]], c_double(isg), c_double(fx),
                                 c_double(fy), c_double(cx), c_double(cy), c_double(B), c_double(huber_k),
                                 int(bool(behind)))


def posefree_step(Rwb, pwb, Rbc, pbc, lmp_in, host, rmeas, ris, z, isg, fx, fy, cx, cy, huber_k, lam, lmp_out,
                  Hinv_out, ok_out):
    """window.posefree_step (window.py:713-765): lmp_out, Hinv_out (where ok), ok_out in place."""
    L = _fo.lib()
    L.xo_ba_posefree_step.restype = None
    a = _pf_common(Rwb, pwb, Rbc, pbc, lmp_in, host, rmeas, ris, z)
    n = len(a[4])
    for o, dt, shape in ((lmp_out, np.float64, (n, 3)), (Hinv_out, np.float64, (n, 3, 3)), (ok_out, np.bool_, (n,))):
        assert o.dtype == dt and o.flags.c_contiguous and o.shape == shape
    L.xo_ba_posefree_step(len(a[0]), *[ctypes.c_void_p(x.ctypes.data) for x in a[:4]], n,
                          *[ctypes.c_void_p(x.ctypes.data) for x in a[4:]], c_double(isg), c_double(fx), c_double(fy),
                          c_double(cx), c_double(cy), c_double(huber_k), c_double(lam),
                          ctypes.c_void_p(lmp_out.ctypes.data), ctypes.c_void_p(Hinv_out.ctypes.data),
                          ctypes.c_void_p(ok_out.ctypes.data))
    return 0
