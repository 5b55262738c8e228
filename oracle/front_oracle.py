"""CPU ORACLE of the xclean frontend (test infrastructure; never the product path).

Thin numpy wrappers over oracle/liboracle.so (front_oracle.c), with the reference's Python-level conventions:

  response(gray, dy_vend, dx_vend)        = cv2.cornerMinEigenVal(gray, 3, 3)          (features.py:299)
  noise_floor(gray, Q)                    = features.noise_floor_8u                    (features.py:57-73)
  detect(gray, n, Q, vend)                = front/detect.Detector.__call__ keypoints   (detect.py:60-75)
  blur(gray, kf, vr, vc) / orb(...)       = Frontend.describe                          (features.py:405-421)
  stereo(left, right, kp, ...)            = front/stereo1d.disparities                 (stereo1d.py:492-522)
  hamming(A, B) / match_desc(d0, d1)      = mapmatch_fast._bf_mutual / match_desc       (mapmatch_fast.py:46-111)
  mapmatch(kp, desc, uv, S, lmd, lnd, W, H) = mapmatch.MapMatcher.match                  (mapmatch.py:148-169)
  predict_projection(...)                 = vio/window.predict_projection               (window.py:1032-1144)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

HALF_REF = 5                    # the reference's patch half-size (stereo/epipolar.py:35)
MAX_DISP = 128                  # stereo/sgm32.py:68
HAMMING_CHANCE = 104            # features.py:50
RATIO = 0.8                     # features.py:51
CHI2_2_999 = 13.815510557964274  # mapmatch.py:29
GRID = 16                       # mapmatch.py:30

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = _build.OUT
        if not os.path.exists(path):
            _build.build()
        _LIB = ctypes.CDLL(path)
        _LIB.xo_noise_floor.restype = ctypes.c_double
        _LIB.xo_cell.restype = ctypes.c_double
        _LIB.xo_min_dist.restype = ctypes.c_double
        _LIB.xo_frames.restype = ctypes.c_long
    return _LIB


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def response(gray, dy_vend, dx_vend):
    g = np.ascontiguousarray(gray, np.uint8)
    H, W = g.shape
    R = np.empty((H, W), np.float32)
    lib().xo_response(_p(g), H, W, int(dy_vend), int(dx_vend), _p(R))
    return R


def noise_floor(gray, Q):
    g = np.ascontiguousarray(gray, np.uint8)
    H, W = g.shape
    ff = ctypes.c_float(0.0)
    fl = lib().xo_noise_floor(_p(g), H, W, ctypes.c_double(Q), ctypes.byref(ff))
    return float(fl), np.float32(ff.value)


def detect_from_response(R, budget, floor_f, cap=None):
    R = np.ascontiguousarray(R, np.float32)
    H, W = R.shape
    cap = int(cap or budget)
    kp = np.empty((max(cap, 1), 2), np.float32)
    nc = ctypes.c_int(0)
    n = lib().xo_detect(_p(R), H, W, int(budget), ctypes.c_float(floor_f), cap, _p(kp), ctypes.byref(nc))
    return kp[:n].copy()


def detect(gray, budget, Q, dy_vend, dx_vend, cap=None):
    R = response(gray, dy_vend, dx_vend)
    _fl, ff = noise_floor(gray, Q)
    return detect_from_response(R, budget, ff, cap)


def blur(gray, kf, vr, vc):
    g = np.ascontiguousarray(gray, np.uint8)
    H, W = g.shape
    out = np.empty((H + 64, W + 64), np.uint8)
    kf = np.ascontiguousarray(kf, np.float32)
    lib().xo_blur(_p(g), H, W, _p(kf), int(vr), int(vc), _p(out))
    return out


def orb(blurred, kp, pattern):
    B = np.ascontiguousarray(blurred, np.uint8)
    kp = np.ascontiguousarray(kp, np.float32).reshape(-1, 2)
    pat = np.ascontiguousarray(pattern, np.int8).reshape(256, 4)
    d = np.zeros((len(kp), 32), np.uint8)
    if len(kp):
        lib().xo_orb(_p(B), B.shape[1], _p(kp), len(kp), _p(pat), _p(d))
    return d


def shift_rows(right, dy):
    r = np.ascontiguousarray(right, np.uint8)
    H, W = r.shape
    out = np.empty((H, W), np.float32)
    lib().xo_shift_rows(_p(r), H, W, ctypes.c_double(float(dy)), _p(out))
    return out


def stereo(left, right, kp, dlo=None, dhi=None, dy=0.0, band=0, half=HALF_REF):
    """stereo1d.disparities -> (d, sig, ok, zn, last_dy) (last_dy = column-scan offset + dy, NaN unless set)."""
    L = np.ascontiguousarray(left, np.uint8)
    H, W = L.shape
    kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 2)
    n = len(kp)
    lo = np.zeros(n, np.int64) if dlo is None else np.ascontiguousarray(dlo, np.int64)
    hi = np.full(n, MAX_DISP - 1, np.int64) if dhi is None else np.ascontiguousarray(dhi, np.int64)
    d = np.zeros(n)
    s = np.full(n, np.inf)
    ok = np.zeros(n, np.uint8)
    zn = np.zeros(n)
    ody = np.full(n, np.nan)
    if n:
        bad = ~(np.isfinite(kp[:, 0]) & np.isfinite(kp[:, 1]) & (kp[:, 0] >= 0) & (kp[:, 0] < W) & (kp[:, 1] >= 0)
                & (kp[:, 1] < H))
        if bad.any():
            kp = kp.copy()
            kp[bad] = -float(half + 3)
        Rs = shift_rows(right, dy)
        lib().xo_stereo(_p(L), _p(Rs), H, W, _p(kp), _p(lo), _p(hi), n, int(band), int(half), _p(d), _p(s), _p(ok),
                        _p(zn), _p(ody))
    return d, s, ok.astype(bool), zn, ody + float(dy)


def hamming(A, B):
    A = np.ascontiguousarray(A, np.uint8)
    B = np.ascontiguousarray(B, np.uint8)
    L, N = len(A), len(B)
    o1 = np.empty(L, np.int32)
    o2 = np.empty(L, np.int32)
    oi = np.empty(L, np.int32)
    ci = np.empty(N, np.int32)
    lib().xo_hamming(_p(A), L, _p(B), N, _p(o1), _p(o2), _p(oi), _p(ci))
    return o1.astype(np.int64), o2.astype(np.int64), oi.astype(np.int64), ci.astype(np.int64)


def match_desc(d0, d1):
    A = np.ascontiguousarray(d0, np.uint8)
    B = np.ascontiguousarray(d1, np.uint8)
    m0 = np.empty(max(len(A), 1), np.int64)
    m1 = np.empty(max(len(A), 1), np.int64)
    m = lib().xo_match(_p(A), len(A), _p(B), len(B), HAMMING_CHANCE, ctypes.c_double(RATIO), _p(m0), _p(m1))
    return m0[:m].copy(), m1[:m].copy()


def mapmatch(kp, desc, uv_pred, S_uv, lm_desc, lm_ndesc, W, H, chi2=CHI2_2_999):
    """MapMatcher(W, H).match(kp, desc, uv_pred, S_uv, lm_desc, lm_ndesc, chi2) -> (kp index per landmark or -1,
    Hamming distance, Mahalanobis d2), the reference's dtypes (int64, int64, float64)."""
    L = len(uv_pred)
    out_kp = np.full(L, -1, np.int64)
    out_d = np.full(L, 9999, np.int64)
    out_d2 = np.full(L, np.inf)
    if L == 0 or len(kp) == 0:
        return out_kp, out_d, out_d2
    kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 2)
    kd = np.ascontiguousarray(desc, np.uint8).reshape(len(kp), 32)
    uv = np.ascontiguousarray(uv_pred, np.float64).reshape(L, 2)
    S = np.ascontiguousarray(S_uv, np.float64).reshape(L, 2, 2)
    D = lm_desc.shape[1]
    ld = np.ascontiguousarray(lm_desc, np.uint8).reshape(L, D, 32)
    lnd = np.ascontiguousarray(lm_ndesc, np.int64).reshape(L)
    if (lnd > D).any():
        raise ValueError("lm_ndesc above the descriptor slots of lm_desc")
    gw, gh = -(-int(W) // GRID), -(-int(H) // GRID)
    lib().xo_mapmatch(_p(kp), len(kp), _p(kd), _p(uv), _p(S), _p(ld), D, _p(lnd), L, gw, gh, ctypes.c_double(chi2),
                      ctypes.c_double(RATIO), HAMMING_CHANCE, _p(out_kp), _p(out_d), _p(out_d2))
    return out_kp, out_d, out_d2


def predict_projection(Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, sig_px, fx, fy, cx, cy, W, H, uv, S, ok,
                       depth):
    """window.predict_projection: writes ok, and uv / depth / S where the reference writes them (in place)."""
    ins = [np.ascontiguousarray(a, np.float64) for a in (Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl)]
    L = len(ins[6])
    for a, dt in ((uv, np.float64), (S, np.float64), (depth, np.float64), (ok, np.bool_)):
        assert a.dtype == dt and a.flags.c_contiguous and len(a) == L
    lib().xo_predict_projection(*[_p(a) for a in ins], ctypes.c_double(sig_px), ctypes.c_double(fx),
                                ctypes.c_double(fy), ctypes.c_double(cx), ctypes.c_double(cy), ctypes.c_double(W),
                                ctypes.c_double(H), L, _p(uv), _p(S), _p(ok.view(np.uint8)), _p(depth))
    return 0


def mapmatch_frames(kp32, counts_kp, desc, uv, S, lm_desc, lm_ndesc, counts_lm, W, H, chi2=CHI2_2_999,
                    nthreads=None):
    """F frames of mapmatch with float32 keypoints (F, Nmax, 2), descriptors (F, Nmax, 32), landmark arrays
    (F, Lmax, ...); OpenMP over frames.  -> (out_kp, out_d, out_d2) of shape (F, Lmax)."""
    kp32 = np.ascontiguousarray(kp32, np.float32)
    F, Nmax = kp32.shape[:2]
    Lmax, D = lm_desc.shape[1], lm_desc.shape[2]
    desc = np.ascontiguousarray(desc, np.uint8)
    uv = np.ascontiguousarray(uv, np.float64)
    S = np.ascontiguousarray(S, np.float64)
    ld = np.ascontiguousarray(lm_desc, np.uint8)
    lnd = np.ascontiguousarray(lm_ndesc, np.int64)
    ck = np.ascontiguousarray(counts_kp, np.int32)
    cl = np.ascontiguousarray(counts_lm, np.int32)
    out_kp = np.full((F, Lmax), -1, np.int64)
    out_d = np.full((F, Lmax), 9999, np.int64)
    out_d2 = np.full((F, Lmax), np.inf)
    gw, gh = -(-int(W) // GRID), -(-int(H) // GRID)
    lib().xo_mapmatch_frames(_p(kp32), _p(ck), Nmax, _p(desc), _p(uv), _p(S), _p(ld), D, _p(lnd), _p(cl), Lmax, F, gw,
                             gh, ctypes.c_double(chi2), int(nthreads or os.cpu_count() or 1), _p(out_kp), _p(out_d),
                             _p(out_d2))
    return out_kp, out_d, out_d2


def lk_solve_inv(As, gs):
    As = np.ascontiguousarray(As, np.float64).reshape(-1, 3, 3)
    gs = np.ascontiguousarray(gs, np.float64).reshape(-1, 3)
    n = len(As)
    X = np.empty((n, 3))
    Inv = np.empty((n, 3, 3))
    lib().xo_lk_solve_inv(_p(As), _p(gs), n, _p(X), _p(Inv))
    return X, Inv


def frames(left, right, budget, Q, calib, pattern, half, dlo, dhi, cap=None, nthreads=None):
    """The whole per-frame path over F frames (frames f-1 -> f matched), OpenMP over frames.  -> dict of arrays."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    F, H, W = left.shape
    cap = int(cap or budget)
    nthreads = int(nthreads or os.cpu_count() or 1)
    kf = np.ascontiguousarray(calib["kf"], np.float32)
    pat = np.ascontiguousarray(pattern, np.int8)
    out = dict(counts=np.zeros(F, np.int32), kp=np.zeros((F, cap, 2), np.float32),
               desc=np.zeros((F, cap, 32), np.uint8), d=np.zeros((F, cap)), sig=np.zeros((F, cap)),
               ok=np.zeros((F, cap), np.uint8), zn=np.zeros((F, cap)), dy=np.zeros((F, cap)),
               m0=np.zeros((F, cap), np.int64), m1=np.zeros((F, cap), np.int64), nmatch=np.zeros(F, np.int32))
    lib().xo_frames(_p(left), _p(right), F, H, W, int(budget), cap, ctypes.c_double(Q), int(calib["dy_vend"]),
                    int(calib["dx_vend"]), _p(kf), int(calib["blur_vr"]), int(calib["blur_vc"]), _p(pat), int(half),
                    int(dlo), int(dhi), nthreads, _p(out["counts"]), _p(out["kp"]), _p(out["desc"]), _p(out["d"]),
                    _p(out["sig"]), _p(out["ok"]), _p(out["zn"]), _p(out["dy"]), _p(out["m0"]), _p(out["m1"]),
                    _p(out["nmatch"]))
    return out
