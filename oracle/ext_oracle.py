"""CPU oracle of the frontend's multi-scale, oriented extras (test infrastructure; never the product path):
oracle/ext_oracle.c for the pixel work, and the host-side definitions restated here:

  fast(img, t, nms)                  = cv2.FastFeatureDetector_create(t, nms, TYPE_9_16).detect, scores as responses
  pyr_down(img, wd, hd)              = cv2.resize(img, (wd, hd), interpolation=cv2.INTER_LINEAR_EXACT)
  level_sizes(w, h, levels, scale)   = the level sizes cv2's ORB gives (rint(n / scale^l) in float32)
  steered_patterns(pattern)          = the reference's ORB tests rotated as cv2.ORB.compute rotates them at
                                       KeyPoint.angle = 12 k (float32 cos / sin, float32 products, round half even)
  blur(...) / orb                    = the reference's describe stage (features.py:405-421), from front_oracle
  orbx(img, ...)                     = the per-frame multi-scale pipeline of xcb_orbx, slot for slot

These extras go beyond the reference (src/xclean/stages/features.py:27-28, :102-103; gpu_front.py:1712-1717: one
level, no orientation).  Only tests/ import this module.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import front_oracle as _fo

BINS = 30
PAD = 32


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _lib():
    L = _fo.lib()
    if not getattr(L, "_ext_sigs", False):
        L.xo_fast.restype = ctypes.c_long
        L.xo_fast.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                              ctypes.c_void_p, ctypes.c_void_p]
        L.xo_fast_select.restype = ctypes.c_long
        L.xo_fast_select.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
        L.xo_pyr_down.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.c_int]
        L.xo_ic_bins.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_long,
                                 ctypes.c_void_p, ctypes.c_void_p]
        L.xo_orb_steer.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L._ext_sigs = True
    return L


def fast(img, threshold, nonmax=True):
    """-> (kp (n, 2) float32 (x, y) row-major, score (n,) float32)."""
    g = np.ascontiguousarray(img, np.uint8)
    H, W = g.shape
    cap = H * W
    kp = np.zeros((cap, 2), np.float32)
    rs = np.zeros(cap, np.float32)
    n = _lib().xo_fast(_p(g), H, W, int(threshold), 1 if nonmax else 0, cap, _p(kp), _p(rs))
    return kp[:n].copy(), rs[:n].copy()


def select(kp, resp, W, H, edge, quota):
    kp = np.ascontiguousarray(kp, np.float32).reshape(-1, 2)
    resp = np.ascontiguousarray(resp, np.float32)
    ko = np.zeros((max(quota, 1), 2), np.float32)
    ro = np.zeros(max(quota, 1), np.float32)
    n = _lib().xo_fast_select(_p(kp), _p(resp), len(kp), int(W), int(H), int(edge), int(quota), _p(ko), _p(ro))
    return ko[:n].copy(), ro[:n].copy()


def pyr_down(img, wd, hd):
    g = np.ascontiguousarray(img, np.uint8)
    out = np.zeros((hd, wd), np.uint8)
    _lib().xo_pyr_down(_p(g), g.shape[0], g.shape[1], _p(out), int(hd), int(wd))
    return out


def ic_bins(img, kp):
    """-> (bins (n,) int32, moments (n, 2) int64 (m10, m01))."""
    g = np.ascontiguousarray(img, np.uint8)
    kp = np.ascontiguousarray(kp, np.float32).reshape(-1, 2)
    bins = np.zeros(len(kp), np.int32)
    mom = np.zeros((len(kp), 2), np.int64)
    if len(kp):
        _lib().xo_ic_bins(_p(g), g.shape[0], g.shape[1], _p(kp), len(kp), _p(bins), _p(mom))
    return bins, mom


def orb_steer(blurred, kp, bins, patterns, pad=PAD):
    B = np.ascontiguousarray(blurred, np.uint8)
    kp = np.ascontiguousarray(kp, np.float32).reshape(-1, 2)
    bins = np.ascontiguousarray(bins, np.int32)
    pats = np.ascontiguousarray(patterns, np.int8).reshape(BINS, 256, 4)
    d = np.zeros((len(kp), 32), np.uint8)
    if len(kp):
        _lib().xo_orb_steer(_p(B), B.shape[0], B.shape[1], int(pad), _p(kp), len(kp), _p(bins), _p(pats), _p(d))
    return d


def level_sizes(W, H, levels, scale):
    out = []
    for lv in range(levels):
        s = np.float32(scale ** lv)
        out.append((int(np.rint(np.float32(W) / s)), int(np.rint(np.float32(H) / s)), float(s)))
    return out


def quotas(nfeatures, levels, scale):
    """A geometric share of nfeatures per level (ratio 1 / scale), rounded half to even; the last level the rest."""
    f = 1.0 / scale
    share = nfeatures * (1.0 - f) / (1.0 - f ** levels)
    q, tot = [], 0
    for _ in range(levels - 1):
        n = min(int(np.rint(share)), nfeatures - tot)
        q.append(n)
        tot += n
        share *= f
    q.append(max(nfeatures - tot, 0))
    return q


def steered_patterns(pattern):
    """(256, 4) test pairs -> (30, 256, 4) int8: bin k rotated by 12 k degrees in cv2.ORB.compute's arithmetic."""
    pat = np.asarray(pattern).reshape(256, 4)
    out = np.zeros((BINS, 256, 4), np.int8)
    d2r = np.float32(math.pi / 180.0)
    for k in range(BINS):
        ang = np.float32(np.float32(12 * k) * d2r)
        a = np.float32(math.cos(float(ang)))
        b = np.float32(math.sin(float(ang)))
        for j in range(256):
            for (cx, cy, c) in ((0, 1, 0), (2, 3, 2)):
                px, py = np.float32(pat[j, cx]), np.float32(pat[j, cy])
                out[k, j, c] = int(np.rint(np.float32(np.float32(px * a) - np.float32(py * b))))
                out[k, j, c + 1] = int(np.rint(np.float32(np.float32(px * b) + np.float32(py * a))))
    return out


def orbx(img, levels, scale, nfeatures, threshold, edge, nonmax, patterns, blur_calib):
    """The per-frame pipeline, slot for slot: blur_calib[l] = (kf7, vr, vc) of level l's padded width.
    -> dict of slot arrays (kp, kp_level, resp, level, bins, desc) and per-level counts, plus the level images."""
    sizes = level_sizes(img.shape[1], img.shape[0], levels, scale)
    q = quotas(nfeatures, levels, scale)
    off = np.concatenate([[0], np.cumsum(q)]).astype(int)
    out = {"kp": np.zeros((nfeatures, 2), np.float32), "kp_level": np.zeros((nfeatures, 2), np.float32),
           "resp": np.zeros(nfeatures, np.float32), "level": np.zeros(nfeatures, np.int32),
           "bins": np.zeros(nfeatures, np.int32), "desc": np.zeros((nfeatures, 32), np.uint8),
           "counts": np.zeros(levels, np.int32), "levels": []}
    cur = np.ascontiguousarray(img, np.uint8)
    for lv in range(levels):
        W, H, s = sizes[lv]
        if lv:
            cur = pyr_down(cur, W, H)
        out["levels"].append(cur)
        kp, rs = fast(cur, threshold, nonmax)
        ks, rsel = select(kp, rs, W, H, edge, q[lv])
        n = len(ks)
        o = off[lv]
        out["counts"][lv] = n
        bins, _m = ic_bins(cur, ks)
        kf, vr, vc = blur_calib[lv]
        B = _fo.blur(cur, kf, vr, vc)
        out["kp_level"][o:o + n] = ks
        out["kp"][o:o + n] = ks * np.float32(s)
        out["resp"][o:o + n] = rsel
        out["level"][o:o + n] = lv
        out["bins"][o:o + n] = bins
        out["desc"][o:o + n] = orb_steer(B, ks, bins, patterns)
    return out
