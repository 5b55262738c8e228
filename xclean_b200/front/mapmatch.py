"""Gated map matching on the device: the drop-in for xclean.front.mapmatch / xclean.front.mapmatch_fast.

Same API and the same outputs as the reference (src/xclean/front/mapmatch.py:132-169, mapmatch_fast.py:164-184):

    mm = MapMatcher(width, height)
    lm_kp, dist, d2 = mm.match(kp, desc, uv_pred, S_uv, lm_desc, lm_ndesc, chi2=CHI2_2_999)

- candidates of landmark l: the keypoints inside its chi2 (2 dof, 0.999) ellipse of S_uv[l], found through a 16-px
  grid over the image;
- score: the minimum Hamming distance over the landmark's first lm_ndesc[l] descriptors;
- acceptance: best <= HAMMING_CHANCE (104), best < RATIO (0.8) x second best among the in-gate candidates, then one
  landmark per keypoint (smaller distance, then smaller d2, then lower landmark index).

Every call runs three kernels of libxcb200.so (xcb_mm_match_host, include/xcb200.h); there is no CPU path.
`match_dev` (no reference counterpart) matches a batch of frames already in device memory, e.g. the frontend's
keypoints and descriptors, in the same three launches.

Also here, the gating prediction that feeds the matcher (src/xclean/vio/window.py:1032-1144):

    predict_projection(Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, sig_px, fx, fy, cx, cy, W, H,
                       uv, S, ok, depth)                 # = window.predict_projection, in place, bit-identical
    uv, S, ok, depth, k, d, d2 = mm.predict_match(...)  # _project + match on the in-view landmarks, one call
"""
from __future__ import annotations

import ctypes
import math
import threading

import numpy as np

from .. import _lib

CHI2_2_999 = 13.815510557964274        # mapmatch.py:29
GRID = 16                              # mapmatch.py:30
HAMMING_CHANCE = 104                   # features.py:50
RATIO = 0.8                            # features.py:51


class MapMatcher:
    """mapmatch.MapMatcher on the device; `max_frames`, `max_kp`, `max_lm` size the batched `match_dev` (the
    single-frame `match` grows its buffers as needed)."""

    def __init__(self, width, height, max_frames=1, max_kp=2048, max_lm=2048):
        self.W = int(width)
        self.H = int(height)
        self.gw = int(math.ceil(self.W / GRID))
        self.gh = int(math.ceil(self.H / GRID))
        self.stats = {"calls": 0, "landmarks": 0, "matched": 0}
        self.max_frames, self.max_kp, self.max_lm = int(max_frames), int(max_kp), int(max_lm)
        self.L = _lib.lib()
        h = ctypes.c_void_p()
        self._chk(self.L.xcb_mm_create(self.W, self.H, self.max_frames, self.max_kp, self.max_lm, ctypes.byref(h)),
                  "xcb_mm_create", None)
        self._h = h
        self._owner = threading.get_ident()

    def close(self):
        if getattr(self, "_h", None):
            self.L.xcb_mm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what, h="self"):
        if rc == _lib.XCB_OK:
            return
        hh = self._h if h == "self" else h
        msg = (self.L.xcb_mm_last_error(hh) if hh else self.L.xcb_last_error()) or b""
        msg = msg.decode(errors="replace")
        if rc in (_lib.XCB_ERR_ARG, _lib.XCB_ERR_CAPACITY):
            raise ValueError("%s: %s" % (what, msg))
        raise RuntimeError("%s failed (%d): %s" % (what, rc, msg))

    def _own(self):
        if threading.get_ident() != self._owner:
            raise RuntimeError("mapmatch: called from a second thread (the MapMatcher buffers are single-owner)")

    def match(self, kp, desc, uv_pred, S_uv, lm_desc, lm_ndesc, chi2=CHI2_2_999, stream=0):
        """kp (N,2), desc (N,32) uint8; uv_pred (L,2); S_uv (L,2,2) innovation covariances; lm_desc (L,D,32) uint8,
        lm_ndesc (L,) number of valid descriptors.  -> (kp index per landmark or -1, Hamming distance, Mahalanobis
        d2) as int64, int64, float64 arrays of length L."""
        self._own()
        L = len(uv_pred)
        out_kp = np.full(L, -1, np.int64)
        out_d = np.full(L, 9999, np.int64)
        out_d2 = np.full(L, np.inf)
        self.stats["calls"] += 1
        self.stats["landmarks"] += L
        if L == 0 or len(kp) == 0:
            return out_kp, out_d, out_d2
        kp64 = np.ascontiguousarray(kp, np.float64).reshape(-1, 2)
        N = len(kp64)
        kd = np.ascontiguousarray(desc, np.uint8).reshape(N, 32)
        uv = np.ascontiguousarray(uv_pred, np.float64).reshape(L, 2)
        S = np.ascontiguousarray(S_uv, np.float64).reshape(L, 2, 2)
        lm_desc = np.asarray(lm_desc)
        D = int(lm_desc.shape[1])
        ld = np.ascontiguousarray(lm_desc, np.uint8).reshape(L, D, 32)
        lnd = np.ascontiguousarray(lm_ndesc, np.int64).reshape(L)
        p = _lib.ptr
        self._chk(self.L.xcb_mm_match_host(self._h, p(kp64), N, p(kd), p(uv), p(S), p(ld), D, p(lnd), L,
                                           float(chi2), p(out_kp), p(out_d), p(out_d2),
                                           ctypes.c_void_p(int(stream) or None)), "mapmatch")
        self.stats["matched"] += int((out_kp >= 0).sum())
        return out_kp, out_d, out_d2

    def predict_match(self, Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, sig_px, fx, fy, cx, cy, kp, desc,
                      lm_desc, lm_ndesc, chi2=CHI2_2_999, stream=0):
        """The engine's tracking step (engine_live.py:1580-1582): predict_projection of the L landmarks into the
        predicted pose over this matcher's W x H (uv NaN / S 0 / depth 0 where the reference writes nothing, as
        _project pre-fills them), then the gated matching of the in-view ones.  -> (uv, S, ok, depth, kp index,
        distance, d2); the last three have one entry per landmark and equal match(kp, desc, uv[sel], S[sel],
        lm_desc[sel], lm_ndesc[sel]) at sel = nonzero(ok), defaults elsewhere."""
        self._own()
        lmp = np.ascontiguousarray(lmp, np.float64).reshape(-1, 3)
        L = len(lmp)
        uv = np.full((L, 2), np.nan)
        S = np.zeros((L, 2, 2))
        ok = np.zeros(L, np.bool_)
        depth = np.zeros(L)
        out_kp = np.full(L, -1, np.int64)
        out_d = np.full(L, 9999, np.int64)
        out_d2 = np.full(L, np.inf)
        kp64 = np.ascontiguousarray(kp, np.float64).reshape(-1, 2)
        N = len(kp64)
        kd = np.ascontiguousarray(desc, np.uint8).reshape(N, 32)
        lm_desc = np.asarray(lm_desc)
        D = int(lm_desc.shape[1]) if lm_desc.ndim == 3 else 0
        ld = np.ascontiguousarray(lm_desc, np.uint8).reshape(L, D, 32)
        lnd = np.ascontiguousarray(lm_ndesc, np.int64).reshape(L)
        ins = _pred_inputs(Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, L)
        p = _lib.ptr
        self._chk(self.L.xcb_mm_predict_match_host(self._h, *[p(a) for a in ins], float(sig_px), float(fx), float(fy),
                                                   float(cx), float(cy), L, p(kp64), N, p(kd), p(ld), D, p(lnd),
                                                   float(chi2), p(uv), p(S), p(ok.view(np.uint8)), p(depth),
                                                   p(out_kp), p(out_d), p(out_d2),
                                                   ctypes.c_void_p(int(stream) or None)), "mapmatch.predict_match")
        self.stats["calls"] += 1
        self.stats["landmarks"] += int(ok.sum())
        self.stats["matched"] += int((out_kp >= 0).sum())
        return uv, S, ok, depth, out_kp, out_d, out_d2

    def set_tuning(self, knob, value):
        """A launch-shape knob (xclean_b200.tune / XCB_TUNE_MM_LANES); results do not depend on it."""
        self._chk(self.L.xcb_mm_set_tuning(self._h, int(knob), int(value)), "mapmatch.set_tuning")

    def match_dev(self, kp, nkp, desc, uv, S, lm_desc, lm_ndesc, nlm, chi2=CHI2_2_999, out=None, stream=0):
        """F frames in device memory (torch CUDA tensors): kp (F,Nk,2) float32, nkp (F,) int32, desc (F,Nk,32) uint8,
        uv (F,Nl,2) float64, S (F,Nl,2,2) float64, lm_desc (F,Nl,D,32) uint8, lm_ndesc (F,Nl) int64, nlm (F,) int32.
        -> dict(kp, d, d2) of (F,Nl) device tensors (rows past nlm[f] not written); launches only, no sync."""
        import torch
        self._own()
        F, Nk = int(kp.shape[0]), int(kp.shape[1])
        Nl, D = int(lm_desc.shape[1]), int(lm_desc.shape[2])
        for t, dt in ((kp, torch.float32), (nkp, torch.int32), (desc, torch.uint8), (uv, torch.float64),
                      (S, torch.float64), (lm_desc, torch.uint8), (lm_ndesc, torch.int64), (nlm, torch.int32)):
            if t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError("mapmatch.match_dev: expected contiguous CUDA tensors of the documented dtypes")
        if out is None:
            out = dict(kp=torch.empty((F, Nl), dtype=torch.int64, device=kp.device),
                       d=torch.empty((F, Nl), dtype=torch.int64, device=kp.device),
                       d2=torch.empty((F, Nl), dtype=torch.float64, device=kp.device))
        v = lambda t: ctypes.c_void_p(t.data_ptr())
        self._chk(self.L.xcb_mm_match_dev(self._h, F, v(kp), v(nkp), Nk, v(desc), v(uv), v(S), v(lm_desc), D,
                                          v(lm_ndesc), v(nlm), Nl, float(chi2), v(out["kp"]), v(out["d"]),
                                          v(out["d2"]), ctypes.c_void_p(int(stream) or None)), "mapmatch.match_dev")
        return out


def _pred_inputs(Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, L):
    f = lambda a, shape: np.ascontiguousarray(a, np.float64).reshape(shape)
    return [f(Rwb_t, (3, 3)), f(pwb_t, (3,)), f(Rbc, (3, 3)), f(pbc, (3,)), f(Rwc_h, (L, 3, 3)), f(pwc_h, (L, 3)),
            f(lmp, (L, 3)), f(Spose, (6, 6)), f(Sl, (L, 3, 3))]


_tls = threading.local()


def _pred_handle():
    h = getattr(_tls, "mm", None)
    if h is None:
        h = _tls.mm = MapMatcher(16, 16, max_kp=1, max_lm=1)
    return h


def predict_projection(Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, sig_px, fx, fy, cx, cy, W, H, uv, S, ok,
                       depth):
    """window.predict_projection on the device: ok (L,) for every landmark, uv (L,2) / depth (L,) where the point is
    in front, S (L,2,2) where it also projects inside W x H, written into the caller's arrays (float64 / bool,
    C-contiguous) exactly where the reference writes them; bit-identical values.  Returns 0."""
    lmp = np.ascontiguousarray(lmp, np.float64).reshape(-1, 3)
    L = len(lmp)
    for a, dt, shape in ((uv, np.float64, (L, 2)), (S, np.float64, (L, 2, 2)), (ok, np.bool_, (L,)),
                         (depth, np.float64, (L,))):
        if not (isinstance(a, np.ndarray) and a.dtype == dt and a.flags.c_contiguous and a.shape == shape):
            raise ValueError("predict_projection: outputs must be C-contiguous arrays of the reference's shapes")
    if L == 0:
        return 0
    mm = _pred_handle()
    ins = _pred_inputs(Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, L)
    p = _lib.ptr
    mm._chk(mm.L.xcb_mm_predict_host(mm._h, *[p(a) for a in ins], float(sig_px), float(fx), float(fy), float(cx),
                                     float(cy), float(W), float(H), L, p(uv), p(S), p(ok.view(np.uint8)), p(depth),
                                     None), "predict_projection")
    return 0


def warmup():
    """Build the handle and run one tiny match (the reference's warmup compiles its numba kernels)."""
    mm = MapMatcher(64, 64)
    mm.match(np.array([[10.0, 10.0], [20.0, 20.0]]), np.zeros((2, 32), np.uint8), np.array([[10.0, 10.0]]),
             np.eye(2)[None] * 4.0, np.zeros((1, 3, 32), np.uint8), np.array([1]))
    mm.close()
