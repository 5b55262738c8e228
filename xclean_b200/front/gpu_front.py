"""B200 frontend: the drop-in for xclean.front.gpu_front (src/xclean/front/gpu_front.py).

Same API as the reference module (the engine swaps it by import, nothing else changes):

    det = Detector(rig)                          # front/detect.Detector budget logic; __call__ on the device
    kp, desc = det(gray)                         # (N,2) float32, (N,32) uint8, bit-identical to the CPU Detector
    d, sig, ok, zn = disparities(left, right, kp, dlo=None, dhi=None, dy=0.0, band=0)   # = front/stereo1d
    d, sig, ok, amb, span, zn = disparities_ex(...);  disparities.last_dy / last_amb / last_span
    i0, i1 = det.fe.match_desc(f0, f1)           # = Frontend.match_desc (stage A)
    warmup(rig)                                  # build the front, calibrate + self-check against cv2 / numpy

Under it, every call goes through the C ABI of libxcb200.so (include/xcb200.h) by ctypes; there is no CPU or
library fallback (a missing library or device raises).  Start-up self-check policy as the reference's
(gpu_front.py:17-25): a failed check raises RuntimeError; only the 3x3 solver check (a different LAPACK build) is
recorded and reported without refusing, unless XCLEAN_STRICT_SELFCHECK=1.

New on this path (no reference counterpart): GpuFront.detect_batch / pipeline for many frames per launch sequence,
the patch half-size `half` of the stereo (3, 4 or 5 = the reference's 11x11), and a calibration cache.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import threading

import numpy as np

from .. import _lib
from .detect import Detector as _BaseDetector
from .features import (HALF, HAMMING_CHANCE, KLT_WIN, LR_THRESHOLD_PX, MAX_DISP, ORB_PAD, ORB_PATCH, RATIO,
                       UNIQUENESS, ZNCC_MIN, Frontend, noise_floor_host, noise_q99)

POOL_LIMIT_BYTES = 1 << 30
STEREO_CAP = 4096          # kept for API compatibility: the device stereo takes any number of points per call
LM_CAP = 16384             # landmark descriptors per Hamming call (as the reference)

CONTEXT_KEPT_NOTE = ("Its CUDA context stays open for the rest of the run (its device memory was freed): closing it "
                     "while other libraries still hold handles in this process could crash the program later.")


def strict_selfcheck():
    """XCLEAN_STRICT_SELFCHECK=1: every failed start-up self-check raises."""
    return (os.environ.get("XCLEAN_STRICT_SELFCHECK") or "").strip() not in ("", "0")


def _cache_dir():
    d = os.environ.get("XCB200_CACHE_DIR") or os.path.join(os.path.expanduser("~"), ".cache", "xclean_b200")
    os.makedirs(d, exist_ok=True)
    return d


def _cv2_build_key():
    import cv2
    info = cv2.getBuildInformation()
    return hashlib.sha1((cv2.__version__ + info).encode()).hexdigest()[:16]


# ================================================================================== ORB pattern (probed from cv2)
_PATTERN = None


def _orb():
    import cv2
    return cv2.ORB_create(nfeatures=100000, scaleFactor=1.2, nlevels=1, edgeThreshold=ORB_PATCH, firstLevel=0,
                          WTA_K=2, patchSize=ORB_PATCH)


def cpu_orb(gray, kp):
    """Frontend.describe on the CPU with cv2 (reflect-101 pad, one KeyPoint per point, class_id map)."""
    import cv2
    pad = cv2.copyMakeBorder(gray, ORB_PAD, ORB_PAD, ORB_PAD, ORB_PAD, cv2.BORDER_REFLECT_101)
    kps = [cv2.KeyPoint(float(x) + ORB_PAD, float(y) + ORB_PAD, ORB_PATCH, 0.0, 0.0, 0, int(i))
           for i, (x, y) in enumerate(kp)]
    out_k, desc = _orb().compute(pad, kps)
    res = np.zeros((len(kp), 32), np.uint8)
    if desc is not None and len(out_k):
        cid = np.array([k.class_id for k in out_k], np.int64)
        res[cid] = desc
    return res


def probe_orb_pattern():
    """The 256 (x1, y1, x2, y2) test pairs of the cv2 ORB we call, recovered from its own outputs.

    Keypoints at the centres of a random-texture canvas; the blurred canvas is OpenCV's (sepFilter2D with ORB's
    Gaussian taps).  For each descriptor bit, every ordered pair of patch offsets is a candidate; a keypoint's bit
    keeps the candidates whose blurred comparison agrees with it.  With enough keypoints one pair remains.  The
    result is cached per cv2 build.  -> int array (256, 4)."""
    global _PATTERN
    if _PATTERN is not None:
        return _PATTERN.copy()
    import cv2
    path = os.path.join(_cache_dir(), "orb_pattern_%s.npy" % _cv2_build_key())
    if os.path.exists(path):
        pat = np.load(path)
        if pat.shape == (256, 4):
            _PATTERN = pat.astype(np.int64)
            return _PATTERN.copy()
    R, T, K, M = 15, 48, 160, 64
    side = int(np.ceil(np.sqrt(K)))
    rng = np.random.default_rng(20261203)
    canvas = (rng.random((2 * M + side * T, 2 * M + side * T)) * 255).astype(np.uint8)
    kps, cen = [], []
    for i in range(K):
        r_, c_ = divmod(i, side)
        y, x = M + r_ * T + T // 2, M + c_ * T + T // 2
        kps.append(cv2.KeyPoint(float(x), float(y), ORB_PATCH, 0.0, 0.0, 0, i))
        cen.append((x, y))
    out_k, desc = _orb().compute(canvas, kps)
    cid = np.array([k.class_id for k in out_k])
    if len(cid) != K:
        raise RuntimeError("probe_orb_pattern: cv2 dropped probe keypoints")
    D = np.zeros((K, 32), np.uint8)
    D[cid] = desc
    bits = np.unpackbits(D, axis=1, bitorder="little").astype(bool)
    kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
    B = cv2.sepFilter2D(canvas, -1, kf, kf, borderType=cv2.BORDER_REFLECT_101)
    offs = np.array([(dx, dy) for dy in range(-R, R + 1) for dx in range(-R, R + 1)])
    V = np.stack([B[y + offs[:, 1], x + offs[:, 0]] for (x, y) in cen]).astype(np.int16)
    lt0 = V[0][:, None] < V[0][None, :]
    pat = np.zeros((256, 4), np.int64)
    for b in range(256):
        ia, ib = np.nonzero(lt0 == bits[0, b])
        keep = ia != ib
        ia, ib = ia[keep], ib[keep]
        for k in range(1, K):
            m = (V[k, ia] < V[k, ib]) == bits[k, b]
            ia, ib = ia[m], ib[m]
            if len(ia) <= 1:
                break
        if len(ia) != 1:
            raise RuntimeError("probe_orb_pattern: bit %d is not determined by the probe (%d candidates)" % (b, len(ia)))
        pat[b] = (*offs[ia[0]], *offs[ib[0]])
    np.save(path + ".%d.npy" % os.getpid(), pat)
    os.replace(path + ".%d.npy" % os.getpid(), path)
    _PATTERN = pat
    return pat.copy()


def _nb_solve_inv():
    """numba's np.linalg.solve / inv (the calls stereo1d._lk_v makes) for the solver self-check."""
    from numba import njit

    @njit(cache=False)
    def f(As, gs, X, Inv):
        for k in range(As.shape[0]):
            A = As[k].copy()
            X[k] = np.linalg.solve(A, gs[k].copy())
            Inv[k] = np.linalg.inv(As[k].copy())
    return f


def warn_lk_mismatch(k, n):
    import sys
    print("xclean_b200: note: the device 3x3 solver does not match this machine's CPU LAPACK bit for bit (%d of %d "
          "test systems differ at rounding level). The device front end stays on; results can differ from a CPU-only "
          "run in the last digits." % (k, n), file=sys.stderr, flush=True)


def lk_test_systems(rng, n=1024):
    """LK-shaped 3x3 systems: J^T J + 1e-9 I with J = (-a gx, I, 1), a fifth with a zero gradient column, a fifth
    with a flat patch (gpu_front.check_lk_solver's construction)."""
    As = np.empty((n, 3, 3))
    gs = rng.normal(0.0, 1.0, (n, 3)) * (10.0 ** rng.uniform(-6, 4, (n, 1)))
    for k in range(n):
        J0 = -rng.uniform(0.4, 2.2) * rng.normal(0.0, 10.0 ** rng.uniform(-2, 2.5), 121)
        J1 = np.clip(rng.uniform(0, 255) + rng.normal(0.0, 10.0 ** rng.uniform(-1, 1.8), 121), 0, 255)
        if k % 5 == 1:
            J0[:] = 0.0
        elif k % 5 == 2:
            J1[:] = round(J1[0])
        J = np.stack([J0, J1, np.ones(121)], axis=1)
        As[k] = J.T @ J + 1e-9 * np.eye(3)
    return As, gs


# ======================================================================================================== GpuFront
class GpuFront:
    """Device-resident frontend for one image size; every device buffer is allocated here, once.

    max_frames > 1 sizes the batched path (detect_batch / pipeline) for that many frames per call."""

    def __init__(self, W, H, cap=2048, verbose=False, max_frames=1):
        self.W, self.H, self.cap = int(W), int(H), int(cap)
        self.Hp, self.Wp = self.H + 2 * ORB_PAD, self.W + 2 * ORB_PAD
        self.max_frames = int(max_frames)
        self.L = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(self.L.xcb_front_create(self.W, self.H, self.cap, self.max_frames, ctypes.byref(h)), None,
                   "xcb_front_create")
        self._h = h
        self.calibrated = False
        self.calib = {}
        self.pattern = None
        self.last = {}
        self.verbose = verbose
        self._owner = threading.get_ident()
        self._desc_ref = None
        self._desc_n = 0
        self.n_ham_fallback = 0
        self.h_ham_b = np.empty(max(self.cap, 4096) * 32, np.uint8)      # capacity marker, as the reference's

    # -------------------------------------------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self.L.xcb_front_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _own(self):
        if threading.get_ident() != self._owner:
            raise RuntimeError("gpu_front: called from a second thread (the GpuFront buffers are single-owner)")

    def _chk(self, rc, what):
        _lib.check(rc, self._h, what)

    def pool_bytes(self):
        return int(self.L.xcb_front_device_bytes(self._h))

    # -------------------------------------------------------------------------------------------------- probes
    def response(self, gray, dy_vend=None, dx_vend=None):
        g = np.ascontiguousarray(gray, np.uint8)
        R = np.empty((self.H, self.W), np.float32)
        dyv = self.calib.get("dy_vend", (self.W // 32) * 32) if dy_vend is None else dy_vend
        dxv = self.calib.get("dx_vend", self.W) if dx_vend is None else dx_vend
        self._chk(self.L.xcb_front_response_host(self._h, _lib.ptr(g), int(dyv), int(dxv), _lib.ptr(R)), "response")
        return R

    def noise_floor(self, gray):
        g = np.ascontiguousarray(gray, np.uint8)
        out = np.zeros(1)
        self._chk(self.L.xcb_front_noise_floor_host(self._h, _lib.ptr(g), _lib.ptr(out)), "noise_floor")
        return float(out[0])

    def blur(self, gray, vr=None, vc=None):
        g = np.ascontiguousarray(gray, np.uint8)
        out = np.empty((self.Hp, self.Wp), np.uint8)
        vr = self.calib["blur_vr"] if vr is None else vr
        vc = self.calib["blur_vc"] if vc is None else vc
        self._chk(self.L.xcb_front_blur_host(self._h, _lib.ptr(g), int(vr), int(vc), _lib.ptr(out)), "blur")
        return out

    # -------------------------------------------------------------------------------------------------- calibration
    def set_calibration(self, calib, pattern):
        """Apply a calibration (dict with dy_vend, dx_vend, blur_vr, blur_vc, kf, q99) and the ORB pattern."""
        kf = np.ascontiguousarray(calib["kf"], np.float32).ravel()
        pat = np.ascontiguousarray(np.asarray(pattern).reshape(256, 4), np.int8)
        self._chk(self.L.xcb_front_set_calibration(self._h, int(calib["dy_vend"]), int(calib["dx_vend"]),
                                                   int(calib["blur_vr"]), int(calib["blur_vc"]), _lib.ptr(kf),
                                                   _lib.ptr(pat), float(calib["q99"])), "set_calibration")
        self.calib = dict(calib)
        self.calib["kf"] = [float(x) for x in kf]
        self.pattern = np.asarray(pattern).reshape(256, 4).astype(np.int64)
        self.calibrated = True

    def calibrate(self, seed=0, cache=True):
        """Find OpenCV's SIMD / scalar split points for this image size and verify every bit-exact claim against cv2 /
        numpy on random data (gpu_front.GpuFront.calibrate).  Raises RuntimeError if a check fails."""
        import cv2
        W, H = self.W, self.H
        key = "calib_%dx%d_%s.json" % (W, H, _cv2_build_key())
        path = os.path.join(_cache_dir(), key)
        pat = probe_orb_pattern()
        q99 = noise_q99()
        kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
        rng = np.random.default_rng(seed)
        img = (rng.random((H, W)) * 255).astype(np.uint8)
        img = cv2.GaussianBlur(img, (0, 0), 1.0)
        img[: H // 8, : W // 8] = 77
        if cache and os.path.exists(path):
            with open(path) as fh:
                c = json.load(fh)
            self.set_calibration(c, pat)
            if np.array_equal(self.response(img).view(np.uint32), cv2.cornerMinEigenVal(img, 3, 3).view(np.uint32)):
                self.calib["lk_solver_equal"] = c.get("lk_solver_equal")
                self.calib["cached"] = True
                return self.calib
        R_cv = cv2.cornerMinEigenVal(img, 3, 3)
        cands = sorted(set([W] + [(W // m) * m for m in (4, 8, 16, 32, 64, 128)] + [0]), reverse=True)
        found = None
        for dxv in (W,) + tuple(c for c in cands if c != W):
            for dyv in cands:
                if np.array_equal(self.response(img, dyv, dxv).view(np.uint32), R_cv.view(np.uint32)):
                    found = (dyv, dxv)
                    break
            if found:
                break
        if not found:
            raise RuntimeError("gpu_front: no SIMD-boundary model reproduces cv2.cornerMinEigenVal on this build")
        pad = cv2.copyMakeBorder(img, ORB_PAD, ORB_PAD, ORB_PAD, ORB_PAD, cv2.BORDER_REFLECT_101)
        B_cv = cv2.sepFilter2D(pad, -1, kf, kf, borderType=cv2.BORDER_REFLECT_101)
        Wp = self.Wp
        bc = sorted(set([Wp] + [(Wp // m) * m for m in (4, 8, 16, 32, 64, 128)] + [0]), reverse=True)
        c0 = {"dy_vend": found[0], "dx_vend": found[1], "blur_vr": Wp, "blur_vc": Wp, "kf": kf, "q99": q99}
        self.set_calibration(c0, pat)
        foundb = None
        for vr in bc:
            for vc in bc:
                if np.array_equal(self.blur(img, vr, vc), B_cv):
                    foundb = (vr, vc)
                    break
            if foundb:
                break
        if not foundb:
            raise RuntimeError("gpu_front: no SIMD-boundary model reproduces cv2.sepFilter2D (ORB blur)")
        c0.update(blur_vr=foundb[0], blur_vc=foundb[1])
        self.set_calibration(c0, pat)
        fl = self.noise_floor(img)
        ref = noise_floor_host(img)
        if fl != ref:
            raise RuntimeError("gpu_front: pairwise noise sum differs from numpy (%r vs %r)" % (fl, ref))
        nk = min(self.cap, 1500)
        kx = rng.uniform(11, W - 12, nk).astype(np.float32)
        ky = rng.uniform(11, H - 12, nk).astype(np.float32)
        kx[:50] = np.floor(kx[:50]) + np.float32(0.5)
        ky[50:100] = np.floor(ky[50:100]) + np.float32(0.5)
        kpr = np.stack([kx, ky], axis=1)
        dref = cpu_orb(img, kpr)
        dg = self.describe_points(img, kpr)
        if not np.array_equal(dg, dref):
            raise RuntimeError("gpu_front: ORB descriptors differ from cv2 (%d bits)" % int(np.unpackbits(dg ^ dref).sum()))
        self.calib.update(response_vend={"dy_row": found[0], "dx_col": found[1], "W": W},
                          blur_vend={"row": foundb[0], "col": foundb[1], "Wp": Wp}, noise_floor_equal=True,
                          orb_equal_random=nk)
        self.calib["lk_solver_equal"] = self.check_lk_solver(rng)
        if cache:
            out = {k: self.calib[k] for k in ("dy_vend", "dx_vend", "blur_vr", "blur_vc", "q99", "lk_solver_equal")}
            out["kf"] = [float(x) for x in kf]
            tmp = path + ".%d" % os.getpid()
            with open(tmp, "w") as fh:
                json.dump(out, fh)
            os.replace(tmp, path)
        return self.calib

    def lk_solve_inv(self, As, gs):
        """The device 3x3 solve + inverse (the LK's arithmetic) of n systems."""
        As = np.ascontiguousarray(As, np.float64).reshape(-1, 3, 3)
        gs = np.ascontiguousarray(gs, np.float64).reshape(-1, 3)
        n = len(As)
        X = np.empty((n, 3))
        Inv = np.empty((n, 3, 3))
        self._chk(self.L.xcb_front_lk_check_host(self._h, _lib.ptr(As), _lib.ptr(gs), n, _lib.ptr(X), _lib.ptr(Inv)),
                  "lk_check")
        return X, Inv

    def check_lk_solver(self, rng, n=1024):
        """The device 3x3 solve / inverse vs numba's np.linalg.solve / inv.  -> n when bit for bit; False with the
        mismatch count recorded (RuntimeError under XCLEAN_STRICT_SELFCHECK=1); None when numba is absent."""
        try:
            nb = _nb_solve_inv()
        except Exception:
            return None
        As, gs = lk_test_systems(rng, n)
        Xr = np.empty((n, 3))
        Ir = np.empty((n, 3, 3))
        nb(As, gs, Xr, Ir)
        Xg, Ig = self.lk_solve_inv(As, gs)
        if not (np.array_equal(Xg.view(np.uint64), Xr.view(np.uint64))
                and np.array_equal(Ig.view(np.uint64), Ir.view(np.uint64))):
            k = int((~(Xg == Xr).all(1) | ~(Ig == Ir).all((1, 2))).sum())
            if strict_selfcheck():
                raise RuntimeError("gpu_front: the device 3x3 solve/inverse differs from numba's LAPACK on %d of %d "
                                   "systems" % (k, n))
            self.calib["lk_solver_mismatch"] = k
            self.calib["lk_solver_systems"] = int(n)
            warn_lk_mismatch(k, n)
            return False
        return n

    # -------------------------------------------------------------------------------------------------- detection
    def _require(self):
        if not self.calibrated:
            raise RuntimeError("gpu_front: the front is not calibrated (calibrate() or set_calibration())")

    def detect_batch(self, grays, budget):
        """Detection + ORB for F frames of one budget.  -> (counts [F], kp [F,cap,2], desc [F,cap,32], floor [F],
        anypos [F])."""
        self._own()
        self._require()
        g = np.ascontiguousarray(grays, np.uint8).reshape(-1, self.H, self.W)
        F = len(g)
        if F > self.max_frames:
            raise ValueError("detect_batch: %d frames > max_frames %d" % (F, self.max_frames))
        if int(budget) > self.cap:
            raise ValueError("detect: budget %d > cap %d" % (budget, self.cap))
        counts = np.zeros(F, np.int32)
        kp = np.zeros((F, self.cap, 2), np.float32)
        desc = np.zeros((F, self.cap, 32), np.uint8)
        floor = np.zeros(F)
        anypos = np.zeros(F, np.int32)
        self._chk(self.L.xcb_front_detect_host(self._h, _lib.ptr(g), F, int(budget), _lib.ptr(counts), _lib.ptr(kp),
                                               _lib.ptr(desc), _lib.ptr(floor), _lib.ptr(anypos)), "detect")
        return counts, kp, desc, floor, anypos

    def detect(self, gray, budget, fe):
        """Detector.__call__ (cell scope, budget n): -> (kp (N,2) float32, desc (N,32) uint8)."""
        counts, kp, desc, floor, anypos = self.detect_batch(np.asarray(gray)[None], budget)
        cnt = int(counts[0])
        kpo = kp[0, :cnt].copy()
        do = desc[0, :cnt].copy()
        if anypos[0]:
            fe.stats["noise_floor_last"] = float(floor[0])
        self._desc_ref = do
        self._desc_n = cnt
        self.last = {"n": int(budget), "count": cnt, "floor": float(floor[0])}
        return kpo, do

    def describe_points(self, gray, kp):
        """ORB descriptors of given keypoints (test / calibration path)."""
        self._own()
        g = np.ascontiguousarray(gray, np.uint8)
        kp = np.ascontiguousarray(kp, np.float32).reshape(-1, 2)
        n = len(kp)
        out = np.zeros((n, 32), np.uint8)
        self._desc_ref = None
        for a in range(0, n, self.cap):
            e = min(n, a + self.cap)
            blk = np.ascontiguousarray(kp[a:e])
            o = np.zeros((e - a, 32), np.uint8)
            self._chk(self.L.xcb_front_describe_host(self._h, _lib.ptr(g), _lib.ptr(blk), e - a, _lib.ptr(o)),
                      "describe")
            out[a:e] = o
        return out

    # -------------------------------------------------------------------------------------------------- stereo
    def stereo(self, left, right, kp, lo, hi, dy=0.0, band=0, half=HALF):
        """stereo1d.stereo_points_band on the device -> (d, sig, ok, zn, ody) host float64 / bool arrays."""
        self._own()
        kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 2)
        N = len(kp)
        d = np.zeros(N)
        sg = np.full(N, np.inf)
        ok = np.zeros(N, np.uint8)
        zn = np.zeros(N)
        ody = np.full(N, np.nan)
        if N == 0:
            return d, sg, ok.astype(bool), zn, ody
        L = np.ascontiguousarray(left, np.uint8)
        R = np.ascontiguousarray(right, np.uint8)
        lo = np.ascontiguousarray(lo, np.int64)
        hi = np.ascontiguousarray(hi, np.int64)
        self._chk(self.L.xcb_front_stereo_host(self._h, _lib.ptr(L), _lib.ptr(R), _lib.ptr(kp), _lib.ptr(lo),
                                               _lib.ptr(hi), N, float(dy), int(band), int(half), _lib.ptr(d),
                                               _lib.ptr(sg), _lib.ptr(ok), _lib.ptr(zn), _lib.ptr(ody)), "stereo")
        return d, sg, ok.astype(bool), zn, ody

    # -------------------------------------------------------------------------------------------------- hamming
    def hamming(self, A, B):
        """Row best / second / index (first minimum) of A (L,32) against B (N,32), and the column best index."""
        self._own()
        A = np.ascontiguousarray(A, np.uint8).reshape(-1, 32)
        B = np.ascontiguousarray(B, np.uint8).reshape(-1, 32)
        L, N = len(A), len(B)
        if L > LM_CAP:
            raise ValueError("hamming: %d landmark descriptors > LM_CAP %d" % (L, LM_CAP))
        if N > self.h_ham_b.size // 32:
            raise ValueError("hamming: %d keypoint descriptors > capacity" % N)
        b1 = np.zeros(L, np.int32)
        b2 = np.zeros(L, np.int32)
        bi = np.zeros(L, np.int32)
        ci = np.zeros(N, np.int32)
        self._chk(self.L.xcb_front_hamming_host(self._h, _lib.ptr(A), L, _lib.ptr(B), N, _lib.ptr(b1), _lib.ptr(b2),
                                                _lib.ptr(bi), _lib.ptr(ci)), "hamming")
        return b1.astype(np.int64), b2.astype(np.int64), bi.astype(np.int64), ci.astype(np.int64)

    def match(self, A, B, ham_max=HAMMING_CHANCE, ratio=RATIO):
        """Mutual NN + ratio + chance bound with the epilogue on the device -> (q, t) int64 in query order."""
        self._own()
        A = np.ascontiguousarray(A, np.uint8).reshape(-1, 32)
        B = np.ascontiguousarray(B, np.uint8).reshape(-1, 32)
        L, N = len(A), len(B)
        i0 = np.zeros(max(L, 1), np.int64)
        i1 = np.zeros(max(L, 1), np.int64)
        nm = np.zeros(1, np.int32)
        self._chk(self.L.xcb_front_match_host(self._h, _lib.ptr(A), L, _lib.ptr(B), N, int(ham_max), float(ratio),
                                              _lib.ptr(i0), _lib.ptr(i1), _lib.ptr(nm)), "match")
        m = int(nm[0])
        return i0[:m].copy(), i1[:m].copy()

    # -------------------------------------------------------------------------------------------------- pipeline
    def pipeline_dev(self, left_ptr, right_ptr, nframes, budget, half=HALF, dlo=0, dhi=MAX_DISP - 1, match_prev=True,
                     stream=0):
        """The batched per-frame path on device memory (graph-replayed); results stay in device_buffers()."""
        self._require()
        self._chk(self.L.xcb_front_pipeline_dev(self._h, ctypes.c_void_p(int(left_ptr)), ctypes.c_void_p(int(right_ptr)),
                                                int(nframes), int(budget), int(half), int(dlo), int(dhi),
                                                int(bool(match_prev)), ctypes.c_void_p(int(stream) or None)),
                  "pipeline")

    def sync_check(self, stream=0):
        self._chk(self.L.xcb_front_sync_check(self._h, ctypes.c_void_p(int(stream) or None)), "pipeline")

    def device_buffers(self):
        b = _lib.FrontBufs()
        self._chk(self.L.xcb_front_buffers(self._h, ctypes.byref(b)), "buffers")
        return {n: int(getattr(b, n) or 0) for n, _ in _lib.FrontBufs._fields_}

    def set_tuning(self, knob, value):
        """A launch-shape knob (xclean_b200.tune / XCB_TUNE_STEREO_*); results do not depend on it."""
        self._chk(self.L.xcb_front_set_tuning(self._h, int(knob), int(value)), "set_tuning")

    def last_launches(self):
        return int(self.L.xcb_front_last_launches(self._h))

    def set_stage_timing(self, on):
        """Record device events at the stage boundaries of every (re)captured pipeline graph."""
        self._chk(self.L.xcb_front_set_stage_timing(self._h, int(bool(on))), "stage timing")

    def stage_times(self):
        """-> ({stage: ms summed over the graphs replayed since the last read}, number of graphs); sync first."""
        ms = np.zeros(len(_lib.FRONT_STAGES), np.float32)
        n = ctypes.c_int(0)
        self._chk(self.L.xcb_front_stage_times(self._h, _lib.ptr(ms), ctypes.byref(n)), "stage times")
        return dict(zip(_lib.FRONT_STAGES, (float(x) for x in ms))), int(n.value)

    def pipeline(self, left, right, budget, half=HALF, dlo=0, dhi=MAX_DISP - 1, match_prev=True, out=None, stream=0):
        """The batched per-frame path from host arrays: left/right [F,H,W] -> dict of host arrays (frame-major)."""
        self._own()
        self._require()
        Lh = np.ascontiguousarray(left, np.uint8).reshape(-1, self.H, self.W)
        Rh = np.ascontiguousarray(right, np.uint8).reshape(-1, self.H, self.W)
        F, cap = len(Lh), self.cap
        if out is None:
            out = self.alloc_outputs(F)
        b = _lib.FrontBufs()
        for n, _ in _lib.FrontBufs._fields_:
            a = out.get(n)
            setattr(b, n, a.ctypes.data if a is not None else None)
        self._chk(self.L.xcb_front_pipeline_host(self._h, _lib.ptr(Lh), _lib.ptr(Rh), F, int(budget), int(half),
                                                 int(dlo), int(dhi), int(bool(match_prev)), ctypes.byref(b),
                                                 ctypes.c_void_p(int(stream) or None)), "pipeline")
        return out

    def pipeline_batches(self, left, right, budget, batch, half=HALF, dlo=0, dhi=MAX_DISP - 1, match_prev=True,
                         out=None, stream=0):
        """pipeline() over any number of frames in batches of `batch` (<= max_frames), one call: the next batch's
        frames are copied to the device while the current batch computes (page-locked `left` / `right` make the copy
        overlap).  Results as consecutive pipeline() calls on the batches, in one dict of host arrays."""
        self._own()
        self._require()
        Lh = np.ascontiguousarray(left, np.uint8).reshape(-1, self.H, self.W)
        Rh = np.ascontiguousarray(right, np.uint8).reshape(-1, self.H, self.W)
        F = len(Lh)
        if out is None:
            out = self.alloc_outputs(F)
        b = _lib.FrontBufs()
        for n, _ in _lib.FrontBufs._fields_:
            a = out.get(n)
            setattr(b, n, a.ctypes.data if a is not None else None)
        self._chk(self.L.xcb_front_pipeline_host_batches(self._h, _lib.ptr(Lh), _lib.ptr(Rh), F, int(batch),
                                                         int(budget), int(half), int(dlo), int(dhi),
                                                         int(bool(match_prev)), ctypes.byref(b),
                                                         ctypes.c_void_p(int(stream) or None)), "pipeline_batches")
        return out

    def alloc_outputs(self, F):
        cap = self.cap
        return dict(counts=np.zeros(F, np.int32), kp=np.zeros((F, cap, 2), np.float32),
                    desc=np.zeros((F, cap, 32), np.uint8), d=np.zeros((F, cap)), sig=np.zeros((F, cap)),
                    ok=np.zeros((F, cap), np.uint8), zn=np.zeros((F, cap)), dy=np.zeros((F, cap)),
                    m0=np.zeros((F, cap), np.int64), m1=np.zeros((F, cap), np.int64), nmatch=np.zeros(F, np.int32),
                    floor=np.zeros(F), anypos=np.zeros(F, np.int32))


# =============================================================================== start-up policy helpers
def cuda_context_active():
    """True when this process holds a CUDA context (asks the driver; creates none)."""
    try:
        lib = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    try:
        if lib.cuInit(0) != 0:
            return False
        cur = ctypes.c_void_p(0)
        if lib.cuCtxGetCurrent(ctypes.byref(cur)) == 0 and cur.value:
            return True
        n = ctypes.c_int(0)
        if lib.cuDeviceGetCount(ctypes.byref(n)) != 0:
            return False
        for i in range(n.value):
            dev = ctypes.c_int(0)
            flags, active = ctypes.c_uint(0), ctypes.c_int(0)
            if lib.cuDeviceGet(ctypes.byref(dev), i) == 0 and \
                    lib.cuDevicePrimaryCtxGetState(dev, ctypes.byref(flags), ctypes.byref(active)) == 0 and active.value:
                return True
    except Exception:
        return False
    return False


def release_device(cp=None, context_active=None):
    """Drop every front of this module (their device buffers are freed); an existing CUDA context is kept.
    cp / context_active: stand-ins for tests.  -> {"cuda_context_released", "gpu_memory_freed", "note", "errors"}."""
    import gc
    out = {"cuda_context_released": True, "gpu_memory_freed": None, "note": None, "errors": []}
    try:
        for f in list(_FRONT.values()):
            f.close()
        out["gpu_memory_freed"] = bool(_FRONT) or None
    except Exception as e:
        out["gpu_memory_freed"] = False
        out["errors"].append("freeing the device fronts: %s: %s" % (type(e).__name__, e))
    _FRONT.clear()
    gc.collect()
    if cp is not None:
        try:
            cp.get_default_memory_pool().free_all_blocks()
            cp.get_default_pinned_memory_pool().free_all_blocks()
            out["gpu_memory_freed"] = True
        except Exception as e:
            out["gpu_memory_freed"] = False
            out["errors"].append("freeing the memory pools: %s: %s" % (type(e).__name__, e))
    active = context_active or cuda_context_active
    try:
        held = bool(active())
    except Exception as e:
        held = True
        out["errors"].append("asking the driver for a CUDA context: %s: %s" % (type(e).__name__, e))
    if held:
        out["cuda_context_released"] = False
        out["note"] = CONTEXT_KEPT_NOTE
    return out


# ======================================================================================== engine-facing API
_FRONT = {}


def front_for(W, H, cap=2048):
    """The front for this image size (a larger cap replaces the cached one), calibrated."""
    key = (int(W), int(H))
    f = _FRONT.get(key)
    if f is None or f.cap < int(cap):
        f = GpuFront(W, H, max(int(cap), 2048 if f is None else f.cap))
        f.calibrate()
        _FRONT[key] = f
    return f


class Detector(_BaseDetector):
    """front/detect.Detector with the extraction on the device; fe.match_desc is the device Hamming (hamming=True)."""

    def __init__(self, rig, cap=2048, window=10, hamming=True):
        super().__init__(rig, cap=cap, window=window)
        self.gpu = front_for(rig.width, rig.height, max(cap, 2048))
        if hamming:
            self.fe.match_desc = self._match_desc

    def __call__(self, gray):
        n = self.budget
        kp, desc = self.gpu.detect(gray, n, self.fe)
        self.fe.stats["detected"] += int(len(kp))
        self.stats["frames"] += 1
        self.stats["detected"] += int(len(kp))
        return kp, desc

    def _match_desc(self, f0, f1, mask0=None, mask1=None):
        return match_desc_gpu(self.gpu, f0, f1, mask0, mask1)


def match_desc_gpu(gf, f0, f1, mask0=None, mask1=None):
    """Frontend.match_desc semantics (mutual NN + Lowe ratio + Hamming chance bound) with the device Hamming."""
    d0, d1 = f0["descriptors"], f1["descriptors"]
    i0 = np.arange(len(d0)) if mask0 is None else np.nonzero(mask0)[0]
    i1 = np.arange(len(d1)) if mask1 is None else np.nonzero(mask1)[0]
    z = np.zeros(0, np.int64)
    if len(i0) < 2 or len(i1) < 2:
        return z, z
    if len(i0) > LM_CAP or len(i1) > gf.h_ham_b.size // 32:
        raise ValueError("match_desc_gpu: %d x %d descriptors exceed the device matcher's capacity" % (len(i0), len(i1)))
    A = d0 if mask0 is None else np.ascontiguousarray(d0[i0])
    B = d1 if mask1 is None else np.ascontiguousarray(d1[i1])
    q, t = gf.match(np.ascontiguousarray(A), np.ascontiguousarray(B))
    if not len(q):
        return z, z
    return i0[q].astype(np.int64), i1[t].astype(np.int64)


def disparities(left, right, kp, dlo=None, dhi=None, dy=0.0, band=0, half=HALF):
    """front/stereo1d.disparities on the device (same signature, same outputs; sets last_dy / last_amb / last_span).
    `half` (new): the ZNCC patch half-size, 5 = the reference's 11x11."""
    kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 2)
    n = len(kp)
    lo = np.zeros(n, np.int64) if dlo is None else np.ascontiguousarray(dlo, np.int64)
    hi = np.full(n, MAX_DISP - 1, np.int64) if dhi is None else np.ascontiguousarray(dhi, np.int64)
    H, W = left.shape
    gf = _FRONT.get((int(W), int(H))) or front_for(W, H)
    bad = ~(np.isfinite(kp[:, 0]) & np.isfinite(kp[:, 1]) & (kp[:, 0] >= 0) & (kp[:, 0] < W) & (kp[:, 1] >= 0)
            & (kp[:, 1] < H))
    if bad.any():
        kp = kp.copy()
        kp[bad] = -float(half + 3)          # off the image: rejected by the kernel's own border test
    d, s, ok, zn, ody = gf.stereo(left, right, kp, lo, hi, float(dy), int(band), int(half))
    disparities.last_amb = np.zeros(n, np.bool_)
    disparities.last_span = np.zeros(n)
    disparities.last_dy = ody + float(dy)
    return d, s, ok, zn


def disparities_ex(left, right, kp, dlo=None, dhi=None, dy=0.0, band=0, half=HALF):
    """-> (d, sigma, ok, amb, span, zncc) as stereo1d.disparities_ex."""
    d, s, ok, zn = disparities(left, right, kp, dlo, dhi, dy, band, half)
    return d, s, ok, disparities.last_amb, disparities.last_span, zn


def warmup(rig):
    """Create the device front for the rig's size, calibrate + self-check, and run one detection, two stereo calls and
    one Hamming call on synthetic data.  -> calibration dict."""
    import cv2
    W, H = int(rig.width), int(rig.height)
    gf = front_for(W, H)
    rng = np.random.default_rng(0)
    img = cv2.GaussianBlur((rng.random((H, W)) * 255).astype(np.uint8), (0, 0), 1.0)
    fe = Frontend(rig, cap=2048)
    kp, desc = gf.detect(img, 1500, fe)
    disparities(img, np.roll(img, -8, axis=1), kp[:64].astype(np.float64))
    disparities(img, np.roll(img, -8, axis=1), kp[:64].astype(np.float64), dy=0.25, band=1)
    if len(desc) >= 2:
        match_desc_gpu(gf, {"descriptors": desc[::-1].copy()}, {"descriptors": desc})
    gf._desc_ref = None
    return dict(gf.calib, pool_bytes=gf.pool_bytes())
