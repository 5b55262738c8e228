"""Multi-scale, oriented ORB on B200: image pyramid, FAST-9 corners, orientation bins and steered rBRIEF
(libxcb200 xcb_orbx_* / xcb_fast_dev ..., csrc/front_ext.cu).

These go beyond the reference.  Its frontend is single-scale Shi-Tomasi with unoriented ORB
(src/xclean/stages/features.py:27-28, :102-103; src/xclean/front/gpu_front.py:1712-1717: cv2.ORB with nlevels=1 and
KeyPoint.angle 0).  The definitions follow OpenCV where OpenCV has one, bit for bit:

  FAST          cv2.FastFeatureDetector(threshold, nonmax, TYPE_9_16): keypoints and (with nonmax) scores
  pyramid       cv2.resize(INTER_LINEAR_EXACT) from the previous level, sizes rint(n / scale^l): cv2 ORB's pyramid
  descriptor    the reference's describe stage (cv2 ORB on the reflect-101 pad-32 image) at KeyPoint.angle = 12 k for
                orientation bin k; level 0 at bin 0 is the reference's own descriptor

Two parts are this package's own definitions.  Per level, the geometric share of `nfeatures` is kept: the best by FAST
score, ties in row-major order.  Orientation uses 30 bins of 12 degrees from the intensity centroid over a radius-15
disc.

    ox = OrbPyramid(1280, 720, levels=4, scale=1.2, nfeatures=4000)
    ox.calibrate()                         # ORB pattern, steered tables, per-level blur split points (needs cv2)
    f = ox.detect(gray_u8)                 # host arrays: kp (level-0 px), level, angle (deg), response, desc
    ox.detect_gpu(gray_cuda_u8)            # asynchronous, on the current stream; ox.read() for the slots

There is no CPU fallback: without libxcb200 or a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from collections import namedtuple

import numpy as np

from .. import _lib
from .gpu_front import _cache_dir, _cv2_build_key, probe_orb_pattern

BINS = 30
BIN_DEG = 12.0
PAD = 32
ORB_EDGE = 31                    # cv2 ORB's default edgeThreshold (= patchSize 31)

OrbFeatures = namedtuple("OrbFeatures", "kp level angle response desc")


def steered_patterns(pattern):
    """(256, 4) ORB test pairs (x1, y1, x2, y2) -> (30, 256, 4) int8, bin k rotated by 12 k degrees the way
    cv2.ORB.compute rotates a keypoint's tests: angle = float32(12 k) * float32(pi / 180); a, b = float32 cos, sin;
    x' = rint(x a - y b), y' = rint(x b + y a) in float32 (round half to even)."""
    p = np.asarray(pattern).reshape(256, 4).astype(np.float32)
    out = np.empty((BINS, 256, 4), np.int8)
    d2r = np.float32(math.pi / 180.0)
    for k in range(BINS):
        ang = np.float32(np.float32(12 * k) * d2r)
        a, b = np.float32(math.cos(float(ang))), np.float32(math.sin(float(ang)))
        for c in (0, 2):
            x, y = p[:, c], p[:, c + 1]
            out[k, :, c] = np.rint((x * a).astype(np.float32) - (y * b).astype(np.float32))
            out[k, :, c + 1] = np.rint((x * b).astype(np.float32) + (y * a).astype(np.float32))
    return out


def _blur_taps():
    import cv2
    return cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)


class OrbPyramid:
    """One image size; device buffers and a stream allocated once (xcb_orbx_create)."""

    def __init__(self, width, height, levels=4, scale=1.2, nfeatures=2000, fast_threshold=20, edge=ORB_EDGE,
                 nonmax=True, calibrate=True):
        self.L = _lib.lib()
        self.W, self.H = int(width), int(height)
        self.nlevels, self.scale, self.nfeatures = int(levels), float(scale), int(nfeatures)
        self.threshold, self.edge, self.nonmax = int(fast_threshold), int(edge), bool(nonmax)
        h = ctypes.c_void_p()
        rc = self.L.xcb_orbx_create(self.W, self.H, self.nlevels, self.scale, self.nfeatures, self.threshold,
                                    self.edge, 1 if self.nonmax else 0, ctypes.byref(h))
        _lib.check(rc, None, "xcb_orbx_create")
        self._h = h
        self.levels = []
        for lv in range(self.nlevels):
            w, hh, q, o = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            s = ctypes.c_float()
            self._chk(self.L.xcb_orbx_level(self._h, lv, ctypes.byref(w), ctypes.byref(hh), ctypes.byref(s),
                                            ctypes.byref(q), ctypes.byref(o)), "xcb_orbx_level")
            self.levels.append({"width": w.value, "height": hh.value, "scale": s.value, "quota": q.value,
                                "offset": o.value})
        self.calib = None
        if calibrate:
            self.calibrate()

    def close(self):
        if getattr(self, "_h", None):
            self.L.xcb_orbx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        if rc != _lib.XCB_OK:
            msg = (self.L.xcb_orbx_last_error(self._h) or b"").decode(errors="replace")
            if rc == _lib.XCB_ERR_CAPACITY:
                raise ValueError("%s: %s" % (what, msg))
            raise RuntimeError("%s failed (%d): %s" % (what, rc, msg))

    # ------------------------------------------------------------------------------------------------ calibration
    def set_calibration(self, blur, patterns, kf=None):
        """blur: [(vr, vc)] per level; patterns: (30, 256, 4) steered tables."""
        kf = np.ascontiguousarray(_blur_taps() if kf is None else kf, np.float32)
        for lv, (vr, vc) in enumerate(blur):
            self._chk(self.L.xcb_orbx_set_blur(self._h, lv, int(vr), int(vc), _lib.ptr(kf)), "xcb_orbx_set_blur")
        pats = np.ascontiguousarray(patterns, np.int8).reshape(BINS, 256, 4)
        self._chk(self.L.xcb_orbx_set_patterns(self._h, _lib.ptr(pats)), "xcb_orbx_set_patterns")
        self.calib = {"blur": [tuple(int(v) for v in b) for b in blur], "kf": kf, "patterns": pats}

    def calibrate(self, seed=0, cache=True):
        """The ORB pattern of this cv2 build, its steered tables, and per level the blur split points that make the
        device blur equal cv2.sepFilter2D of the pad-32 level image (GpuFront.calibrate's probe, per level size)."""
        pats = steered_patterns(probe_orb_pattern())
        kf = _blur_taps()
        blur = [blur_split_points(lvl["width"], lvl["height"], kf, seed=seed, cache=cache) for lvl in self.levels]
        self.set_calibration(blur, pats, kf)
        return self.calib

    # ---------------------------------------------------------------------------------------------------- detect
    def _slots(self):
        n = self.nfeatures
        return {"kp": np.zeros((n, 2), np.float32), "kp_level": np.zeros((n, 2), np.float32),
                "resp": np.zeros(n, np.float32), "level": np.zeros(n, np.int32), "bins": np.zeros(n, np.int32),
                "desc": np.zeros((n, 32), np.uint8), "counts": np.zeros(self.nlevels, np.int32)}

    def detect_slots(self, gray):
        """Host frame -> the slot arrays (level l's first counts[l] slots from its offset are valid)."""
        g = np.ascontiguousarray(gray, np.uint8).reshape(self.H, self.W)
        s = self._slots()
        p = _lib.ptr
        self._chk(self.L.xcb_orbx_detect_host(self._h, p(g), p(s["kp"]), p(s["kp_level"]), p(s["resp"]),
                                              p(s["level"]), p(s["bins"]), p(s["desc"]), p(s["counts"])),
                  "xcb_orbx_detect_host")
        return s

    def compact(self, s):
        idx = np.concatenate([np.arange(lvl["offset"], lvl["offset"] + int(c))
                              for lvl, c in zip(self.levels, s["counts"])]).astype(np.int64)
        return OrbFeatures(s["kp"][idx], s["level"][idx], s["bins"][idx].astype(np.float32) * np.float32(BIN_DEG),
                           s["resp"][idx], s["desc"][idx])

    def detect(self, gray):
        """Host frame -> OrbFeatures (kp in level-0 pixels, level, angle in degrees, FAST score, 32-byte desc)."""
        return self.compact(self.detect_slots(gray))

    def detect_gpu(self, gray, stream=None):
        """gray: torch CUDA uint8 (H, W), contiguous.  Enqueued on `stream` (default: torch's current stream)."""
        import torch
        if not (gray.is_cuda and gray.dtype == torch.uint8 and gray.is_contiguous()
                and tuple(gray.shape) == (self.H, self.W)):
            raise ValueError("OrbPyramid.detect_gpu: a contiguous CUDA uint8 (H, W) tensor")
        st = torch.cuda.current_stream(gray.device).cuda_stream if stream is None else int(stream)
        self._chk(self.L.xcb_orbx_detect_dev(self._h, ctypes.c_void_p(gray.data_ptr()), ctypes.c_void_p(st or None)),
                  "xcb_orbx_detect_dev")

    def read(self):
        """The slot arrays of the last detect (waits for the device)."""
        s = self._slots()
        p = _lib.ptr
        self._chk(self.L.xcb_orbx_read(self._h, p(s["kp"]), p(s["kp_level"]), p(s["resp"]), p(s["level"]),
                                       p(s["bins"]), p(s["desc"]), p(s["counts"])), "xcb_orbx_read")
        return s

    def level_image(self, lv):
        lvl = self.levels[lv]
        out = np.empty((lvl["height"], lvl["width"]), np.uint8)
        self._chk(self.L.xcb_orbx_read_level(self._h, int(lv), _lib.ptr(out)), "xcb_orbx_read_level")
        return out

    def launches(self):
        return int(self.L.xcb_orbx_launches(self._h))


def blur_split_points(width, height, kf=None, seed=0, cache=True):
    """(vr, vc) for which the device blur of a width x height image equals cv2.sepFilter2D of its reflect-101 pad-32
    copy with ORB's Gaussian taps (OpenCV's row / column filters switch between fused and unfused float arithmetic at
    these columns).  Probed on the device against cv2 on random data; cached per size and cv2 build."""
    import cv2
    import torch
    key = os.path.join(_cache_dir(), "orbx_blur_%dx%d_%s.json" % (width, height, _cv2_build_key()))
    if cache and os.path.exists(key):
        with open(key) as fh:
            c = json.load(fh)
        return int(c["vr"]), int(c["vc"])
    kf = np.ascontiguousarray(_blur_taps() if kf is None else kf, np.float32)
    rng = np.random.default_rng(seed)
    img = (rng.random((height, width)) * 255).astype(np.uint8)
    pad = cv2.copyMakeBorder(img, PAD, PAD, PAD, PAD, cv2.BORDER_REFLECT_101)
    want = cv2.sepFilter2D(pad, -1, kf, kf, borderType=cv2.BORDER_REFLECT_101)
    Wp = width + 2 * PAD
    cands = sorted(set([Wp] + [(Wp // m) * m for m in (4, 8, 16, 32, 64, 128)] + [0]), reverse=True)
    L = _lib.lib()
    dev = torch.device("cuda")
    g = torch.from_numpy(img).to(dev)
    k = torch.from_numpy(kf).to(dev)
    out = torch.empty((height + 2 * PAD, Wp), dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    found = None
    for vr in cands:
        for vc in cands:
            _lib.check(L.xcb_blur_dev(ctypes.c_void_p(g.data_ptr()), width, height, ctypes.c_void_p(k.data_ptr()),
                                      int(vr), int(vc), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st or None)),
                       None, "xcb_blur_dev")
            if np.array_equal(out.cpu().numpy(), want):
                found = (vr, vc)
                break
        if found:
            break
    if not found:
        raise RuntimeError("orb_ext: no split-point model reproduces cv2.sepFilter2D at %dx%d" % (width, height))
    if cache:
        tmp = key + ".%d" % os.getpid()
        with open(tmp, "w") as fh:
            json.dump({"vr": found[0], "vc": found[1]}, fh)
        os.replace(tmp, key)
    return found
