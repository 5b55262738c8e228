"""Dense 32-direction SGM on B200: the drop-in for xclean.stereo.sgm32 (src/xclean/stereo/sgm32.py).

    sgm = SGM32(width, height)
    disp, conf = sgm.compute(rect_left_u8, rect_right_u8)     # numpy float32, 0 = INVALID
    disp_t, conf_t = sgm.compute_gpu(left_t, right_t)         # torch CUDA uint8 in, float32 device tensors out

The algorithm and its outputs are the reference's (census 9x9 in two words, Hamming cost, one 32-direction
aggregation into an exact uint16 volume, left winner with 5 % uniqueness and parabola, right winner off the same
volume, left-right check, d < 0.5 px invalid); the kernels are libxcb200's (xcb_sgm_*, csrc/stereo_sgm.cu).  There
is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from .. import _lib

MAX_DISP = 128
CENSUS_HALF = 4
CENSUS_BITS = (2 * CENSUS_HALF + 1) ** 2 - 1        # 80
PROTOTYPE_EFFECTIVE_BITS = 63
PROTOTYPE_P1, PROTOTYPE_P2 = 10, 120
P1 = int(round(PROTOTYPE_P1 * CENSUS_BITS / PROTOTYPE_EFFECTIVE_BITS))     # 13
P2 = int(round(PROTOTYPE_P2 * CENSUS_BITS / PROTOTYPE_EFFECTIVE_BITS))     # 152
UNIQUENESS = 0.05
LR_THRESHOLD_PX = 1.0
MIN_DISP_PX = 0.5
FAMILIES = (((1, 1), (1, 1)), ((1, 2), (9, 4)), ((2, 1), (9, 4)), ((1, 3), (19, 6)), ((3, 1), (19, 6)),
            ((2, 3), (18, 5)), ((3, 2), (18, 5)))


def directions():
    """[(dx, dy, num, den)]: the 4 axis paths, then every sign combination of the 7 oblique families (sgm32.py:84-93)."""
    out = [(1, 0, 1, 1), (-1, 0, 1, 1), (0, 1, 1, 1), (0, -1, 1, 1)]
    for (ax, ay), (n, d) in FAMILIES:
        for sx in (1, -1):
            for sy in (1, -1):
                out.append((sx * ax, sy * ay, n, d))
    return out


def path_starts(H, W, dx, dy):
    """The pixels whose predecessor p - (dx, dy) lies outside the image (sgm32.py:96-102): (n, 2) int32 (x, y)."""
    ys, xs = np.mgrid[0:H, 0:W]
    m = (xs - dx < 0) | (xs - dx >= W) | (ys - dy < 0) | (ys - dy >= H)
    return np.stack([xs[m], ys[m]], axis=1).astype(np.int32)


class SGM32:
    """Dense SGM on rectified uint8 pairs of one fixed size (width <= 2048); device volumes allocated once."""

    NAME = "sgm32"

    def __init__(self, width, height, p1=P1, p2=P2, uniqueness=UNIQUENESS, lr_threshold=LR_THRESHOLD_PX,
                 verbose=False):
        self.W, self.H = int(width), int(height)
        self.p1, self.p2 = int(p1), int(p2)
        self.uniq = float(uniqueness)
        self.lr_thr = float(lr_threshold)
        p2s = [self.p2 * n // d for (_x, _y, n, d) in directions()]
        self.s_bound = 32 * (CENSUS_BITS + max(p2s))
        if self.s_bound >= 65536:
            raise ValueError("uint16 aggregation not exact: bound %d" % self.s_bound)
        self.L = _lib.lib()
        h = ctypes.c_void_p()
        rc = self.L.xcb_sgm_create(self.W, self.H, self.p1, self.p2, ctypes.c_float(self.uniq),
                                   ctypes.c_float(self.lr_thr), ctypes.c_float(MIN_DISP_PX), ctypes.byref(h))
        _lib.check(rc, None, "xcb_sgm_create")
        self._h = h
        n = ctypes.c_int(0)
        self.L.xcb_sgm_buffers(self._h, None, None, ctypes.byref(n))
        self.npaths = int(n.value)
        self.n_aggregations = 0
        self.n_frames = 0
        self.ms = []
        if verbose:
            print(" [sgm32] %dx%d, 32 directions (%d paths), census 9x9 = %d bits, P1 %d P2 %d, uint16 aggregation "
                  "(bound %d), one aggregation per frame, no hole fill"
                  % (self.W, self.H, self.npaths, CENSUS_BITS, self.p1, self.p2, self.s_bound))

    def close(self):
        if getattr(self, "_h", None):
            self.L.xcb_sgm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        if rc != _lib.XCB_OK:
            msg = (self.L.xcb_sgm_last_error(self._h) or b"").decode(errors="replace")
            raise RuntimeError("%s failed (%d): %s" % (what, rc, msg))

    def compute_gpu(self, left, right, disp=None, conf=None, stream=0):
        """left / right: torch CUDA uint8 (H, W) -> (disp, conf) torch CUDA float32 (H, W); asynchronous."""
        import torch
        for t in (left, right):
            if not (t.is_cuda and t.dtype == torch.uint8 and t.is_contiguous() and tuple(t.shape) == (self.H, self.W)):
                raise ValueError("SGM32.compute_gpu: contiguous CUDA uint8 (H, W) tensors")
        if disp is None:
            disp = torch.empty((self.H, self.W), dtype=torch.float32, device=left.device)
        if conf is None:
            conf = torch.empty((self.H, self.W), dtype=torch.float32, device=left.device)
        v = lambda t: ctypes.c_void_p(t.data_ptr())
        self._chk(self.L.xcb_sgm_compute_dev(self._h, v(left), v(right), v(disp), v(conf),
                                             ctypes.c_void_p(int(stream) or None)), "xcb_sgm_compute_dev")
        self.n_aggregations += 1
        self.n_frames += 1
        return disp, conf

    def compute(self, left, right):
        """(H, W) uint8 rectified pair -> (disp, conf) host float32; disp 0 = invalid (no measurement)."""
        t0 = time.perf_counter()
        L = np.ascontiguousarray(left, np.uint8).reshape(self.H, self.W)
        R = np.ascontiguousarray(right, np.uint8).reshape(self.H, self.W)
        disp = np.empty((self.H, self.W), np.float32)
        conf = np.empty((self.H, self.W), np.float32)
        p = lambda a: ctypes.c_void_p(a.ctypes.data)
        self._chk(self.L.xcb_sgm_compute_host(self._h, p(L), p(R), p(disp), p(conf)), "xcb_sgm_compute_host")
        self.n_aggregations += 1
        self.n_frames += 1
        self.ms.append((time.perf_counter() - t0) * 1e3)
        return disp, conf

    def set_stage_timing(self, on=True):
        """In-stream events around the cost, aggregation and selection kernels of each compute (for profiling)."""
        self._chk(self.L.xcb_sgm_set_stage_timing(self._h, 1 if on else 0), "xcb_sgm_set_stage_timing")

    def stage_times(self):
        """-> ({"cost", "aggregate", "select"} ms summed over the timed calls since the last read, calls); waits."""
        ms = (ctypes.c_float * 3)()
        n = ctypes.c_int(0)
        self._chk(self.L.xcb_sgm_stage_times(self._h, ms, ctypes.byref(n)), "xcb_sgm_stage_times")
        return {"cost": ms[0], "aggregate": ms[1], "select": ms[2]}, int(n.value)

    def _volume(self, which, dtype):
        n = self.H * self.W * MAX_DISP
        out = np.empty(n, dtype)
        p = ctypes.c_void_p(out.ctypes.data)
        self._chk(self.L.xcb_sgm_read_volumes(self._h, p if which == "cost" else None, p if which == "sum" else None),
                  "xcb_sgm_read_volumes")
        return out.reshape(self.H, self.W, MAX_DISP)

    def aggregated_volume(self):
        """The last uint16 aggregated volume (H, W, 128) on the host (tests only)."""
        return self._volume("sum", np.uint16)

    def cost_volume(self):
        return self._volume("cost", np.uint8)


class SgmDepth:
    """The depth stage: compute(left, right) -> (H, W) float32 positive disparity, 0 = invalid; one SGM32 per image
    size, built lazily (sgm32.py:378-411)."""

    def __init__(self, verbose=True):
        self.verbose = verbose
        self._sgm = None
        self.last_conf = None

    def _get(self, W, H):
        if self._sgm is None or (self._sgm.W, self._sgm.H) != (W, H):
            self._sgm = SGM32(W, H, verbose=self.verbose)
        return self._sgm

    def compute(self, left, right):
        H, W = left.shape[:2]
        d, c = self._get(W, H).compute(left, right)
        self.last_conf = c
        return d

    def stats(self):
        s = self._sgm
        if s is None or not s.ms:
            return None
        a = np.asarray(s.ms)
        return {"frames": int(s.n_frames), "aggregations": int(s.n_aggregations),
                "p50_ms": float(np.percentile(a, 50)), "p95_ms": float(np.percentile(a, 95)), "size": [s.W, s.H]}
