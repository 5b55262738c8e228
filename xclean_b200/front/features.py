"""The frontend constants and the host-side pieces of xclean's classical frontend that the device path needs.

Constants (src/xclean/stages/features.py:43-51, src/xclean/stereo/epipolar.py:35-44, src/xclean/stereo/sgm32.py:68-76,
src/xclean/core/derive.py:47-49) and the cell / min-distance geometry of Frontend._cell / _min_dist
(features.py:135-140).  `Frontend` here is the light object the engine reaches through `Detector.fe`: the budget
geometry, the stats dict and `match_desc` (replaced by the device matcher in front.gpu_front.Detector)."""
from __future__ import annotations

import math

import numpy as np

KLT_WIN = 21
SHI_QUALITY = 0.01
ORB_PATCH = 31
ORB_PAD = 32
HAMMING_BITS = 256
HAMMING_CHANCE = int(HAMMING_BITS / 2 - 3 * math.sqrt(HAMMING_BITS) / 2)    # 104
RATIO = 0.8

HALF = 5
ZNCC_MIN = 0.5
LK_ITERS = 6
MAX_DISP = 128
UNIQUENESS = 0.05
LR_THRESHOLD_PX = 1.0

HUBER_K = 1.345
MIN_PNP_INLIERS = 25
COLD_MATCH_RATE = 0.5
COLD_INLIER_RATE = 0.5

_NOISE_Q99 = None


def noise_q99():
    """99th percentile of cv2.cornerMinEigenVal(3, 3) at 3x3 local maxima of unit Gaussian noise (seed 12345, 512x512,
    float input), the constant of features.noise_floor_8u (features.py:64-69); computed once with cv2 as the
    reference computes it."""
    global _NOISE_Q99
    if _NOISE_Q99 is None:
        import cv2
        rng = np.random.default_rng(12345)
        z = rng.normal(0.0, 1.0, (512, 512)).astype(np.float32)
        Rz = cv2.cornerMinEigenVal(z, 3, 3)
        mx = Rz >= cv2.dilate(Rz, np.ones((3, 3), np.uint8))
        _NOISE_Q99 = float(np.quantile(Rz[8:-8, 8:-8][mx[8:-8, 8:-8]], 0.99))
    return _NOISE_Q99


def noise_floor_host(gray):
    """features.noise_floor_8u with cv2 / numpy on the host (the start-up check's reference value)."""
    import cv2
    Nk = np.array([[1, -2, 1], [-2, 4, -2], [1, -2, 1]], np.float32)
    H, W = gray.shape
    c = cv2.filter2D(gray.astype(np.float32), -1, Nk)[1:-1, 1:-1]
    sn = float(np.sqrt(np.pi / 2.0) / (6.0 * (W - 2) * (H - 2)) * np.abs(c).sum())
    return noise_q99() * sn * sn / (255.0 * 255.0)


class Frontend:
    """The slice of stages/features.Frontend the P1 detector uses (budget geometry, stats, match_desc)."""

    def __init__(self, rig=None, cap=None, verbose=False):
        self.rig = rig
        self.cap = int(cap or 2048)
        self.detect_mode = "cell"
        self.stats = {"detected": 0}

    def _cell(self, W, H, budget):
        return max(4.0, math.sqrt(W * H / max(budget, 1)))

    def _min_dist(self, W, H, budget):
        return max(2.0, math.sqrt(W * H / (2.0 * math.sqrt(3.0) * max(budget, 1))))

    def match_desc(self, f0, f1, mask0=None, mask1=None):
        raise RuntimeError("Frontend.match_desc: attach a device matcher (front.gpu_front.Detector does)")
