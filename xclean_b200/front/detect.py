"""Per-frame detector base: the budget control of front/detect.Detector (src/xclean/front/detect.py:34-58).

N = ceil(3 x 3 x MIN_PNP_INLIERS / y), y = running median over the last `window` frames of (inliers / detections),
cold start y = COLD_MATCH_RATE x COLD_INLIER_RATE; clamped to [rig.conditioning_floor(), cap].  The extraction itself
is the device path in front.gpu_front.Detector."""
from __future__ import annotations

import math

import numpy as np

from .features import COLD_INLIER_RATE, COLD_MATCH_RATE, MIN_PNP_INLIERS, Frontend


class Detector:
    def __init__(self, rig, cap=2048, window=10):
        self.fe = Frontend(rig, cap=cap, verbose=False)
        self.fe.detect_mode = "cell"
        self.rig = rig
        self.cap = int(cap)
        self.window = int(window)
        self._yields = []
        self.budget = self._budget()
        self.stats = {"frames": 0, "detected": 0}

    def _budget(self):
        y = float(np.median(self._yields)) if self._yields else COLD_MATCH_RATE * COLD_INLIER_RATE
        y = max(y, 1e-3)
        n = int(math.ceil(3 * 3 * MIN_PNP_INLIERS / y))
        floor = self.rig.conditioning_floor() if hasattr(self.rig, "conditioning_floor") else 0
        return int(min(max(n, floor), self.cap))

    def report_yield(self, n_inliers, n_detected):
        if n_detected > 0:
            self._yields.append(float(n_inliers) / float(n_detected))
            self._yields = self._yields[-self.window:]
        self.budget = self._budget()

    def __call__(self, gray):
        raise NotImplementedError("the device detector is front.gpu_front.Detector")
