"""The frontend's host-side budget control and grid geometry on the CPU (no device): front/detect.Detector's budget
(src/xclean/front/detect.py:46-58) and stages/features.Frontend's cell and minimum-distance geometry
(src/xclean/stages/features.py:135-139), with the constants of src/xclean/core/derive.py:48, :55-56 and
stages/features.py's Hamming chance bound.

Budget: N = ceil(3 x 3 x MIN_PNP_INLIERS / y), y the median of the last `window` yields (inliers / detections; a
frame with no detections leaves them unchanged), cold start y = 0.5 x 0.5, y at least 1e-3, N clamped to
[rig.conditioning_floor(), cap]."""
import math

from xclean_b200.front import detect as D
from xclean_b200.front import features as F


class Rig:
    def __init__(self, floor=100, W=1241, H=376):
        self.floor, self.width, self.height = floor, W, H

    def conditioning_floor(self):
        return self.floor


def test_constants():
    assert (F.MIN_PNP_INLIERS, F.COLD_MATCH_RATE, F.COLD_INLIER_RATE) == (25, 0.5, 0.5)
    assert F.HAMMING_CHANCE == 104 and F.RATIO == 0.8


def test_budget_control():
    d = D.Detector(Rig(100), cap=2048, window=10)
    assert d.budget == 900                           # cold start: ceil(225 / 0.25)
    d.report_yield(50, 1000)                         # y = 0.05 -> 4,500, capped
    assert d.budget == 2048
    d.report_yield(300, 1000)                        # median(0.05, 0.3) = 0.175 -> ceil(1285.7)
    assert d.budget == math.ceil(225 / 0.175)
    d.report_yield(10, 0)                            # no detections: yields unchanged
    assert d._yields == [0.05, 0.3] and d.budget == math.ceil(225 / 0.175)
    for k in range(12):                              # only the last 10 yields count
        d.report_yield(100 + 50 * k, 1000)
    assert len(d._yields) == 10 and d._yields[0] == 0.2
    assert d.budget == math.ceil(225 / ((0.4 + 0.45) / 2))
    d2 = D.Detector(Rig(100), cap=2048)
    d2.report_yield(0, 500)                          # y = 0 -> 1e-3 -> 225,000, capped
    assert d2.budget == 2048
    d3 = D.Detector(Rig(1000), cap=2048)
    d3.report_yield(900, 1000)                       # y = 0.9 -> 250, under the conditioning floor
    assert d3.budget == 1000
    d4 = D.Detector(Rig(100), cap=500)
    assert d4.budget == 500                          # cold start above the cap


def test_grid_geometry():
    fe = F.Frontend(Rig(), cap=2048)
    assert fe._cell(1241, 376, 2000) == math.sqrt(1241 * 376 / 2000)
    assert fe._cell(64, 48, 10_000) == 4.0
    assert fe._cell(100, 100, 0) == 100.0
    assert fe._min_dist(1241, 376, 2000) == math.sqrt(1241 * 376 / (2.0 * math.sqrt(3.0) * 2000))
    assert fe._min_dist(64, 48, 10_000) == 2.0
