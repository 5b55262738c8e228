"""The dense SGM oracle (oracle/sgm_oracle.c, the reference's sgm32.py restated in C) on the host: its path geometry
against the reference's formulas as the drop-in module states them, the exactness bound of the uint16 volume, and the
disparities it recovers on a pair whose true disparity is known (a textured image shifted by whole pixels)."""
import numpy as np

from oracle import sgm_oracle as SO
from xclean_b200.stereo import sgm32 as M


def test_directions_and_path_starts():
    d = M.directions()
    assert len(d) == 32 and len({(a, b) for a, b, _n, _d in d}) == 32
    for H, W in ((7, 9), (64, 96), (2, 5)):
        for dx, dy, _n, _d in d:
            st = M.path_starts(H, W, dx, dy)
            bx, by = min(abs(dx), W), min(abs(dy), H)
            assert len(st) == bx * H + by * (W - bx)          # the count the device derives its starts from
    p2s = [M.P2 * n // dd for (_x, _y, n, dd) in d]
    assert 32 * (M.CENSUS_BITS + max(p2s)) < 65536 and (M.P1, M.P2) == (13, 152)


def test_oracle_recovers_a_known_shift():
    rng = np.random.default_rng(3)
    H, W, shift = 48, 120, 7
    base = (rng.random((H, W + shift)) * 255).astype(np.uint8)
    left = np.ascontiguousarray(base[:, :W])                # left(x) = right(x - shift)
    right = np.ascontiguousarray(base[:, shift:])
    disp, conf, C, S = SO.sgm(left, right, volumes=True)
    inner = disp[:, 20:-8]
    ok = inner > 0
    assert ok.mean() > 0.8
    assert np.abs(inner[ok] - shift).max() < 0.6
    assert (C[:, :3, 5:] == 80).all()                       # x - d < 0: the census maximum
    assert S.max() < 32 * (80 + max(M.P2 * n // dd for (_x, _y, n, dd) in M.directions()))
