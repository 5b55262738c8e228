"""The stress shape of the frontend on the device: 1280x720 frames, 4,000 features, capacity 4,096, disparities
0-127 (the reference's 128-value range, MAX_DISP 128), the reference's 11x11 ZNCC window and the 9x9 one.

Bit-exact against the oracle (the reference's CPU path restated in C) on the same seeded frames: keypoints,
descriptors, disparities / sigmas / flags / ZNCC / dy, match counts and indices; the front is calibrated against this
machine's cv2 first, as the reference's start-up does (gpu_front.py:1423-1513).  Also: keypoint counts at the
capacity, one stereo call over more points than the reference's 4,096-point chunk (gpu_front.py:1342-1383), and the
Hamming matcher at 4k x 4k with many ties."""
import numpy as np
import pytest

from oracle import front_oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu

W, H = 1280, 720
BUDGET = 4000
CAP = 4096
DLO, DHI = 0, 127


@pytest.fixture(scope="module")
def hd():
    from xclean_b200 import synth
    from xclean_b200.front.gpu_front import GpuFront
    L, R = synth.sequence(synth.CAM_HD, 6, seed=3)
    gf = GpuFront(W, H, cap=CAP, max_frames=4)
    cal = gf.calibrate(cache=False)
    yield gf, cal, L.numpy(), R.numpy()
    gf.close()


def _same_frames(out, ref, frames):
    assert np.array_equal(out["counts"][:frames], ref["counts"][:frames])
    for f in range(frames):
        n = int(ref["counts"][f])
        assert G.same_bits(out["kp"][f, :n], ref["kp"][f, :n]), f
        assert np.array_equal(out["desc"][f, :n], ref["desc"][f, :n]), f
        for k in ("d", "sig", "zn"):
            assert G.same_bits(out[k][f, :n], ref[k][f, :n]), (f, k)
        assert np.array_equal(out["ok"][f, :n], ref["ok"][f, :n]), f
        assert G.same_bits(np.nan_to_num(out["dy"][f, :n], nan=-1e300), np.nan_to_num(ref["dy"][f, :n], nan=-1e300))
        m = int(ref["nmatch"][f])
        assert out["nmatch"][f] == m, f
        assert np.array_equal(out["m0"][f, :m], ref["m0"][f, :m]) and np.array_equal(out["m1"][f, :m], ref["m1"][f, :m])


@pytest.mark.parametrize("half", [5, 4])
def test_hd_pipeline_bitexact(hd, half):
    gf, cal, L, R = hd
    out = gf.pipeline(L[:4], R[:4], BUDGET, half=half, dlo=DLO, dhi=DHI, match_prev=False)
    ref = O.frames(L[:4], R[:4], BUDGET, cal["q99"], cal, gf.pattern, half=half, dlo=DLO, dhi=DHI, cap=CAP)
    assert ref["counts"].min() > 3000 and ref["nmatch"][1:].min() > 100
    _same_frames(out, ref, 4)


def test_hd_pipeline_batches_bitexact(hd):
    """Six frames in batches of four (the second batch's upload overlaps the first's compute); matches run across the
    batch boundary."""
    import torch
    gf, cal, L, R = hd
    Lp = torch.from_numpy(L).pin_memory().numpy()
    Rp = torch.from_numpy(R).pin_memory().numpy()
    out = gf.pipeline_batches(Lp, Rp, BUDGET, batch=4, half=5, dlo=DLO, dhi=DHI, match_prev=False)
    ref = O.frames(L, R, BUDGET, cal["q99"], cal, gf.pattern, half=5, dlo=DLO, dhi=DHI, cap=CAP)
    assert ref["nmatch"][4] > 0
    _same_frames(out, ref, 6)


def test_hd_counts_at_capacity(hd):
    """budget = cap = 4,096 on dense noise texture: more than 4,000 keypoints per frame, the per-frame buffers filled
    to within 2 % of their end."""
    import cv2
    gf, cal, _L, _R = hd
    rng = np.random.default_rng(5)
    L = np.stack([cv2.GaussianBlur((rng.random((H, W)) * 255).astype(np.uint8), (0, 0), s) for s in (1.0, 1.5)])
    R = np.roll(L, -9, axis=2).copy()
    out = gf.pipeline(L, R, CAP, half=5, dlo=DLO, dhi=DHI, match_prev=False)
    ref = O.frames(L, R, CAP, cal["q99"], cal, gf.pattern, half=5, dlo=DLO, dhi=DHI, cap=CAP)
    assert (ref["counts"] > 4000).all()
    _same_frames(out, ref, 2)


def test_hd_stereo_past_one_chunk(hd):
    """One stereo call over 6,000 points (the reference splits calls into 4,096-point chunks), with a row band."""
    gf, cal, L, R = hd
    rng = np.random.default_rng(7)
    kp = np.stack([rng.uniform(-3, W + 3, 6000), rng.uniform(-3, H + 3, 6000)], axis=1)
    lo = rng.integers(0, 40, 6000).astype(np.int64)
    hi = lo + rng.integers(0, 88, 6000).astype(np.int64)
    for dy, band in ((0.0, 0), (0.25, 2)):
        d, s, ok, zn, ody = gf.stereo(L[0], R[0], kp, lo, hi, dy=dy, band=band, half=5)
        od, osg, ook, ozn, oody = O.stereo(L[0], R[0], kp, lo, hi, dy=dy, band=band, half=5)
        assert ok.sum() > 600
        assert G.same_bits(d, od) and G.same_bits(s, osg) and np.array_equal(ok, ook) and G.same_bits(zn, ozn)
        assert G.same_bits(np.nan_to_num(ody + dy, nan=-1e300), np.nan_to_num(oody, nan=-1e300))


def test_hd_hamming_4k_by_4k(hd):
    """4,096 x 4,096 descriptors, a third of them drawn from a small pool (many exact ties): best / second / index, the
    column first-minimum, and the gated mutual matches equal the CPU scan."""
    gf = hd[0]
    rng = np.random.default_rng(11)
    pool = rng.integers(0, 256, (24, 32), dtype=np.uint8)
    A = np.where(rng.random((4096, 1)) < 0.33, pool[rng.integers(0, 24, 4096)],
                 rng.integers(0, 256, (4096, 32), dtype=np.uint8)).astype(np.uint8)
    B = np.where(rng.random((4096, 1)) < 0.33, pool[rng.integers(0, 24, 4096)],
                 rng.integers(0, 256, (4096, 32), dtype=np.uint8)).astype(np.uint8)
    B[:1000] = A[rng.permutation(4096)[:1000]] ^ (rng.random((1000, 32)) < 0.02).astype(np.uint8)
    got = gf.hamming(A, B)
    ref = O.hamming(A, B)
    for g, r, nm in zip(got, ref, ("best", "second", "index", "column index")):
        assert np.array_equal(g, r), nm
    i0, i1 = gf.match(A, B)
    q, t = O.match_desc(A, B)
    assert len(q) > 500 and np.array_equal(i0, q) and np.array_equal(i1, t)
