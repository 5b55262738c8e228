"""The CPU oracle of the multi-scale oriented extras (oracle/ext_oracle.{c,py}) pinned to OpenCV, which defines them:
FAST against cv2.FastFeatureDetector (TYPE_9_16), the pyramid against cv2.resize(INTER_LINEAR_EXACT), the steered
descriptor against cv2.ORB.compute at KeyPoint.angle = 12 k on the reference's pad-32 convention
(src/xclean/stages/features.py:405-421), and the blur model against cv2.sepFilter2D at every level size.  The
selection and the orientation bins are this package's own definitions and are checked against plain numpy
restatements."""
import math

import numpy as np
import pytest

cv2 = pytest.importorskip("cv2")

from oracle import ext_oracle as X
from oracle import front_oracle as O


def _frame(seed=3):
    from xclean_b200 import synth
    L, _R = synth.sequence(synth.CAM_SMALL, 1, seed=seed)
    return L.numpy()[0]


def _cv_fast(img, t, nms):
    det = cv2.FastFeatureDetector_create(t, nms, cv2.FAST_FEATURE_DETECTOR_TYPE_9_16)
    ks = det.detect(img)
    c = np.array([k.pt for k in ks], np.float32).reshape(-1, 2)
    r = np.array([k.response for k in ks], np.float32)
    o = np.lexsort((c[:, 0], c[:, 1]))
    return c[o], r[o]


@pytest.mark.parametrize("t", [20, 7, 0])
@pytest.mark.parametrize("nms", [True, False])
def test_fast_matches_cv2(t, nms):
    img = _frame()[100:300, 200:520].copy()
    kp, rs = X.fast(img, t, nms)
    c, r = _cv_fast(img, t, nms)
    assert np.array_equal(kp, c)
    if nms:                       # cv2 reports scores only when it suppresses (response 0 otherwise)
        assert np.array_equal(rs, r)
    assert len(kp) > 50


def test_fast_noise_and_tiny_images():
    rng = np.random.default_rng(5)
    img = (rng.random((61, 97)) * 255).astype(np.uint8)
    for t in (10, 40):
        kp, rs = X.fast(img, t, True)
        c, r = _cv_fast(img, t, True)
        assert np.array_equal(kp, c) and np.array_equal(rs, r)
    for shape in ((7, 7), (6, 9), (1, 1)):
        z = (rng.random(shape) * 255).astype(np.uint8)
        kp, _ = X.fast(z, 5, True)
        c, _ = _cv_fast(z, 5, True)
        assert np.array_equal(kp, c)


@pytest.mark.parametrize("src,dst", [((752, 480), (627, 400)), ((1280, 720), (1067, 600)), ((97, 61), (81, 51)),
                                     ((9, 5), (8, 4)), ((33, 17), (1, 2)), ((100, 100), (67, 33)), ((5, 5), (5, 5))])
def test_pyramid_step_matches_cv2_linear_exact(src, dst):
    rng = np.random.default_rng(sum(src) + sum(dst))
    img = (rng.random((src[1], src[0])) * 255).astype(np.uint8)
    want = cv2.resize(img, dst, interpolation=cv2.INTER_LINEAR_EXACT)
    assert np.array_equal(X.pyr_down(img, dst[0], dst[1]), want)


def test_pyramid_chain_on_a_frame():
    img = _frame()
    cur = img
    for (w, h, _s) in X.level_sizes(img.shape[1], img.shape[0], 4, 1.2)[1:]:
        nxt = X.pyr_down(cur, w, h)
        assert np.array_equal(nxt, cv2.resize(cur, (w, h), interpolation=cv2.INTER_LINEAR_EXACT))
        cur = nxt
    assert [s[:2] for s in X.level_sizes(752, 480, 4, 1.2)] == [(752, 480), (627, 400), (522, 333), (435, 278)]


def test_quotas():
    for (n, L, s) in ((2000, 4, 1.2), (4000, 4, 1.2), (500, 8, 1.2), (3, 4, 2.0), (1, 1, 1.5)):
        q = X.quotas(n, L, s)
        assert sum(q) == n and len(q) == L and all(v >= 0 for v in q)
    assert X.quotas(2000, 4, 1.2)[0] > X.quotas(2000, 4, 1.2)[1]


def test_steered_tables_and_descriptors_match_cv2_at_every_bin():
    from xclean_b200.front.gpu_front import _orb, probe_orb_pattern
    from xclean_b200.front.orb_ext import steered_patterns
    pat = probe_orb_pattern().reshape(256, 4)
    T = X.steered_patterns(pat)
    assert np.array_equal(steered_patterns(pat), T)          # the product's vectorised builder
    assert np.array_equal(T[0], pat)                         # bin 0 = the reference's unrotated tests
    assert np.abs(T).max() <= 18
    img = _frame(seed=4)[60:260, 100:400].copy()
    kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
    pad = cv2.copyMakeBorder(img, 32, 32, 32, 32, cv2.BORDER_REFLECT_101)
    B = cv2.sepFilter2D(pad, -1, kf, kf, borderType=cv2.BORDER_REFLECT_101)
    assert np.array_equal(O.blur(img, kf, img.shape[1] + 64, img.shape[1] + 64), B)
    pts = np.array([(x, y) for y in range(0, 200, 17) for x in range(0, 300, 19)], np.float32)
    for k in range(X.BINS):
        bins = np.full(len(pts), k, np.int32)
        d = X.orb_steer(B, pts, bins, T)
        kps = [cv2.KeyPoint(float(x) + 32, float(y) + 32, 31, 12.0 * k, 0.0, 0, i) for i, (x, y) in enumerate(pts)]
        ok, dc = _orb().compute(pad, kps)
        cid = np.array([q.class_id for q in ok])
        assert len(cid) == len(pts)
        assert np.array_equal(d[cid], dc), "bin %d" % k


def test_orientation_bins():
    img = _frame()
    kp, rs = X.fast(img, 20, True)
    ks, _ = X.select(kp, rs, img.shape[1], img.shape[0], 16, 800)
    bins, mom = X.ic_bins(img, ks)
    # the moments restated in numpy
    for i in range(0, len(ks), 37):
        x, y = int(ks[i, 0]), int(ks[i, 1])
        v, u = np.mgrid[-15:16, -15:16]
        m = u * u + v * v <= 240
        P = img[y - 15:y + 16, x - 15:x + 16].astype(np.int64)
        assert mom[i, 0] == int((u * P)[m].sum()) and mom[i, 1] == int((v * P)[m].sum())
    # the bin is floor((atan2 + 6) / 12) away from the boundaries
    ang = np.degrees(np.arctan2(mom[:, 1], mom[:, 0])) % 360.0
    far = np.abs(((ang + 6.0) % 12.0) - 6.0) < 5.999
    assert np.array_equal(bins[far], (np.floor((ang[far] + 6.0) / 12.0).astype(int) % 30))
    assert len(np.unique(bins)) > 20
    # a flat patch has no direction: bin 0
    flat = np.full((64, 64), 90, np.uint8)
    b0, m0 = X.ic_bins(flat, np.array([[32, 32]], np.float32))
    assert b0[0] == 0 and m0[0, 0] == 0 and m0[0, 1] == 0


def test_orientation_bins_partition_the_plane():
    # vectors on and next to every boundary direction get exactly one bin, the geometrically right one
    bd =[(math.cos(math.radians(12 * k - 6)), math.sin(math.radians(12 * k - 6))) for k in range(30)]
    for k in range(30):
        for eps in (-1e-3, 0.0, 1e-3):
            a = math.radians(12 * k - 6) + eps
            X_, Y_ = round(1e6 * math.cos(a)), round(1e6 * math.sin(a))
            hits = []
            for j in range(30):
                j1 = (j + 1) % 30
                c0 = bd[j][0] * Y_ - bd[j][1] * X_
                c1 = bd[j1][0] * Y_ - bd[j1][1] * X_
                dc = math.cos(math.radians(12 * j)) * X_ + math.sin(math.radians(12 * j)) * Y_
                if c0 >= 0 and c1 < 0 and dc > 0:
                    hits.append(j)
            assert len(hits) == 1
            if eps > 0:
                assert hits[0] == k
            if eps < 0:
                assert hits[0] == (k - 1) % 30


def test_selection_is_a_stable_top_k():
    rng = np.random.default_rng(9)
    n, W, H, edge = 3000, 200, 150, 16
    kp = np.stack([rng.integers(0, W, n), rng.integers(0, H, n)], 1).astype(np.float32)
    rs = rng.integers(20, 60, n).astype(np.float32)
    for quota in (0, 1, 100, 1000, 5000):
        ks, rsel = X.select(kp, rs, W, H, edge, quota)
        inside = np.nonzero((kp[:, 0] >= edge) & (kp[:, 0] < W - edge) & (kp[:, 1] >= edge) & (kp[:, 1] < H - edge))[0]
        order = inside[np.argsort(-rs[inside], kind="stable")][:quota]
        want = np.sort(order)
        assert np.array_equal(ks, kp[want]) and np.array_equal(rsel, rs[want])


@pytest.mark.parametrize("W,H", [(752, 480), (1280, 720)])
def test_blur_model_reproduces_cv2_at_every_level_size(W, H):
    kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
    rng = np.random.default_rng(W)
    for (w, h, _s) in X.level_sizes(W, H, 4, 1.2):
        img = (rng.random((h, w)) * 255).astype(np.uint8)
        pad = cv2.copyMakeBorder(img, 32, 32, 32, 32, cv2.BORDER_REFLECT_101)
        want = cv2.sepFilter2D(pad, -1, kf, kf, borderType=cv2.BORDER_REFLECT_101)
        Wp = w + 64
        cands = sorted(set([Wp] + [(Wp // m) * m for m in (4, 8, 16, 32, 64, 128)] + [0]), reverse=True)
        assert any(np.array_equal(O.blur(img, kf, vr, vc), want) for vr in cands for vc in cands)


def test_pipeline_descriptors_are_cv2_orb_at_the_bin_angles():
    """The whole per-frame oracle: each level's descriptors equal cv2.ORB.compute on that level's pad-32 image."""
    from xclean_b200.front.gpu_front import _orb, probe_orb_pattern
    img = _frame(seed=6)
    kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
    sizes = X.level_sizes(img.shape[1], img.shape[0], 4, 1.2)
    calib = [(kf, w + 64, w + 64) for (w, _h, _s) in sizes]
    pats = X.steered_patterns(probe_orb_pattern())
    out = X.orbx(img, 4, 1.2, 1000, 20, 31, True, pats, calib)
    q = X.quotas(1000, 4, 1.2)
    off = np.concatenate([[0], np.cumsum(q)])
    assert out["counts"].sum() > 500
    for lv in range(4):
        n = int(out["counts"][lv])
        sl = slice(off[lv], off[lv] + n)
        lvl = out["levels"][lv]
        pad = cv2.copyMakeBorder(lvl, 32, 32, 32, 32, cv2.BORDER_REFLECT_101)
        kps = [cv2.KeyPoint(float(x) + 32, float(y) + 32, 31, 12.0 * float(b), 0.0, 0, i)
               for i, ((x, y), b) in enumerate(zip(out["kp_level"][sl], out["bins"][sl]))]
        ok, dc = _orb().compute(pad, kps)
        cid = np.array([k.class_id for k in ok])
        assert len(cid) == n
        assert np.array_equal(out["desc"][sl][cid], dc)
        assert np.array_equal(out["kp"][sl], out["kp_level"][sl] * np.float32(sizes[lv][2]))
