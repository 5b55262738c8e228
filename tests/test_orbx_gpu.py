"""The device multi-scale oriented extras (csrc/front_ext.cu through the C ABI) bit for bit against the CPU oracle
(oracle/ext_oracle) and against OpenCV where OpenCV defines the result: FAST (cv2.FastFeatureDetector TYPE_9_16), the
pyramid (cv2.resize INTER_LINEAR_EXACT), the steered descriptors (cv2.ORB.compute at KeyPoint.angle = 12 k on the
reference's pad-32 convention, src/xclean/stages/features.py:405-421).  Level 0 at bin 0 is the reference's own
descriptor (GpuFront.describe_points)."""
import ctypes

import numpy as np
import pytest

cv2 = pytest.importorskip("cv2")

from oracle import ext_oracle as X

pytestmark = pytest.mark.gpu


def _frame(cam="small", seed=3):
    from xclean_b200 import synth
    c = synth.CAM_SMALL if cam == "small" else synth.CAM_HD
    L, _R = synth.sequence(c, 1, seed=seed)
    return L.numpy()[0]


def _v(t):
    return ctypes.c_void_p(t.data_ptr())


def _dev_fast(img, t, nms, cap=None):
    import torch
    from xclean_b200 import _lib
    L = _lib.lib()
    H, W = img.shape
    cap = H * W if cap is None else cap
    g = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    kp = torch.zeros((max(cap, 1), 2), dtype=torch.float32, device="cuda")
    rs = torch.zeros(max(cap, 1), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    nb = L.xcb_fast_scratch_bytes(W, H)
    scr = torch.empty(nb, dtype=torch.uint8, device="cuda")
    _lib.check(L.xcb_fast_dev(_v(g), W, H, int(t), 1 if nms else 0, int(cap), _v(kp), _v(rs), _v(cnt), _v(scr), nb,
                              None), None, "xcb_fast_dev")
    torch.cuda.synchronize()
    n = int(cnt.item())
    m = min(n, cap)
    return n, kp[:m].cpu().numpy(), rs[:m].cpu().numpy()


@pytest.mark.parametrize("t,nms", [(20, True), (7, True), (0, True), (20, False), (0, False)])
def test_fast_matches_oracle_and_cv2(t, nms):
    img = _frame()
    n, kp, rs = _dev_fast(img, t, nms)
    ok, ors = X.fast(img, t, nms)
    assert n == len(ok)
    assert np.array_equal(kp, ok) and np.array_equal(rs, ors)
    det = cv2.FastFeatureDetector_create(t, nms, cv2.FAST_FEATURE_DETECTOR_TYPE_9_16)
    c = np.array([k.pt for k in det.detect(img)], np.float32).reshape(-1, 2)
    c = c[np.lexsort((c[:, 0], c[:, 1]))]
    assert np.array_equal(kp, c)


def test_fast_capacity_tiny_and_hd():
    img = _frame()
    n, kp, _ = _dev_fast(img, 20, True, cap=100)
    ok, _ = X.fast(img, 20, True)
    assert n == len(ok) and np.array_equal(kp, ok[:100])          # the count is the total; the first cap written
    rng = np.random.default_rng(1)
    for shape in ((7, 7), (5, 9), (1, 1)):
        z = (rng.random(shape) * 255).astype(np.uint8)
        n, kp, _ = _dev_fast(z, 5, True)
        assert n == len(X.fast(z, 5, True)[0])
    hd = _frame("hd", 2)
    n, kp, rs = _dev_fast(hd, 20, True)
    ok, ors = X.fast(hd, 20, True)
    assert np.array_equal(kp, ok) and np.array_equal(rs, ors)


def test_pyramid_step_matches_oracle_and_cv2():
    import torch
    from xclean_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(2)
    for (src, dst) in (((752, 480), (627, 400)), ((1280, 720), (1067, 600)), ((97, 61), (81, 51)), ((9, 5), (8, 4)),
                       ((33, 17), (1, 2))):
        img = (rng.random((src[1], src[0])) * 255).astype(np.uint8)
        tabs = []
        for ns, nd in ((src[0], dst[0]), (src[1], dst[1])):
            i = np.zeros(nd, np.int32)
            w = np.zeros(nd, np.int32)
            _lib.check(L.xcb_pyr_tables(ns, nd, _lib.ptr(i), _lib.ptr(w)), None, "xcb_pyr_tables")
            tabs += [torch.from_numpy(i).cuda(), torch.from_numpy(w).cuda()]
        g = torch.from_numpy(img).cuda()
        out = torch.empty((dst[1], dst[0]), dtype=torch.uint8, device="cuda")
        _lib.check(L.xcb_pyr_down_dev(_v(g), src[0], src[1], _v(out), dst[0], dst[1], *[_v(t) for t in tabs], None),
                   None, "xcb_pyr_down_dev")
        got = out.cpu().numpy()
        assert np.array_equal(got, X.pyr_down(img, dst[0], dst[1]))
        assert np.array_equal(got, cv2.resize(img, dst, interpolation=cv2.INTER_LINEAR_EXACT))


def _orbx(W, H, levels, scale, nfeat, thr=20, edge=31, nonmax=True):
    from xclean_b200.front.orb_ext import OrbPyramid
    return OrbPyramid(W, H, levels=levels, scale=scale, nfeatures=nfeat, fast_threshold=thr, edge=edge, nonmax=nonmax)


def _oracle_slots(ox, img):
    calib = [(ox.calib["kf"], vr, vc) for (vr, vc) in ox.calib["blur"]]
    return X.orbx(img, ox.nlevels, ox.scale, ox.nfeatures, ox.threshold, ox.edge, ox.nonmax, ox.calib["patterns"],
                  calib)


def _same_slots(got, want, ox):
    assert np.array_equal(got["counts"], want["counts"])
    for lvl, n in zip(ox.levels, got["counts"]):
        sl = slice(lvl["offset"], lvl["offset"] + int(n))
        for k in ("kp", "kp_level", "resp", "level", "bins", "desc"):
            assert np.array_equal(got[k][sl], want[k][sl]), k


@pytest.mark.parametrize("cam,levels,scale,nfeat", [("small", 4, 1.2, 2000), ("hd", 4, 1.2, 4000),
                                                    ("small", 3, 1.5, 300)])
def test_pipeline_matches_the_oracle_slot_for_slot(cam, levels, scale, nfeat):
    img = _frame(cam, 5)
    H, W = img.shape
    ox = _orbx(W, H, levels, scale, nfeat)
    try:
        got = ox.detect_slots(img)
        want = _oracle_slots(ox, img)
        _same_slots(got, want, ox)
        for lv in range(levels):
            assert np.array_equal(ox.level_image(lv), want["levels"][lv])
        f = ox.detect(img)
        assert len(f.kp) == int(got["counts"].sum()) > 0.5 * nfeat
        assert set(np.unique(f.level)) == set(range(levels))
    finally:
        ox.close()


def test_pipeline_levels_and_descriptors_are_cv2():
    from xclean_b200.front.gpu_front import _orb
    img = _frame("small", 7)
    H, W = img.shape
    ox = _orbx(W, H, 4, 1.2, 1500)
    try:
        s = ox.detect_slots(img)
        cur = img
        for lv, lvl in enumerate(ox.levels):
            im = ox.level_image(lv)
            if lv:
                cur = cv2.resize(cur, (lvl["width"], lvl["height"]), interpolation=cv2.INTER_LINEAR_EXACT)
            assert np.array_equal(im, cur)
            n = int(s["counts"][lv])
            sl = slice(lvl["offset"], lvl["offset"] + n)
            pad = cv2.copyMakeBorder(im, 32, 32, 32, 32, cv2.BORDER_REFLECT_101)
            kps = [cv2.KeyPoint(float(x) + 32, float(y) + 32, 31, 12.0 * float(b), 0.0, 0, i)
                   for i, ((x, y), b) in enumerate(zip(s["kp_level"][sl], s["bins"][sl]))]
            ok, dc = _orb().compute(pad, kps)
            cid = np.array([k.class_id for k in ok])
            assert len(cid) == n
            assert np.array_equal(s["desc"][sl][cid], dc), "level %d" % lv
    finally:
        ox.close()


def test_bin_zero_at_level_zero_is_the_reference_descriptor():
    import torch
    from xclean_b200 import _lib
    from xclean_b200.front.gpu_front import cpu_orb
    from xclean_b200.front.orb_ext import PAD, steered_patterns
    from xclean_b200.front.gpu_front import probe_orb_pattern
    L = _lib.lib()
    img = _frame("small", 8)
    H, W = img.shape
    kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
    g = torch.from_numpy(img).cuda()
    B = torch.empty((H + 2 * PAD, W + 2 * PAD), dtype=torch.uint8, device="cuda")
    kft = torch.from_numpy(kf).cuda()
    from xclean_b200.front.orb_ext import blur_split_points
    vr, vc = blur_split_points(W, H, kf)
    _lib.check(L.xcb_blur_dev(_v(g), W, H, _v(kft), vr, vc, _v(B), None), None, "xcb_blur_dev")
    rng = np.random.default_rng(3)
    kp = np.stack([rng.uniform(0, W - 1, 700), rng.uniform(0, H - 1, 700)], 1).astype(np.float32)
    pats = torch.from_numpy(steered_patterns(probe_orb_pattern())).cuda()
    bins = torch.zeros(len(kp), dtype=torch.int32, device="cuda")
    kpt = torch.from_numpy(kp).cuda()
    d = torch.zeros((len(kp), 32), dtype=torch.uint8, device="cuda")
    _lib.check(L.xcb_orb_steered_dev(_v(B), W + 2 * PAD, H + 2 * PAD, PAD, _v(kpt), len(kp), None, _v(bins), _v(pats),
                                     _v(d), None), None, "xcb_orb_steered_dev")
    assert np.array_equal(d.cpu().numpy(), cpu_orb(img, kp))


def test_detect_gpu_and_graph_replay_match_the_host_entry():
    import torch
    img0, img1 = _frame("small", 9), _frame("small", 10)
    H, W = img0.shape
    ox = _orbx(W, H, 4, 1.2, 2000)
    try:
        want0, want1 = ox.detect_slots(img0), ox.detect_slots(img1)
        static = torch.from_numpy(img0).cuda()
        ox.detect_gpu(static)
        _same_slots(ox.read(), want0, ox)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            ox.detect_gpu(static)                    # warm-up on the capture stream
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            ox.detect_gpu(static)
        static.copy_(torch.from_numpy(img1).cuda())
        g.replay()
        torch.cuda.synchronize()
        _same_slots(ox.read(), want1, ox)
        assert ox.launches() == 4 * 8 + 3
        del g
    finally:
        ox.close()


def test_errors():
    from xclean_b200.front.orb_ext import OrbPyramid
    with pytest.raises(RuntimeError):
        OrbPyramid(64, 48, levels=4, calibrate=False)          # level 1 smaller than 2 edge + 1
    with pytest.raises(RuntimeError):
        OrbPyramid(640, 480, levels=9, calibrate=False)
    ox = OrbPyramid(320, 240, levels=2, nfeatures=100, calibrate=False)
    try:
        with pytest.raises(RuntimeError):
            ox.detect(np.zeros((240, 320), np.uint8))           # not calibrated
        ox.calibrate()
        f = ox.detect(np.full((240, 320), 128, np.uint8))       # flat: no corners
        assert len(f.kp) == 0
        import torch
        with pytest.raises(ValueError):
            ox.detect_gpu(torch.zeros((240, 321), dtype=torch.uint8, device="cuda"))
    finally:
        ox.close()
