"""Device frontend (libxcb200.so through the C ABI) against the reference's golden outputs and the CPU oracle.

Bit-exact throughout: keypoints, descriptors, noise floor, disparities / sigmas / flags / ZNCC / dy, Hamming
distances and match indices."""
import numpy as np
import pytest

from oracle import front_oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=G.CASES)
def setup(request):
    from xclean_b200.front.gpu_front import GpuFront
    c = G.load_case(request.param)
    H, W = c["left0"].shape
    gf = GpuFront(W, H, cap=max(2048, int(c["budget"])), max_frames=4)
    gf.set_calibration(G.calib_of(c), G.pattern())
    yield request.param, c, gf
    gf.close()


def test_response_bitexact(setup):
    name, c, gf = setup
    cal = G.calib_of(c)
    Rd = gf.response(c["left0"])
    Ro = O.response(c["left0"], cal["dy_vend"], cal["dx_vend"])
    assert G.same_bits(Rd, Ro), name


def test_detect_bitexact(setup):
    from xclean_b200.front.features import Frontend
    name, c, gf = setup
    fe = Frontend()
    for img, kp_ref, desc_ref, fl in ((c["left0"], c["kp0"], c["desc0"], c["floor0"]),
                                      (c["left1"], c["kp1"], c["desc1"], c["floor1"])):
        kp, desc = gf.detect(img, int(c["budget"]), fe)
        assert G.same_bits(kp, kp_ref), name
        assert np.array_equal(desc, desc_ref), name
        assert fe.stats["noise_floor_last"] == float(fl)


def test_detect_batch_equals_single(setup):
    name, c, gf = setup
    imgs = np.stack([c["left0"], c["left1"], c["left0"]])
    counts, kp, desc, floor, anypos = gf.detect_batch(imgs, int(c["budget"]))
    assert counts[0] == len(c["kp0"]) and counts[1] == len(c["kp1"]) and counts[2] == counts[0]
    assert G.same_bits(kp[1, :counts[1]], c["kp1"])
    assert np.array_equal(desc[2, :counts[2]], c["desc0"])


def test_stereo_bitexact_reference_window(setup):
    name, c, gf = setup
    kp = c["kp0"].astype(np.float64)
    for tag, dlo, dhi, dy, band in G.stereo_variants(c):
        lo = np.full(len(kp), 0 if dlo is None else dlo, np.int64)
        hi = np.full(len(kp), 127 if dhi is None else dhi, np.int64)
        d, s, ok, zn, ody = gf.stereo(c["left0"], c["right0"], kp, lo, hi, dy=dy, band=band, half=5)
        assert G.same_bits(d, c["st_%s_d" % tag]), (name, tag)
        assert G.same_bits(s, c["st_%s_sig" % tag]), (name, tag)
        assert np.array_equal(ok, c["st_%s_ok" % tag]), (name, tag)
        assert G.same_bits(zn, c["st_%s_zn" % tag]), (name, tag)
        assert G.same_bits(np.nan_to_num(ody + dy, nan=-1e300), np.nan_to_num(c["st_%s_dy" % tag], nan=-1e300))


@pytest.mark.parametrize("half", [3, 4])
def test_stereo_small_windows_vs_oracle(setup, half):
    """7x7 / 9x9 windows: the reference has only 11x11, so the oracle (the same algorithm, HALF as a parameter) is
    the checker."""
    name, c, gf = setup
    kp = c["kp0"].astype(np.float64)
    for dy, band in ((0.0, 0), (0.25, 1)):
        lo = np.zeros(len(kp), np.int64)
        hi = np.full(len(kp), 96, np.int64)
        d, s, ok, zn, ody = gf.stereo(c["left0"], c["right0"], kp, lo, hi, dy=dy, band=band, half=half)
        od, osg, ook, ozn, oody = O.stereo(c["left0"], c["right0"], kp, lo, hi, dy=dy, band=band, half=half)
        assert G.same_bits(d, od) and G.same_bits(s, osg) and np.array_equal(ok, ook) and G.same_bits(zn, ozn)
        assert G.same_bits(np.nan_to_num(ody + dy, nan=-1e300), np.nan_to_num(oody, nan=-1e300))


def test_hamming_and_match(setup):
    name, c, gf = setup
    b1, b2, bi, ci = gf.hamming(c["desc0"], c["desc1"])
    o1, o2, oi, oci = O.hamming(c["desc0"], c["desc1"])
    assert np.array_equal(b1, o1) and np.array_equal(b2, o2) and np.array_equal(bi, oi) and np.array_equal(ci, oci)
    i0, i1 = gf.match(c["desc0"], c["desc1"])
    assert np.array_equal(i0, c["m_i0"]) and np.array_equal(i1, c["m_i1"]), name


@pytest.mark.parametrize("L,N", [(1, 1), (1, 9), (7, 1), (17, 130), (129, 257), (300, 1025), (5000, 2049)])
def test_hamming_ties_and_ragged_sizes(L, N):
    """Distances drawn from a few repeated descriptors (many exact ties, between and within rows), sizes that are not
    multiples of the device tiles: best / second / first index and the column first index equal the CPU scan."""
    from xclean_b200.front.gpu_front import GpuFront
    rng = np.random.default_rng(L * 7919 + N)
    pool = rng.integers(0, 256, (6, 32), dtype=np.uint8)
    pool[1] = pool[0]
    pool[2, :4] ^= 1                                      # near-duplicates: distances 0..few
    A = np.where(rng.random((L, 1)) < 0.5, pool[rng.integers(0, 6, L)], rng.integers(0, 256, (L, 32), dtype=np.uint8))
    B = np.where(rng.random((N, 1)) < 0.5, pool[rng.integers(0, 6, N)], rng.integers(0, 256, (N, 32), dtype=np.uint8))
    gf = GpuFront(64, 64, cap=4096, max_frames=1)
    try:
        got = gf.hamming(A.astype(np.uint8), B.astype(np.uint8))
    finally:
        gf.close()
    ref = O.hamming(A.astype(np.uint8), B.astype(np.uint8))
    for g, r, nm in zip(got, ref, ("best", "second", "index", "column index")):
        assert np.array_equal(g, r), nm


def test_lk_solver_bitexact():
    from xclean_b200.front.gpu_front import GpuFront
    z = np.load(G.GOLDEN + "/lk_solver.npz")
    gf = GpuFront(160, 120, cap=256)
    X, Inv = gf.lk_solve_inv(z["As"], z["gs"])
    gf.close()
    assert G.same_bits(X, z["X"]) and G.same_bits(Inv, z["Inv"])


def test_pipeline_batched_vs_oracle():
    """The graph-replayed batched path (detect + ORB + 9x9 stereo + match to the previous frame) on four 1241x376
    frames equals the oracle's per-frame path."""
    from xclean_b200 import synth
    from xclean_b200.front.gpu_front import GpuFront
    c = G.load_case("kitti1241")
    cal = G.calib_of(c)
    pat = G.pattern()
    L, R = synth.sequence(synth.CAM_KITTI, 4, seed=3)
    L, R = L.numpy(), R.numpy()
    gf = GpuFront(1241, 376, cap=2048, max_frames=4)
    gf.set_calibration(cal, pat)
    out = gf.pipeline(L, R, 2000, half=4, dlo=0, dhi=96, match_prev=False)
    ref = O.frames(L, R, 2000, cal["q99"], cal, pat, half=4, dlo=0, dhi=96, cap=2048)
    assert np.array_equal(out["counts"], ref["counts"])
    for f in range(4):
        n = int(ref["counts"][f])
        assert G.same_bits(out["kp"][f, :n], ref["kp"][f, :n])
        assert np.array_equal(out["desc"][f, :n], ref["desc"][f, :n])
        for k in ("d", "sig", "zn"):
            assert G.same_bits(out[k][f, :n], ref[k][f, :n]), (f, k)
        assert np.array_equal(out["ok"][f, :n], ref["ok"][f, :n])
        assert G.same_bits(np.nan_to_num(out["dy"][f, :n], nan=-1e300), np.nan_to_num(ref["dy"][f, :n], nan=-1e300))
        m = int(ref["nmatch"][f])
        assert out["nmatch"][f] == m, f
        assert np.array_equal(out["m0"][f, :m], ref["m0"][f, :m]) and np.array_equal(out["m1"][f, :m], ref["m1"][f, :m])
    # a second call carries the last frame's descriptors: frame 0 now matches against the previous call's frame 3
    out2 = gf.pipeline(L, R, 2000, half=4, dlo=0, dhi=96, match_prev=True)
    q, t = O.match_desc(ref["desc"][3, :ref["counts"][3]], ref["desc"][0, :ref["counts"][0]])
    assert out2["nmatch"][0] == len(q) and np.array_equal(out2["m0"][0, :len(q)], q)
    gf.close()


def test_pipeline_batches_equals_consecutive_calls():
    """One call over 7 frames in batches of 3 (inputs copied on a second stream into a second buffer pair while the
    previous batch computes) gives the results of three consecutive pipeline() calls, bit for bit, including the
    matches across batch boundaries."""
    import torch
    from xclean_b200 import synth
    from xclean_b200.front.gpu_front import GpuFront
    c = G.load_case("kitti1241")
    L, R = synth.sequence(synth.CAM_KITTI, 7, seed=11)
    L = L.numpy().copy()
    R = R.numpy().copy()
    Lp = torch.from_numpy(L).pin_memory().numpy()
    Rp = torch.from_numpy(R).pin_memory().numpy()
    fronts = []
    for _ in range(2):
        gf = GpuFront(1241, 376, cap=2048, max_frames=3)
        gf.set_calibration(G.calib_of(c), G.pattern())
        fronts.append(gf)
    try:
        got = fronts[0].pipeline_batches(Lp, Rp, 2000, batch=3, half=4, dlo=0, dhi=96, match_prev=False)
        parts = [fronts[1].pipeline(L[a:a + 3], R[a:a + 3], 2000, half=4, dlo=0, dhi=96, match_prev=a > 0)
                 for a in (0, 3, 6)]
        want = {k: np.concatenate([p[k] for p in parts]) for k in got}
        for k in ("counts", "nmatch", "floor", "anypos"):
            assert np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)), k
        for f in range(7):                       # per-keypoint rows past a frame's count are not written
            n, m = int(want["counts"][f]), int(want["nmatch"][f])
            for k in ("kp", "desc", "d", "sig", "ok", "zn", "dy"):
                assert np.array_equal(got[k][f, :n].view(np.uint8), want[k][f, :n].view(np.uint8)), (f, k)
            for k in ("m0", "m1"):
                assert np.array_equal(got[k][f, :m], want[k][f, :m]), (f, k)
        assert (want["nmatch"][3] > 0) and (want["nmatch"][6] > 0)        # matches across the batch boundaries
    finally:
        for gf in fronts:
            gf.close()


def test_errors_and_edges():
    from xclean_b200.front.gpu_front import GpuFront
    c = G.load_case("calib160")
    gf = GpuFront(160, 120, cap=256, max_frames=2)
    with pytest.raises(RuntimeError):
        gf.detect_batch(c["left0"][None], 100)          # not calibrated
    gf.set_calibration(G.calib_of(c), G.pattern())
    with pytest.raises(ValueError):
        gf.detect_batch(c["left0"][None], 1000)         # budget > cap
    flat = np.full((120, 160), 77, np.uint8)
    counts, kp, desc, floor, anypos = gf.detect_batch(flat[None], 100)
    assert counts[0] == 0 and anypos[0] == 0
    d, s, ok, zn, ody = gf.stereo(flat, flat, np.zeros((0, 2)), np.zeros(0, np.int64), np.zeros(0, np.int64))
    assert len(d) == 0
    kp = np.array([[-8.0, -8.0], [5.0, 5.0], [80.0, 60.0]])
    d, s, ok, zn, ody = gf.stereo(flat, flat, kp, np.zeros(3, np.int64), np.full(3, 127, np.int64))
    assert not ok.any() and (zn == -2.0).all()
    with pytest.raises(RuntimeError):
        gf.stereo(flat, flat, kp, np.zeros(3, np.int64), np.full(3, 127, np.int64), band=17)
    i0, i1 = gf.match(c["desc0"][:1], c["desc1"])
    assert len(i0) == 0
    gf.close()


def test_calibrate_against_this_machines_cv2():
    """The start-up self-check (the reference's GpuFront.calibrate + check_lk_solver) passes against the cv2 / numba
    of the machine the test runs on."""
    from xclean_b200.front.gpu_front import GpuFront
    gf = GpuFront(752, 480, cap=2048)
    cal = gf.calibrate(cache=False)
    assert cal["noise_floor_equal"] and cal["orb_equal_random"] == 1500
    gf.close()


@pytest.mark.parametrize("warps,group", [(1, 1), (4, 8), (6, 16), (8, 32)])
def test_stereo_launch_shapes_give_identical_results(warps, group):
    """The tuner's stereo knobs (warps per block, points per warp) change only the time: the pipeline's outputs stay
    bit-identical to the oracle's for every shape."""
    from xclean_b200 import _lib, synth
    from xclean_b200.front.gpu_front import GpuFront
    c = G.load_case("kitti1241")
    cal = G.calib_of(c)
    L, R = synth.sequence(synth.CAM_KITTI, 2, seed=5)
    L, R = L.numpy(), R.numpy()
    gf = GpuFront(1241, 376, cap=2048, max_frames=2)
    try:
        gf.set_calibration(cal, G.pattern())
        gf.set_tuning(_lib.XCB_TUNE_STEREO_WARPS, warps)
        gf.set_tuning(_lib.XCB_TUNE_STEREO_GROUP, group)
        out = gf.pipeline(L, R, 2000, half=4, dlo=0, dhi=96, match_prev=False)
        ref = O.frames(L, R, 2000, cal["q99"], cal, G.pattern(), half=4, dlo=0, dhi=96, cap=2048)
        for f in range(2):
            n = int(ref["counts"][f])
            for k in ("d", "sig", "zn"):
                assert G.same_bits(out[k][f, :n], ref[k][f, :n]), (f, k)
            assert np.array_equal(out["ok"][f, :n], ref["ok"][f, :n])
            assert G.same_bits(np.nan_to_num(out["dy"][f, :n], nan=-1e300),
                               np.nan_to_num(ref["dy"][f, :n], nan=-1e300))
        kp = c["kp0"].astype(np.float64)
        lo, hi = np.zeros(len(kp), np.int64), np.full(len(kp), 127, np.int64)
        d, s, ok, zn, ody = gf.stereo(c["left0"], c["right0"], kp, lo, hi, dy=0.25, band=2, half=5)
        od, osg, ook, ozn, oody = O.stereo(c["left0"], c["right0"], kp, lo, hi, dy=0.25, band=2, half=5)
        assert G.same_bits(d, od) and G.same_bits(s, osg) and np.array_equal(ok, ook) and G.same_bits(zn, ozn)
        with pytest.raises(RuntimeError):
            gf.set_tuning(_lib.XCB_TUNE_STEREO_GROUP, 33)
    finally:
        gf.close()
