"""Generate the golden fixtures of the frontend from the REFERENCE's own CPU modules.

Run in a container that has the reference checkout (it is not needed anywhere else):
    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden.py <reference>/src

For each case the input images are stored losslessly (PNG bytes) together with the outputs of
    xclean.front.detect.Detector.__call__       (kp, desc; budget set explicitly, cell scope, noise floor)
    xclean.front.stereo1d.disparities            (d, sig, ok, zn, last_dy; HALF = 5, the reference's window)
    xclean.front.mapmatch_fast.match_desc        (i0, i1)
and the calibration of the cv2 build that produced them (SIMD split points, Gaussian taps, the noise quantile and the
hash of the ORB test-pair table).  The LK-solver fixture holds numba's np.linalg.solve / inv outputs on LK-shaped
systems.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_src):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    os.environ["CUDA_VISIBLE_DEVICES"] = "-1"
    sys.path.insert(0, ref_src)
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import cv2
    from xclean.front import gpu_front as RGF
    from xclean.front import mapmatch_fast as RMM
    from xclean.front import stereo1d as RS1
    from xclean.front.detect import Detector as RDetector
    from xclean.stages import features as RFE

    from oracle import front_oracle as O
    from xclean_b200 import synth
    from xclean_b200.front.gpu_front import probe_orb_pattern

    class Rig:
        def __init__(self, W, H):
            self.width, self.height = W, H

        def feature_budget(self):
            return 900

        def conditioning_floor(self):
            return 100

    RFE.noise_floor_8u(np.zeros((8, 8), np.uint8))
    Q = float(RFE._NOISE_Q99)
    kf = cv2.getGaussianKernel(7, 2, ktype=cv2.CV_32F).ravel().astype(np.float32)
    pat = probe_orb_pattern()
    ref_pat = RGF.probe_orb_pattern()
    assert np.array_equal(pat, ref_pat), "pattern probe disagrees with the reference's probe"

    def calibrate(W, H):
        """split points reproducing cv2 on the reference's calibration image (oracle restatement vs cv2)"""
        rng = np.random.default_rng(0)
        img = (rng.random((H, W)) * 255).astype(np.uint8)
        img = cv2.GaussianBlur(img, (0, 0), 1.0)
        img[: H // 8, : W // 8] = 77
        Rcv = cv2.cornerMinEigenVal(img, 3, 3)
        cands = sorted(set([W] + [(W // m) * m for m in (4, 8, 16, 32, 64, 128)] + [0]), reverse=True)
        found = None
        for dxv in (W,) + tuple(c for c in cands if c != W):
            for dyv in cands:
                if np.array_equal(O.response(img, dyv, dxv).view(np.uint32), Rcv.view(np.uint32)):
                    found = (dyv, dxv)
                    break
            if found:
                break
        pad = cv2.copyMakeBorder(img, 32, 32, 32, 32, cv2.BORDER_REFLECT_101)
        Bcv = cv2.sepFilter2D(pad, -1, kf, kf, borderType=cv2.BORDER_REFLECT_101)
        Wp = W + 64
        bc = sorted(set([Wp] + [(Wp // m) * m for m in (4, 8, 16, 32, 64, 128)] + [0]), reverse=True)
        fb = None
        for vr in bc:
            for vc in bc:
                if np.array_equal(O.blur(img, kf, vr, vc), Bcv):
                    fb = (vr, vc)
                    break
            if fb:
                break
        assert found and fb
        return dict(dy_vend=found[0], dx_vend=found[1], blur_vr=fb[0], blur_vc=fb[1])

    def png(a):
        ok, buf = cv2.imencode(".png", np.ascontiguousarray(a, np.uint8))
        assert ok
        return np.frombuffer(buf.tobytes(), np.uint8)

    def case(name, left0, right0, left1, budget, dhi, stereo_variants):
        H, W = left0.shape
        cal = calibrate(W, H)
        det = RDetector(Rig(W, H), cap=max(2048, budget))
        det.budget = budget
        kp0, desc0 = det(left0)
        floor0 = det.fe.stats.get("noise_floor_last", np.nan)
        kp1, desc1 = det(left1)
        floor1 = det.fe.stats.get("noise_floor_last", np.nan)
        out = dict(left0=png(left0), right0=png(right0), left1=png(left1), budget=np.int64(budget),
                   kp0=kp0, desc0=desc0, kp1=kp1, desc1=desc1, floor0=np.float64(floor0), floor1=np.float64(floor1))
        out.update({k: np.int64(v) for k, v in cal.items()})
        for tag, dlo, dhi_, dy, band in stereo_variants:
            kp = kp0.astype(np.float64)
            lo = None if dlo is None else np.full(len(kp), dlo, np.int64)
            hi = None if dhi_ is None else np.full(len(kp), dhi_, np.int64)
            d, s, ok, zn = RS1.disparities(left0, right0, kp, lo, hi, dy=dy, band=band)
            out["st_%s_d" % tag] = d
            out["st_%s_sig" % tag] = s
            out["st_%s_ok" % tag] = ok
            out["st_%s_zn" % tag] = zn
            out["st_%s_dy" % tag] = RS1.disparities.last_dy
            out["st_%s_args" % tag] = np.array([-1 if dlo is None else dlo, -1 if dhi_ is None else dhi_, band, dy])
        i0, i1 = RMM.match_desc({"descriptors": desc0}, {"descriptors": desc1})
        out["m_i0"], out["m_i1"] = i0, i1
        np.savez_compressed(os.path.join(HERE, "front_%s.npz" % name), **out)
        print(name, W, H, "kp", len(kp0), len(kp1), "matches", len(i0), "ok", int(out["st_a_ok"].sum()), cal)

    # 1. the reference's calibration-style image (random, blurred 1 px, flat grey-77 corner), small
    rng = np.random.default_rng(7)
    H, W = 120, 160
    a = cv2.GaussianBlur((rng.random((H, W)) * 255).astype(np.uint8), (0, 0), 1.0)
    a[: H // 8, : W // 8] = 77
    r = np.roll(a, -6, axis=1)
    b = cv2.GaussianBlur((np.clip(a.astype(int) + rng.integers(-3, 4, a.shape), 0, 255)).astype(np.uint8), (0, 0), 0.6)
    case("calib160", a, r, b, 150, None,
         [("a", None, None, 0.0, 0), ("b", 0, 40, 0.25, 1), ("c", 2, 30, -0.4, 2)])
    # 2. config-0 shape: 752x480, six planes, fx 458, B 0.11, sigma 2; second pair after 5 cm / 1 deg
    import math
    cam = synth.CAM_SMALL
    rd = synth.Renderer(synth.scene_planes(0, cam), cam)
    l0, r0 = rd.pair(np.eye(3), np.zeros(3), seed=0)
    l1, _ = rd.pair(synth.yaw(math.radians(1.0)), np.array([0.05, 0.0, 0.0]), seed=1)
    case("small752", l0.numpy(), r0.numpy(), l1.numpy(), 1000, 64,
         [("a", 0, 64, 0.0, 0), ("b", None, None, 0.3, 2)])
    # 3. config-1 shape: 1241x376 driving frames 0 and 1, 2000 features, disparities 0-96
    L, R = synth.sequence(synth.CAM_KITTI, 2, seed=1)
    case("kitti1241", L[0].numpy(), R[0].numpy(), L[1].numpy(), 2000, 96, [("a", 0, 96, 0.0, 0)])
    # LK solver fixture: numba's LAPACK on LK-shaped systems
    from xclean_b200.front.gpu_front import lk_test_systems
    As, gs = lk_test_systems(np.random.default_rng(11), 512)
    X = np.empty((512, 3))
    Inv = np.empty((512, 3, 3))
    RGF._nb_solve_inv()(As, gs, X, Inv)
    np.savez_compressed(os.path.join(HERE, "lk_solver.npz"), As=As, gs=gs, X=X, Inv=Inv)
    meta = dict(cv2_version=cv2.__version__, q99=Q, kf=kf, pattern_sha256=hashlib.sha256(pat.astype(np.int64).tobytes()).hexdigest())
    np.savez(os.path.join(HERE, "front_meta.npz"), **{k: np.asarray(v) for k, v in meta.items()})
    print("meta", meta["cv2_version"], Q)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    main(sys.argv[1])
