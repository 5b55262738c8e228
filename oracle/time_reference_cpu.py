"""Time the reference's own CPU implementation of the hot path (its numba / cv2 modules), single-threaded and as a
process pool over every host core (test and measurement infrastructure: it runs only where the reference checkout
is, and bench.py records its results rather than running it).

    NUMBA_CACHE_DIR=/tmp/nbcache python oracle/time_reference_cpu.py <the reference's src directory> [frames] [windows]

Frontend (the config of the headline: 1241x376 synthetic stereo frames, 2,000 features): per frame
    xclean.front.detect.Detector.__call__ (response, noise floor, cells, greedy, ORB: src/xclean/front/detect.py),
    xclean.front.stereo1d.disparities over the frame's keypoints, disparities 0-96 (its own ZNCC window),
    xclean.front.mapmatch_fast.match_desc against the previous frame's descriptors.
BA (config c2's uneven windows): xcb's synthetic windows through xclean.vio.window.solve (5 LM iterations).
Prints one JSON object: frames/s and windows/s, single process and pool, with the core count.
"""
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _setup(ref_src):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    os.environ["CUDA_VISIBLE_DEVICES"] = "-1"
    os.environ.setdefault("NUMBA_NUM_THREADS", "1")
    for p in (ref_src, ROOT):
        if p not in sys.path:
            sys.path.insert(0, p)


class _Rig:
    def __init__(self, W, H, budget):
        self.width, self.height, self.budget = W, H, budget

    def feature_budget(self):
        return self.budget

    def conditioning_floor(self):
        return 100


def _frames(n, seed=0):
    from xclean_b200 import synth
    L, R = synth.sequence(synth.CAM_KITTI, n, seed=seed)
    return L.numpy(), R.numpy()


def _front_worker(args):
    ref_src, L, R, budget = args
    _setup(ref_src)
    from xclean.front import mapmatch_fast as RMM
    from xclean.front import stereo1d as RS1
    from xclean.front.detect import Detector
    H, W = L.shape[1:]
    det = Detector(_Rig(W, H, budget), cap=max(2048, budget))
    det.budget = budget
    prev = None
    t0 = time.perf_counter()
    for i in range(len(L)):
        kp, desc = det(L[i])
        kpd = kp.astype(np.float64)
        RS1.disparities(L[i], R[i], kpd, np.zeros(len(kpd), np.int64), np.full(len(kpd), 96, np.int64))
        if prev is not None:
            RMM.match_desc({"descriptors": prev}, {"descriptors": desc})
        prev = desc
    return len(L), time.perf_counter() - t0


def _ba_worker(args):
    ref_src, wins = args
    _setup(ref_src)
    from xclean.vio import window as Wn
    t0 = time.perf_counter()
    for w in wins:
        Wn.solve(_problem(Wn, w), iters=5, lam0=1e-4)
    return len(wins), time.perf_counter() - t0


FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")


def _problem(Wn, w):
    a = {k: np.ascontiguousarray(getattr(w, k)).copy() for k in FIELDS}
    for k in ("lm_host", "ob_start", "ob_pose", "ob_cam"):
        a[k] = a[k].astype(np.int64)
    for k in ("lm_mask", "ob_valid"):
        a[k] = a[k].astype(np.bool_)
    return Wn.Problem(**a, **{k: float(getattr(w, k)) for k in SCAL})


def main(ref_src, n_frames=32, n_windows=64):
    _setup(ref_src)
    cores = os.cpu_count() or 1
    L, R = _frames(max(n_frames, 2 * cores))
    budget = 2000
    _front_worker((ref_src, L[:2], R[:2], budget))                  # numba compilation, cv2 warm-up
    n1, t1 = _front_worker((ref_src, L[:n_frames], R[:n_frames], budget))
    ctx = mp.get_context("spawn")
    chunks = np.array_split(np.arange(len(L)), cores)
    with ctx.Pool(cores) as pool:
        pool.map(_front_worker, [(ref_src, L[c[:2]], R[c[:2]], budget) for c in chunks if len(c)])  # warm-up
        t0 = time.perf_counter()
        res = pool.map(_front_worker, [(ref_src, L[c], R[c], budget) for c in chunks if len(c)])
        tp = time.perf_counter() - t0
    np_front = sum(r[0] for r in res)
    from xclean_b200.backend import synth_ba as S
    wins = S.config2_windows(256, seed=1)[:max(n_windows, cores)]
    _ba_worker((ref_src, wins[:2]))
    nb1, tb1 = _ba_worker((ref_src, wins[:min(16, len(wins))]))
    wchunks = [wins[i::cores] for i in range(cores)]
    with ctx.Pool(cores) as pool:
        pool.map(_ba_worker, [(ref_src, c[:1]) for c in wchunks if c])
        t0 = time.perf_counter()
        res = pool.map(_ba_worker, [(ref_src, c) for c in wchunks if c])
        tbp = time.perf_counter() - t0
    nb_pool = sum(r[0] for r in res)
    out = {"cores": cores,
           "frontend": {"workload": "1241x376 synthetic stereo frames, 2000 features, disparities 0-96 (stereo1d's own "
                                    "ZNCC window), matching to the previous frame",
                        "single_process_frames_per_s": n1 / t1,
                        "pool_frames_per_s": np_front / tp, "pool_frames": int(np_front)},
           "ba": {"workload": "config c2's uneven windows (K~U{5..20}, L~U{300..3000}), window.solve 5 LM iterations",
                  "single_process_windows_per_s": nb1 / tb1,
                  "pool_windows_per_s": nb_pool / tbp, "pool_windows": int(nb_pool)}}
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python %s <the reference's src directory> [frames] [windows]" % sys.argv[0])
    main(sys.argv[1], *(int(x) for x in sys.argv[2:4]))
