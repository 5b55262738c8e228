"""Generate the golden fixture of the gated map matcher from the REFERENCE's own CPU modules.

Run in a container that has the reference checkout (it is not needed anywhere else):
    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_mapmatch.py <reference>/src

Each case stores the inputs of MapMatcher(W, H).match(kp, desc, uv_pred, S_uv, lm_desc, lm_ndesc, chi2) and its
outputs (kp index per landmark, Hamming distance, Mahalanobis d2) from xclean.front.mapmatch.MapMatcher; the script
asserts that xclean.front.mapmatch_fast.MapMatcher returns the same arrays.  Keypoints and descriptors of the realistic
cases are the frontend fixtures' (front_<case>.npz: two consecutive frames and their matches); the landmarks are the
first frame's keypoints projected into the second frame with noise, with covariances drawn per landmark.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _spd(rng, L, lo=0.8, hi=4.0):
    sx = rng.uniform(lo, hi, L)
    sy = rng.uniform(lo, hi, L)
    rho = rng.uniform(-0.5, 0.5, L)
    S = np.empty((L, 2, 2))
    S[:, 0, 0] = sx * sx
    S[:, 1, 1] = sy * sy
    S[:, 0, 1] = S[:, 1, 0] = rho * sx * sy
    return S


def _flip(rng, desc, nbits):
    out = desc.copy()
    bits = np.unpackbits(out, axis=1)
    for i in range(len(out)):
        idx = rng.choice(256, int(nbits[i]), replace=False)
        bits[i, idx] ^= 1
    return np.packbits(bits, axis=1)


def realistic(name, W, H, seed, infl=1.0, nlm=None):
    z = np.load(os.path.join(HERE, "front_%s.npz" % name))
    rng = np.random.default_rng(seed)
    kp0, desc0, kp1, desc1 = z["kp0"], z["desc0"], z["kp1"], z["desc1"]
    i0, i1 = z["m_i0"], z["m_i1"]
    L = len(kp0)
    flow = np.median(kp1[i1] - kp0[i0], axis=0) if len(i0) else np.zeros(2)
    uv = kp0.astype(np.float64) + flow + rng.normal(0, 3.0, (L, 2))
    uv[i0] = kp1[i1].astype(np.float64) + rng.normal(0, 0.7, (len(i0), 2))
    S = _spd(rng, L) * infl
    lmd = np.zeros((L, 3, 32), np.uint8)
    lmd[:, 0] = desc0
    lmd[:, 1] = _flip(rng, desc0, rng.integers(0, 24, L))
    lmd[:, 2] = rng.integers(0, 256, (L, 32), dtype=np.uint8)
    lnd = rng.integers(1, 4, L).astype(np.int64)
    uv[rng.random(L) < 0.02] += np.array([W, 0.0])          # a few projected outside the image
    n = L if nlm is None else nlm
    return dict(W=W, H=H, chi2=13.815510557964274, kp=kp1, desc=desc1, uv=uv[:n], S=S[:n], lmd=lmd[:n], lnd=lnd[:n])


def edges(seed):
    """Degenerate inputs: keypoints outside the image, NaN / inf / huge coordinates, duplicated keypoints and
    descriptors, landmarks with NaN / inf predictions, singular, indefinite, negative-definite, NaN, inf and huge
    covariances, no descriptors, fewer descriptors than slots."""
    rng = np.random.default_rng(seed)
    W, H = 160, 120
    pool = rng.integers(0, 256, (5, 32), dtype=np.uint8)
    N = 64
    kp = np.stack([rng.uniform(-20, 180, N), rng.uniform(-20, 140, N)], 1)
    kp[:8] = np.round(kp[:8])
    kp[8:12] = kp[0:4]                                    # duplicated positions
    kp[12] = [np.nan, 3.0]
    kp[13] = [4.0, np.inf]
    kp[14] = [1e300, 50.0]
    kp[15] = [-0.0, 7.0]
    kp[16] = [6.0, np.nan]
    kp[17] = [-np.inf, 9.0]
    desc = pool[rng.integers(0, 5, N)]
    desc[8:12] = desc[0:4]
    U = rng.integers(0, 256, (4, 32), dtype=np.uint8)     # unique descriptors on the non-finite keypoints
    desc[[12, 16, 17, 13]] = U                            # NaN x, NaN y, -inf x, inf y: NaN Mahalanobis distances
    L = 96
    uv = kp[rng.integers(0, N, L)] + rng.normal(0, 1.0, (L, 2))
    uv[:12] = kp[:12] + rng.normal(0, 0.5, (12, 2))
    uv[12:20] = [[5.0, 5.0], [10.0, 8.0], [3.0, 12.0], [14.0, 2.0], [1.0, 1.0], [6.0, 6.0], [12.0, 12.0], [2.0, 9.0]]
    S = _spd(rng, L, 1.0, 12.0)
    S[12:20] = np.eye(2) * 400.0                          # wide gates around the corner cell (NaN d2 candidates)
    lmd = pool[rng.integers(0, 5, (L, 3))]
    lmd[12:20, 0] = desc[[12, 16, 17, 13, 12, 16, 0, 1]]   # two claimants each of keypoints 12 and 16
    lnd = rng.integers(1, 4, L).astype(np.int64)
    lnd[12:20] = 1
    uv[20] = [np.nan, 30.0]
    uv[21] = [40.0, np.inf]
    S[22] = [[4.0, 4.0], [4.0, 4.0]]                      # singular
    S[23] = [[4.0, 9.0], [9.0, 4.0]]                      # indefinite
    S[24] = [[-4.0, 0.5], [0.5, -9.0]]                    # negative definite: det > 0, half-widths 0
    S[25] = [[np.nan, 0.0], [0.0, 4.0]]
    S[26] = [[np.inf, 0.0], [0.0, 4.0]]
    S[27] = [[4.0, 0.0], [0.0, np.inf]]
    S[28] = [[1e200, 0.0], [0.0, 1e200]]
    S[29] = [[1e-300, 0.0], [0.0, 1e-300]]
    lnd[30] = 0
    lnd[31:34] = 1
    uv[34] = [1e300, 1e300]
    uv[35] = [-1e300, 50.0]
    uv[36:40] = uv[32]                                    # identical landmarks: the mutual step keeps the first
    S[36:40] = S[32]
    lmd[36:40] = lmd[32]
    lnd[36:40] = lnd[32]
    return dict(W=W, H=H, chi2=13.815510557964274, kp=kp, desc=desc, uv=uv, S=S, lmd=lmd, lnd=lnd)


def ties(seed):
    """Every distance and Mahalanobis tie the visit order decides: a lattice of keypoints with four descriptors,
    symmetric pairs around each landmark, landmarks sharing predictions and descriptors."""
    rng = np.random.default_rng(seed)
    W, H = 320, 240
    pool = rng.integers(0, 256, (4, 32), dtype=np.uint8)
    xs, ys = np.meshgrid(np.arange(4.0, W, 8.0), np.arange(4.0, H, 8.0))
    kp = np.stack([xs.ravel(), ys.ravel()], 1)
    N = len(kp)
    desc = pool[(np.arange(N) // 3) % 4]
    L = 600
    c = kp[rng.integers(0, N, L)]
    uv = c + np.array([4.0, 0.0]) * rng.integers(0, 2, (L, 1))   # on a keypoint or half-way between two
    S = np.tile(np.eye(2) * rng.choice([4.0, 16.0, 64.0], L)[:, None, None], 1)
    lmd = pool[rng.integers(0, 4, (L, 2))]
    lnd = rng.integers(1, 3, L).astype(np.int64)
    uv[100:200] = uv[:100]
    lmd[100:200] = lmd[:100]
    S[100:200] = S[:100]
    lnd[100:200] = lnd[:100]
    return dict(W=W, H=H, chi2=13.815510557964274, kp=kp, desc=desc, uv=uv, S=S, lmd=lmd, lnd=lnd)


def main(ref_src):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    sys.path.insert(0, ref_src)
    from xclean.front import mapmatch as RM
    from xclean.front import mapmatch_fast as RMF

    cases = {
        "kitti1241": realistic("kitti1241", 1241, 376, 1),
        "kitti1241_infl": realistic("kitti1241", 1241, 376, 2, infl=6.0, nlm=500),
        "small752": realistic("small752", 752, 480, 3),
        "edges": edges(4),
        "ties": ties(5),
    }
    cases["ties_chi2"] = dict(cases["ties"], chi2=2.0)
    out = {}
    for name, c in cases.items():
        args = (c["kp"], c["desc"], c["uv"], c["S"], c["lmd"], c["lnd"])
        with np.errstate(all="ignore"):
            a = RM.MapMatcher(c["W"], c["H"]).match(*args, chi2=c["chi2"])
            b = RMF.MapMatcher(c["W"], c["H"]).match(*args, chi2=c["chi2"])
        for x, y in zip(a, b):
            assert np.array_equal(x, y, equal_nan=True), name
        for k, v in c.items():
            out["%s__%s" % (name, k)] = np.asarray(v)
        out["%s__out_kp" % name], out["%s__out_d" % name], out["%s__out_d2" % name] = a
        print(name, "landmarks", len(c["uv"]), "keypoints", len(c["kp"]), "matched", int((a[0] >= 0).sum()))
    np.savez_compressed(os.path.join(HERE, "mapmatch_golden.npz"), names=np.array(list(cases)), **out)


if __name__ == "__main__":
    main(sys.argv[1])
