"""Generate the golden fixture of the gated map matcher from the REFERENCE's own CPU modules.

Run in a container that has the reference checkout (it is not needed anywhere else):
    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_mapmatch.py <reference>/src

Each case stores the inputs of MapMatcher(W, H).match(kp, desc, uv_pred, S_uv, lm_desc, lm_ndesc, chi2) and its
outputs (kp index per landmark, Hamming distance, Mahalanobis d2) from xclean.front.mapmatch.MapMatcher; the script
asserts that xclean.front.mapmatch_fast.MapMatcher returns the same arrays.  Keypoints and descriptors of the realistic
cases are the frontend fixtures' (front_<case>.npz: two consecutive frames and their matches); the landmarks are the
first frame's keypoints projected into the second frame with noise, with covariances drawn per landmark.

predict_golden.npz: xclean.vio.window.predict_projection on engine-shaped inputs (its outputs pre-filled as the
engine's _project fills them), then MapMatcher.match on the in-view landmarks, as the engine's tracking stage calls
them one after the other.
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


def _rot(rng, scale):
    w = rng.normal(0, scale, 3)
    th = np.linalg.norm(w)
    k = w / th if th > 0 else np.array([1.0, 0.0, 0.0])
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K


def predict_case(seed, L, zero_spose=False, sig_px=1.0, edges=False):
    """window.predict_projection inputs shaped as the engine's _project builds them (host cameras of a few keyframes
    along a forward path, inverse-depth landmarks, a predicted pose near the newest keyframe), then the map matcher
    on the in-view landmarks (keypoints near their projections plus clutter)."""
    rng = np.random.default_rng(seed)
    W, H, fx, fy, cx, cy = 1241, 376, 718.0, 718.0, 607.0, 185.0
    Rbc = np.array([[0.0, 0.0, 1.0], [-1.0, 0.0, 0.0], [0.0, -1.0, 0.0]]) @ _rot(rng, 0.01)   # camera z = body x
    pbc = np.array([0.3, -0.1, 0.05])
    nh = 8
    Rwb_h = [_rot(rng, 0.02) for _ in range(nh)]
    pwb_h = [np.array([1.0 * i, rng.normal(0, 0.05), rng.normal(0, 0.02)]) for i in range(nh)]
    if edges:
        Rwb_h[0] = Rwb_h[0] @ np.diag([-1.0, -1.0, 1.0])            # a host looking backwards: points behind
    host = rng.integers(0, nh, L)
    Rwc_h = np.stack([Rwb_h[h] @ Rbc for h in host])
    pwc_h = np.stack([pwb_h[h] + Rwb_h[h] @ pbc for h in host])
    lmp = np.stack([rng.uniform(-0.7, 0.7, L), rng.uniform(-0.22, 0.22, L), rng.uniform(0.03, 0.3, L)], 1)
    R_t = Rwb_h[-1] @ _rot(rng, 0.01)
    p_t = pwb_h[-1] + np.array([1.0, 0.0, 0.0]) + rng.normal(0, 0.02, 3)
    A = rng.normal(0, 0.05, (6, 6))
    Spose = np.zeros((6, 6)) if zero_spose else A @ A.T + np.diag([1e-4] * 3 + [1e-3] * 3)
    B = rng.normal(0, 0.03, (L, 3, 3))
    Sl = np.einsum("lij,lkj->lik", B, B)
    Sl[rng.random(L) < 0.1] = 0.0
    if edges:
        lmp[0, 2] = 0.0
        lmp[1, 2] = -0.1
        lmp[2, 2] = np.nan
        lmp[3, 0] = np.nan
        lmp[4, 2] = 1e-12
        Sl[5] = np.nan
        pwc_h[6] = np.inf
    uv = np.full((L, 2), np.nan)
    S = np.zeros((L, 2, 2))
    ok = np.zeros(L, np.bool_)
    depth = np.zeros(L)
    return dict(Rwb_t=R_t, pwb_t=p_t, Rbc=Rbc, pbc=pbc, Rwc_h=Rwc_h, pwc_h=pwc_h, lmp=lmp, Spose=Spose, Sl=Sl,
                sig_px=sig_px, fx=fx, fy=fy, cx=cx, cy=cy, W=float(W), H=float(H), uv0=uv, S0=S, ok0=ok, depth0=depth)


def predict_match_inputs(rng, c, uv, ok):
    """Keypoints near 70 % of the in-view projections (and 400 clutter points), their landmarks' descriptors."""
    L = len(uv)
    sel = np.nonzero(ok)[0]
    lmd = rng.integers(0, 256, (L, 3, 32), dtype=np.uint8)
    lnd = rng.integers(1, 4, L).astype(np.int64)
    seen = sel[rng.random(len(sel)) < 0.7]
    kp = np.concatenate([uv[seen] + rng.normal(0, 1.0, (len(seen), 2)),
                         np.stack([rng.uniform(0, c["W"], 400), rng.uniform(0, c["H"], 400)], 1)]).astype(np.float32)
    flips = np.packbits(rng.random((len(seen), 256)) < 0.05, axis=1)
    desc = np.concatenate([lmd[seen, 0] ^ flips, rng.integers(0, 256, (400, 32), dtype=np.uint8)])
    perm = rng.permutation(len(kp))
    return kp[perm], desc[perm], lmd, lnd


def make_predict(ref_src, RM):
    from xclean.vio import window as RW
    cases = {"kitti": predict_case(6, 1500), "track": predict_case(7, 900, zero_spose=True, sig_px=2.3),
             "edges": predict_case(8, 64, edges=True)}
    out = {}
    for ci, (name, c) in enumerate(cases.items()):
        uv, S, ok, depth = c["uv0"].copy(), c["S0"].copy(), c["ok0"].copy(), c["depth0"].copy()
        with np.errstate(all="ignore"):
            RW.predict_projection(c["Rwb_t"], c["pwb_t"], c["Rbc"], c["pbc"], c["Rwc_h"], c["pwc_h"], c["lmp"],
                                  c["Spose"], c["Sl"], c["sig_px"], c["fx"], c["fy"], c["cx"], c["cy"], c["W"],
                                  c["H"], uv, S, ok, depth)
        rng = np.random.default_rng(100 + ci)
        kp, desc, lmd, lnd = predict_match_inputs(rng, c, uv, ok)
        sel = np.nonzero(ok)[0]
        with np.errstate(all="ignore"):
            k, d, d2 = RM.MapMatcher(int(c["W"]), int(c["H"])).match(kp, desc, uv[sel], S[sel], lmd[sel], lnd[sel])
        c.update(uv=uv, S=S, ok=ok, depth=depth, kp=kp, desc=desc, lmd=lmd, lnd=lnd, sel=sel, m_kp=k, m_d=d, m_d2=d2)
        for key, v in c.items():
            out["%s__%s" % (name, key)] = np.asarray(v)
        print("predict", name, "landmarks", len(uv), "in view", len(sel), "matched", int((k >= 0).sum()))
    np.savez_compressed(os.path.join(HERE, "predict_golden.npz"), names=np.array(list(cases)), **out)


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
    make_predict(ref_src, RM)


if __name__ == "__main__":
    main(sys.argv[1])
