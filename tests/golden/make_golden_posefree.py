"""Generate tests/golden/posefree_golden.npz from the reference's pose-free landmark block (run once, where the
reference is).

    NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_posefree.py <reference>/src

For two seeded synthetic windows (xclean_b200.backend.synth_ba.make_window; the second with a non-identity extrinsic
and an inverse-depth prior) it adds a pose-free block (src/xclean/vio/window.py PoseFree: landmarks seen only in
their host's left image, with an inverse-depth prior on most of them and a few degenerate ones) and records the
reference's posefree_cost (behind False / True), posefree_step at lam = 1e-3 and 0 (outputs pre-filled with
sentinels), and the state and stats after solve(pb, iters=5, lam0=1e-4) with the block attached (the same block
without its NaN pixel, which would make every cost NaN).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "posefree_golden.npz")
FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")
CASES = ((6, 150, 31, False, 60), (10, 400, 32, True, 200))


def pose_free(rng, w, n, degenerate, nan_pixel=True):
    """n landmarks hosted by random slots, observed only in the host's left image (pixel noise 1 px, a few outliers),
    an inverse-depth prior (10 % relative noise) on 80 % of them."""
    P = w.Rwb.shape[0]
    host = rng.integers(0, P, n)
    u = rng.uniform(20, 730, n)
    v = rng.uniform(20, 460, n)
    depth = rng.uniform(2.0, 20.0, n)
    a, b, rho = (u - w.cx) / w.fx, (v - w.cy) / w.fy, 1.0 / depth
    z = np.stack([u, v], 1) + rng.normal(0, 1.0, (n, 2))
    z[rng.random(n) < 0.05] += rng.normal(0, 30.0, (1, 2))
    lmp = np.stack([a + rng.normal(0, 0.01, n), b + rng.normal(0, 0.01, n), rho * (1 + rng.normal(0, 0.1, n))], 1)
    rmeas = rho * (1 + rng.normal(0, 0.1, n))
    ris = np.where(rng.random(n) < 0.8, 1.0 / (0.1 * rho), 0.0)
    if degenerate:
        lmp[0, 2] = -0.05                 # behind the host: no observation term
        ris[0] = 0.0                      # and no prior: not solvable
        lmp[1, 2] = 1e-12                 # a step that would take rho <= 1e-9 is refused
        rmeas[1] = -1.0
        ris[1] = 1e6
        if nan_pixel:
            z[2] = np.nan                 # NaN pixel (the cost turns NaN: only the cost / step records have it)
        lmp[3] = [0.1, -0.1, 0.2]
        ris[3] = 0.0                      # rho unconstrained: singular block
    return dict(host=host.astype(np.int64), z=z, isg=1.0, rmeas=rmeas, ris=ris, lmp=lmp)


def main(src):
    sys.path.insert(0, src)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    from xclean.vio import window as Wn
    from xclean_b200.backend.synth_ba import make_window, so3_exp
    out = {}
    for ci, (K, L, seed, extr, npf) in enumerate(CASES):
        kw = dict(Rbc=so3_exp(np.array([0.02, -0.03, 0.01])), pbc=np.array([0.05, -0.02, 0.1]),
                  depth_prior=0.05) if extr else {}
        w = make_window(np.random.default_rng(seed), K=K, L=L, obs_min=2, obs_max=8, rng=np.random.default_rng(seed),
                        **kw)
        arrs = {k: np.ascontiguousarray(getattr(w, k)) for k in FIELDS}
        for k in ("lm_host", "ob_start", "ob_pose", "ob_cam"):
            arrs[k] = arrs[k].astype(np.int64)
        arrs["lm_mask"] = arrs["lm_mask"].astype(np.bool_)
        arrs["ob_valid"] = arrs["ob_valid"].astype(np.bool_)
        sc = {k: float(getattr(w, k)) for k in SCAL}
        pf = pose_free(np.random.default_rng(seed + 1000), w, npf, degenerate=True)
        for k, v in arrs.items():
            out["c%d_%s" % (ci, k)] = v.copy()
        out["c%d_scal" % ci] = np.array([sc[k] for k in SCAL])
        for k, v in pf.items():
            out["c%d_pf_%s" % (ci, k)] = np.asarray(v)
        g = (arrs["Rwb"], arrs["pwb"], arrs["Rbc"], arrs["pbc"])
        pfa = (pf["host"], pf["rmeas"], pf["ris"], pf["z"], pf["isg"])
        with np.errstate(all="ignore"):
            for behind in (False, True):
                c = Wn.posefree_cost(*g, pf["lmp"], *pfa, sc["fx"], sc["fy"], sc["cx"], sc["cy"], sc["B"],
                                     sc["huber_k"], behind)
                out["c%d_cost_%d" % (ci, int(behind))] = np.array([c])
            for tag, lam in (("d", 1e-3), ("u", 0.0)):
                lo = np.full((npf, 3), 7.0)
                Hi = np.full((npf, 3, 3), 5.0)
                ok = np.zeros(npf, np.bool_)
                Wn.posefree_step(*g, pf["lmp"], *pfa, sc["fx"], sc["fy"], sc["cx"], sc["cy"], sc["huber_k"], lam, lo,
                                 Hi, ok)
                out.update({"c%d_%s_lmp" % (ci, tag): lo, "c%d_%s_Hinv" % (ci, tag): Hi, "c%d_%s_ok" % (ci, tag): ok})
            pfs = pose_free(np.random.default_rng(seed + 1000), w, npf, degenerate=True, nan_pixel=False)
            for k, v in pfs.items():
                out["c%d_pfs_%s" % (ci, k)] = np.asarray(v)
            a = {k: v.copy() for k, v in arrs.items()}
            pb = Wn.Problem(**a, **sc)
            pb.pf = Wn.PoseFree(pfs["host"], pfs["z"], pfs["isg"], pfs["rmeas"], pfs["ris"], pfs["lmp"])
            st = Wn.solve(pb, iters=5, lam0=1e-4)
        out.update({"c%d_Rwb_n" % ci: pb.Rwb, "c%d_pwb_n" % ci: pb.pwb, "c%d_lmp_n" % ci: pb.lmp,
                    "c%d_pflmp_n" % ci: pb.pf.lmp,
                    "c%d_stats" % ci: np.array([st["cost0"], st["cost"], st["accepted"], st["lam"]])})
        print("case", ci, "slots", K, "landmarks", L, "pose-free", npf, "stats", st)
    np.savez_compressed(OUT, ncases=np.array(len(CASES)), **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    main(sys.argv[1])
