"""Generate tests/golden/window_golden.npz from the reference's stereo window solve (run once, where the reference is).

    NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_window.py <reference>/src

For three seeded synthetic windows (xclean_b200.backend.synth_ba.make_window: 5, 8 and 12 keyframes, stereo rows,
5 % outliers; the last two with a non-identity body-to-camera extrinsic and an inverse-depth prior) it records the
inputs (the fields of src/xclean/vio/window.py Problem), the reference's build_system outputs at lam = 1e-4 (H, b,
cost, Hll_inv, bl, Hlp, lm_ok) and the state and stats after its solve(pb, iters=5, lam0=1e-4) (no marginal prior,
no IMU, no pose-free block, no held slot).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "window_golden.npz")
FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")
CASES = ((5, 80, 11, False), (8, 300, 12, True), (12, 700, 13, True))


def main(src):
    sys.path.insert(0, src)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    from xclean.vio import window as Wn
    from xclean_b200.backend.synth_ba import make_window, so3_exp
    out = {}
    for ci, (K, L, seed, extr) in enumerate(CASES):
        kw = dict(Rbc=so3_exp(np.array([0.02, -0.03, 0.01])), pbc=np.array([0.05, -0.02, 0.1]),
                  depth_prior=0.05) if extr else {}
        w = make_window(np.random.default_rng(seed), K=K, L=L, obs_min=2, obs_max=8, rng=np.random.default_rng(seed),
                        **kw)
        arrs = {k: np.ascontiguousarray(getattr(w, k)) for k in FIELDS}
        arrs["lm_host"] = arrs["lm_host"].astype(np.int64)
        arrs["ob_start"] = arrs["ob_start"].astype(np.int64)
        arrs["ob_pose"] = arrs["ob_pose"].astype(np.int64)
        arrs["ob_cam"] = arrs["ob_cam"].astype(np.int64)
        arrs["lm_mask"] = arrs["lm_mask"].astype(np.bool_)
        arrs["ob_valid"] = arrs["ob_valid"].astype(np.bool_)
        sc = {k: float(getattr(w, k)) for k in SCAL}
        for k, v in arrs.items():
            out["c%d_%s" % (ci, k)] = v.copy()
        out["c%d_scal" % ci] = np.array([sc[k] for k in SCAL])
        P, Lh, M = arrs["Rwb"].shape[0], arrs["lmp"].shape[0], arrs["ob_pose"].shape[0]
        H = np.zeros((6 * P, 6 * P))
        b = np.zeros(6 * P)
        Hi = np.zeros((Lh, 3, 3))
        bl = np.zeros((Lh, 3))
        Hlp = np.zeros((Lh, P, 3, 6))
        ok = np.zeros(Lh, np.bool_)
        chi = np.zeros(M)
        a = {k: v.copy() for k, v in arrs.items()}
        cost = Wn.build_system(a["Rwb"], a["pwb"], a["Rbc"], a["pbc"], a["lmp"], a["lm_host"], a["lm_mask"],
                               a["rho_meas"], a["rho_isig"], a["ob_start"], a["ob_pose"], a["ob_cam"], a["ob_z"],
                               a["ob_isig"], a["ob_valid"], sc["fx"], sc["fy"], sc["cx"], sc["cy"], sc["B"],
                               sc["huber_k"], 1e-4, H, b, Hi, bl, Hlp, ok, chi)
        out.update({"c%d_H" % ci: H, "c%d_b" % ci: b, "c%d_cost" % ci: np.array([cost]), "c%d_Hi" % ci: Hi,
                    "c%d_bl" % ci: bl, "c%d_Hlp" % ci: Hlp, "c%d_ok" % ci: ok})
        a = {k: v.copy() for k, v in arrs.items()}
        pb = Wn.Problem(**a, **sc)
        st = Wn.solve(pb, iters=5, lam0=1e-4)
        out.update({"c%d_Rwb_n" % ci: pb.Rwb, "c%d_pwb_n" % ci: pb.pwb, "c%d_lmp_n" % ci: pb.lmp,
                    "c%d_stats" % ci: np.array([st["cost0"], st["cost"], st["accepted"], st["lam"]])})
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    main(sys.argv[1])
