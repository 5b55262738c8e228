"""Generate tests/golden/prior_golden.npz from the reference's marginal prior and its window solve (run once, where the
reference is).

    NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_prior.py <reference>/src

Two seeded synthetic windows (xclean_b200.backend.synth_ba.make_window, non-identity body-to-camera extrinsic,
inverse-depth prior, 5 % outliers).  For each, with the reference's own functions (src/xclean/vio/marg.py,
src/xclean/vio/window.py):
  * the window is solved (10 LM iterations), marg_system(pb, landmarks hosted by slot 0) gives (H, b), schur()
    eliminates slot 0, combine() makes a prior over the other slots (no old prior), and a gauge_prior on slot 1 is
    combined in through its information;
  * the algebra on that prior: drop_slot of its first block, combine with the prior as the old one at a moved state,
    cost / terms at the moved state;
  * the window again from its perturbed initial state with the prior attached (bound to its slots), solved by
    window.solve(pb, iters=5, lam0=1e-4), and final_linearisation at the solution (H, b with the prior).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "prior_golden.npz")
FIELDS = ("Rwb", "pwb", "Rbc", "pbc", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose",
          "ob_cam", "ob_z", "ob_isig", "ob_valid")
SCAL = ("fx", "fy", "cx", "cy", "B", "huber_k")
CASES = ((6, 200, 21), (9, 400, 22))


def _arrays(w):
    a = {k: np.ascontiguousarray(getattr(w, k)).copy() for k in FIELDS}
    for k in ("lm_host", "ob_start", "ob_pose", "ob_cam"):
        a[k] = a[k].astype(np.int64)
    a["lm_mask"] = a["lm_mask"].astype(np.bool_)
    a["ob_valid"] = a["ob_valid"].astype(np.bool_)
    return a


def _save_prior(out, tag, pr):
    out[tag + "_sids"] = np.array(pr.sids, np.int64)
    out[tag + "_S"] = pr.S.copy()
    out[tag + "_r"] = pr.r.copy()
    out[tag + "_R0"] = np.stack([x[0] for x in pr.x0])
    out[tag + "_p0"] = np.stack([x[1] for x in pr.x0])


def main(src):
    sys.path.insert(0, src)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    from xclean.vio import marg as M
    from xclean.vio import window as Wn
    from xclean_b200.backend.synth_ba import make_window, so3_exp
    out = {}
    for ci, (K, L, seed) in enumerate(CASES):
        kw = dict(Rbc=so3_exp(np.array([0.02, -0.03, 0.01])), pbc=np.array([0.05, -0.02, 0.1]), depth_prior=0.05)
        w = make_window(np.random.default_rng(seed), K=K, L=L, obs_min=2, obs_max=8, rng=np.random.default_rng(seed),
                        **kw)
        arrs = _arrays(w)
        sc = {k: float(getattr(w, k)) for k in SCAL}
        for k, v in arrs.items():
            out["c%d_%s" % (ci, k)] = v.copy()
        out["c%d_scal" % ci] = np.array([sc[k] for k in SCAL])
        # the prior: marginalise slot 0 (and its landmarks) out of the solved window
        a = {k: v.copy() for k, v in arrs.items()}
        pb = Wn.Problem(**a, **sc)
        Wn.solve(pb, iters=10, lam0=1e-4)
        mask = (a["lm_host"] == 0) & a["lm_mask"]
        H, b, off = Wn.marg_system(pb, mask)
        keep = np.arange(6, 6 * K)
        H2, b2 = M.schur(H, b, keep, np.arange(6))
        sids = list(range(1, K))
        st = [(pb.Rwb[s], pb.pwb[s], None, None, None) for s in sids]
        pr = M.combine(None, sids, [6] * len(sids), st, H2, b2)
        g = M.gauge_prior(1, pb.Rwb[1], pb.pwb[1], info=1e8)
        Hg, bg = g.info()
        Hc, bc = pr.info()
        Hc[:6, :6] += Hg
        bc[:6] += bg
        pr = M.Prior.from_info(pr.sids, pr.dims, pr.x0, Hc, bc)
        out["c%d_marg_H" % ci], out["c%d_marg_b" % ci] = H, b
        out["c%d_schur_H" % ci], out["c%d_schur_b" % ci] = H2, b2
        out["c%d_solved_Rwb" % ci], out["c%d_solved_pwb" % ci] = pb.Rwb.copy(), pb.pwb.copy()
        _save_prior(out, "c%d_prior" % ci, pr)
        # algebra at a moved state
        rng = np.random.default_rng(100 + ci)
        Rm = np.stack([pb.Rwb[s] @ so3_exp(rng.normal(0, 0.01, 3)) for s in range(K)])
        pm = pb.pwb + rng.normal(0, 0.02, (K, 3))
        out["c%d_moved_Rwb" % ci], out["c%d_moved_pwb" % ci] = Rm, pm
        pr.bind({s: s for s in range(K)})
        Ht, bt, ct = pr.terms((Rm, pm, None, None, None), 6 * K)
        out["c%d_terms_H" % ci], out["c%d_terms_b" % ci] = Ht, bt
        out["c%d_terms_cost" % ci] = np.array([ct, pr.cost((Rm, pm, None, None, None))])
        dr = pr.drop_slot(sids[0])
        _save_prior(out, "c%d_drop" % ci, dr)
        Hn = Hc + np.diag(np.linspace(1.0, 2.0, Hc.shape[0]))
        cb = M.combine(pr, sids, [6] * len(sids), [(Rm[s], pm[s], None, None, None) for s in sids], Hn, bc)
        out["c%d_combine_H" % ci] = Hn
        out["c%d_combine_b" % ci] = bc
        _save_prior(out, "c%d_comb" % ci, cb)
        # the window from its initial state with the prior attached
        a = {k: v.copy() for k, v in arrs.items()}
        pb2 = Wn.Problem(**a, **sc)
        pr2 = M.Prior(pr.sids, pr.dims, pr.x0, pr.S, pr.r)
        pr2.bind({s: s for s in range(K)})
        pb2.prior = pr2
        st2 = Wn.solve(pb2, iters=5, lam0=1e-4)
        out.update({"c%d_Rwb_n" % ci: pb2.Rwb.copy(), "c%d_pwb_n" % ci: pb2.pwb.copy(),
                    "c%d_lmp_n" % ci: pb2.lmp.copy(),
                    "c%d_stats" % ci: np.array([st2["cost0"], st2["cost"], st2["accepted"], st2["lam"]])})
        Hf, bf, chi, ok, Hi, _imu, _off = Wn.final_linearisation(pb2)
        out["c%d_final_H" % ci], out["c%d_final_b" % ci] = Hf, bf
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    main(sys.argv[1])
