"""Generate tests/golden/assemble_golden.npz from the reference's window Problem assembly (run once, where the
reference is).

    NUMBA_CACHE_DIR=/tmp/nbcache python tests/golden/make_golden_assemble.py <reference>/src

The reference assembles a window.Problem from its engine state in P1Engine._problem (src/xclean/vio/engine_live.py
:407-530).  Here that method runs unbound on a minimal stand-in for the engine's state: the slots (sid, pose, the
observation lists lid / uv / cam / valid / sig), the landmark arrays (alive, host sid, position, inverse-depth
measurement, LK sigma, ambiguity span) and the constants it reads.  The states come from seeded synthetic windows
(xclean_b200.backend.synth_ba.make_window) turned into engine form: landmark ids spread over a larger id space, dead
landmarks, invalid observations, observations of dead landmarks, both stereo modes ("prior": inverse-depth priors from
the LK sigma and the span; "ur": right-camera rows), with and without a landmark selection.  Recorded: the inputs and
the Problem's arrays, the alive list and the (slot, index) source of every observation.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "assemble_golden.npz")
CASES = ((6, 300, 31, "prior", False), (10, 800, 32, "prior", True), (8, 500, 33, "ur", False))


class _State:
    """The engine attributes _problem reads."""


def engine_state(K, L, seed, mode):
    from xclean_b200.backend.synth_ba import make_window
    rng = np.random.default_rng(seed)
    w = make_window(None, K=K, L=L, obs_min=2, obs_max=6, rng=np.random.default_rng(seed))
    L = w.lmp.shape[0]
    n_lm = L + 200
    ids = np.sort(rng.choice(n_lm, size=L, replace=False)).astype(np.int64)
    st = _State()
    st.n_lm = n_lm
    st.lm_alive = np.zeros(n_lm + 50, bool)
    st.lm_alive[ids] = True
    st.lm_alive[rng.choice(ids, size=L // 20, replace=False)] = False        # died since they were observed
    sids = (100 + 3 * np.arange(K)).astype(np.int64)
    st.lm_host = np.full(n_lm + 50, -1, np.int64)
    st.lm_host[ids] = sids[np.asarray(w.lm_host, np.int64)]
    st.lm_p = np.zeros((n_lm + 50, 3))
    st.lm_p[ids] = w.lmp
    st.lm_rho_meas = rng.uniform(0.02, 0.5, n_lm + 50)
    st.lm_sig_lk = rng.uniform(0.02, 0.6, n_lm + 50)
    st.lm_sig_lk[rng.choice(n_lm, 30)] = np.inf
    st.lm_span = np.where(rng.random(n_lm + 50) < 0.1, rng.uniform(0.5, 4.0, n_lm + 50), 0.0)
    st.stereo_mode = mode
    st.kappa_d, st.fB, st.sig_px = 1.3, float(w.fx * w.B), 1.0
    st.vi, st.prior, st.imu_factors = False, None, []
    st.Rbc, st.pbc = np.asarray(w.Rbc, float), np.asarray(w.pbc, float)
    st.fx, st.fy, st.cx, st.cy, st.B = float(w.fx), float(w.fy), float(w.cx), float(w.cy), float(w.B)
    st.g_w = np.array([0.0, 0.0, -9.81])
    lm_of = np.repeat(np.arange(L), np.diff(np.asarray(w.ob_start, np.int64)))
    pose = np.asarray(w.ob_pose, np.int64)
    slots = []
    for i in range(K):
        sel = np.nonzero(pose == i)[0]
        sel = sel[rng.permutation(len(sel))]                                   # the engine's order of arrival
        lid = ids[lm_of[sel]]
        extra = rng.integers(0, n_lm, 5)                                       # observations of landmarks that
        lid = np.concatenate([lid, extra])                                    # are not in the window
        n = len(lid)
        uv = np.concatenate([np.asarray(w.ob_z, float)[sel], rng.uniform(0, 700, (5, 2))])
        cam = np.concatenate([np.asarray(w.ob_cam, np.int64)[sel], rng.integers(0, 2, 5)])
        valid = rng.random(n) > 0.07
        sig = rng.uniform(0.05, 0.8, n)
        slots.append({"sid": int(sids[i]), "R": np.asarray(w.Rwb[i], float), "p": np.asarray(w.pwb[i], float),
                      "lid": lid, "uv": uv, "cam": cam, "valid": valid, "sig": sig, "full": False})
    st.slots = slots
    return st


def main(src):
    sys.path.insert(0, src)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    from xclean.vio.engine_live import P1Engine
    out = {}
    for ci, (K, L, seed, mode, select) in enumerate(CASES):
        st = engine_state(K, L, seed, mode)
        c = "c%d_" % ci
        sel_mask = None
        if select:
            sel_mask = np.random.default_rng(seed + 7).random(st.n_lm + 50) < 0.8
        pb, meta = P1Engine._problem(st, lm_select=(None if sel_mask is None else (lambda a: sel_mask[a])),
                                     with_prior=False, posefree=False)
        out[c + "K"] = np.array([K])
        out[c + "mode"] = np.array([1 if mode == "prior" else 0])
        out[c + "n_lm"] = np.array([st.n_lm])
        out[c + "consts"] = np.array([st.kappa_d, st.fB, st.sig_px])
        for k in ("lm_alive", "lm_host", "lm_p", "lm_rho_meas", "lm_sig_lk", "lm_span"):
            out[c + k] = getattr(st, k)
        if sel_mask is not None:
            out[c + "select"] = sel_mask
        out[c + "sids"] = np.array([s["sid"] for s in st.slots], np.int64)
        for k in ("lid", "uv", "cam", "valid", "sig"):
            out[c + "slot_" + k] = np.concatenate([s[k] for s in st.slots])
        out[c + "slot_n"] = np.array([len(s["lid"]) for s in st.slots], np.int64)
        for k in ("lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose", "ob_cam", "ob_z",
                  "ob_isig", "ob_valid"):
            out[c + "pb_" + k] = np.asarray(getattr(pb, k))
        out[c + "alive"] = meta["alive"]
        out[c + "src"] = meta["src"]
        print(mode, "L", len(meta["alive"]), "M", len(pb.ob_pose))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    main(sys.argv[1])
