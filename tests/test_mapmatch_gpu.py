"""Device gated map matcher (libxcb200.so through the C ABI) against the reference's golden outputs and the CPU
oracle: landmark -> keypoint index, Hamming distance and Mahalanobis d2, bit for bit (NaN payloads included)."""
import numpy as np
import pytest

from oracle import front_oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu


def _mm(W, H, **kw):
    from xclean_b200.front.mapmatch import MapMatcher
    return MapMatcher(W, H, **kw)


@pytest.mark.parametrize("name", sorted(G.mapmatch_cases()))
def test_golden_bitexact(name):
    c = G.mapmatch_cases()[name]
    mm = _mm(int(c["W"]), int(c["H"]))
    try:
        got = mm.match(c["kp"], c["desc"], c["uv"], c["S"], c["lmd"], c["lnd"], chi2=float(c["chi2"]))
    finally:
        mm.close()
    assert G.same_outputs(got, (c["out_kp"], c["out_d"], c["out_d2"])), name
    assert mm.stats["matched"] == int((c["out_kp"] >= 0).sum())


def _random_case(rng, W, H, N, L, D, dup=0.3):
    pool = rng.integers(0, 256, (max(4, N // 8), 32), dtype=np.uint8)
    kp = np.stack([rng.uniform(-12, W + 12, N), rng.uniform(-12, H + 12, N)], 1)
    desc = np.where(rng.random((N, 1)) < dup, pool[rng.integers(0, len(pool), N)],
                    rng.integers(0, 256, (N, 32), dtype=np.uint8)).astype(np.uint8)
    src = rng.integers(0, N, L)
    uv = kp[src] + rng.normal(0, 1.5, (L, 2))
    sx, sy, rho = rng.uniform(0.5, 9.0, L), rng.uniform(0.5, 9.0, L), rng.uniform(-0.9, 0.9, L)
    S = np.empty((L, 2, 2))
    S[:, 0, 0], S[:, 1, 1] = sx * sx, sy * sy
    S[:, 0, 1] = S[:, 1, 0] = rho * sx * sy
    lmd = rng.integers(0, 256, (L, D, 32), dtype=np.uint8)
    flips = np.packbits(rng.random((L, 256)) < rng.uniform(0, 0.3, (L, 1)), axis=1)
    lmd[:, 0] = desc[src] ^ flips
    lnd = rng.integers(0 if D > 1 else 1, D + 1, L).astype(np.int64)
    return kp, desc, uv, S, lmd, lnd


@pytest.mark.parametrize("W,H,N,L,D,chi2", [(752, 480, 1, 1, 1, 13.815510557964274),
                                            (752, 480, 37, 500, 3, 13.815510557964274),
                                            (1241, 376, 2000, 1500, 3, 13.815510557964274),
                                            (1241, 376, 2000, 3000, 3, 50.0),
                                            (1280, 720, 5000, 2500, 5, 13.815510557964274),
                                            (1280, 720, 4000, 6000, 3, 5.0)])
def test_random_vs_oracle(W, H, N, L, D, chi2):
    """Random frames, sizes past the handle's initial capacities (its buffers grow), several descriptor slots, other
    gate quantiles."""
    rng = np.random.default_rng(W + N + L + D)
    kp, desc, uv, S, lmd, lnd = _random_case(rng, W, H, N, L, D)
    mm = _mm(W, H)
    try:
        got = mm.match(kp, desc, uv, S, lmd, lnd, chi2=chi2)
        again = mm.match(kp[: N // 2 + 1], desc[: N // 2 + 1], uv, S, lmd, lnd, chi2=chi2)   # reused buffers
    finally:
        mm.close()
    assert G.same_outputs(got, O.mapmatch(kp, desc, uv, S, lmd, lnd, W, H, chi2))
    h = N // 2 + 1
    assert G.same_outputs(again, O.mapmatch(kp[:h], desc[:h], uv, S, lmd, lnd, W, H, chi2))


def test_crowded_keypoints_and_shared_claims():
    """All keypoints in a few cells, many landmarks per keypoint: long cell ranges and long owner folds."""
    rng = np.random.default_rng(7)
    W, H, N, L = 320, 240, 3000, 4000
    kp = np.concatenate([rng.normal(40, 3, (N // 2, 2)), rng.normal(200, 1, (N - N // 2, 2))])
    desc = rng.integers(0, 256, (N, 32), dtype=np.uint8)
    src = rng.integers(0, 50, L)                       # 50 keypoints claimed by 80 landmarks each
    uv = kp[src] + rng.normal(0, 0.3, (L, 2))
    S = np.tile(np.eye(2) * 9.0, (L, 1, 1))
    lmd = desc[src][:, None, :].copy()
    lnd = np.ones(L, np.int64)
    mm = _mm(W, H)
    try:
        got = mm.match(kp, desc, uv, S, lmd, lnd)
    finally:
        mm.close()
    want = O.mapmatch(kp, desc, uv, S, lmd, lnd, W, H)
    assert G.same_outputs(got, want)
    assert (want[0] >= 0).sum() > 0


def test_empty_inputs_and_errors():
    mm = _mm(64, 48)
    try:
        out = mm.match(np.zeros((0, 2)), np.zeros((0, 32), np.uint8), np.array([[10.0, 10.0]]), np.eye(2)[None],
                       np.zeros((1, 3, 32), np.uint8), np.array([1]))
        assert out[0].tolist() == [-1] and out[1].tolist() == [9999] and np.isinf(out[2]).all()
        out = mm.match(np.array([[1.0, 1.0]]), np.zeros((1, 32), np.uint8), np.zeros((0, 2)), np.zeros((0, 2, 2)),
                       np.zeros((0, 3, 32), np.uint8), np.zeros(0, np.int64))
        assert all(len(o) == 0 for o in out)
        with pytest.raises(ValueError):
            mm.match(np.array([[1.0, 1.0]]), np.zeros((1, 32), np.uint8), np.array([[1.0, 1.0]]), np.eye(2)[None],
                     np.zeros((1, 2, 32), np.uint8), np.array([3]))
    finally:
        mm.close()
    with pytest.raises(ValueError):
        _mm(8192, 8192)                                # more grid cells than one CTA's shared memory holds


def test_match_dev_batched_vs_oracle():
    """A batch of frames in device memory (float32 keypoints as the frontend stores them, ragged keypoint and
    landmark counts): every frame's rows equal the oracle's; rows past a frame's landmark count are not written."""
    import torch
    from xclean_b200 import synth
    rng = np.random.default_rng(3)
    W, H, F, Nk, Nl = 1241, 376, 6, 2048, 1600
    nkp = np.array([0, 1, 700, 2048, 1500, 1900], np.int32)
    kp = np.zeros((F, Nk, 2), np.float32)
    desc = np.zeros((F, Nk, 32), np.uint8)
    for f in range(F):
        kp[f] = np.stack([rng.uniform(-5, W + 5, Nk), rng.uniform(-5, H + 5, Nk)], 1).astype(np.float32)
        desc[f] = rng.integers(0, 256, (Nk, 32), dtype=np.uint8)
    m = np.tile(np.arange(Nk, dtype=np.int64), (F, 1))
    nmatch = np.minimum(nkp, np.roll(nkp, 1)).astype(np.int32)
    # frame f's landmarks from frame f-1; matches pair the same index (a keypoint that stayed in place)
    kp_lm = kp.copy()
    uv, S, lmd, lnd, nlm = synth.map_landmarks(kp_lm, nkp, desc, m, m, nmatch, n_lm=Nl, D=3, seed=5)
    nlm[2] = 0
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    mm = _mm(W, H, max_frames=F, max_kp=Nk, max_lm=Nl)
    try:
        out = dict(kp=torch.full((F, Nl), -7, dtype=torch.int64, device=dev),
                   d=torch.full((F, Nl), -7, dtype=torch.int64, device=dev),
                   d2=torch.full((F, Nl), -7.0, dtype=torch.float64, device=dev))
        mm.match_dev(T(kp), T(nkp), T(desc), T(uv), T(S), T(lmd), T(lnd), T(nlm), out=out)
        torch.cuda.synchronize()
        got = {k: v.cpu().numpy() for k, v in out.items()}
    finally:
        mm.close()
    for f in range(F):
        L = int(nlm[f])
        want = O.mapmatch(kp[f, :nkp[f]].astype(np.float64), desc[f, :nkp[f]], uv[f, :L], S[f, :L], lmd[f, :L],
                          lnd[f, :L], W, H)
        assert G.same_outputs((got["kp"][f, :L], got["d"][f, :L], got["d2"][f, :L]), want), f
        assert (got["kp"][f, L:] == -7).all() and (got["d2"][f, L:] == -7.0).all()
    want_all = O.mapmatch_frames(kp, nkp, desc, uv, S, lmd, lnd, nlm, W, H)
    for f in range(F):
        L = int(nlm[f])
        assert np.array_equal(want_all[0][f, :L], got["kp"][f, :L])


@pytest.mark.parametrize("name", sorted(G.predict_cases()))
def test_predict_projection_golden(name):
    """window.predict_projection on the device against the reference's outputs, bit for bit; entries the reference
    does not write keep the caller's values (checked with sentinels against the oracle)."""
    from xclean_b200.front.mapmatch import predict_projection
    c = G.predict_cases()[name]
    uv, S, ok, depth = c["uv0"].copy(), c["S0"].copy(), c["ok0"].copy(), c["depth0"].copy()
    assert predict_projection(*G.predict_args(c), uv, S, ok, depth) == 0
    for got, k in ((uv, "uv"), (S, "S"), (depth, "depth")):
        assert np.array_equal(got.view(np.uint64), c[k].view(np.uint64)), k
    assert np.array_equal(ok, c["ok"])
    L = len(ok)
    sent = [np.full((L, 2), 7.0), np.full((L, 2, 2), 3.0), np.ones(L, np.bool_), np.full(L, -1.0)]
    want = [a.copy() for a in sent]
    predict_projection(*G.predict_args(c), *sent)
    with np.errstate(all="ignore"):
        O.predict_projection(*G.predict_args(c), *want)
    for g, w in zip(sent, want):
        assert np.array_equal(g.view(np.uint8), w.view(np.uint8))


@pytest.mark.parametrize("name", sorted(G.predict_cases()))
def test_predict_match_golden(name):
    """The fused tracking step equals predict_projection followed by MapMatcher.match on the in-view landmarks."""
    c = G.predict_cases()[name]
    mm = _mm(int(c["W"]), int(c["H"]))
    try:
        args = G.predict_args(c)[:-2]                       # W, H come from the matcher
        uv, S, ok, depth, k, d, d2 = mm.predict_match(*args, c["kp"], c["desc"], c["lmd"], c["lnd"])
    finally:
        mm.close()
    for got, key in ((uv, "uv"), (S, "S"), (depth, "depth")):
        assert np.array_equal(got.view(np.uint64), c[key].view(np.uint64)), key
    assert np.array_equal(ok, c["ok"])
    sel = c["sel"]
    assert G.same_outputs((k[sel], d[sel], d2[sel]), (c["m_kp"], c["m_d"], c["m_d2"]))
    rest = np.setdiff1d(np.arange(len(ok)), sel)
    assert (k[rest] == -1).all() and (d[rest] == 9999).all() and np.isinf(d2[rest]).all()


def test_predict_match_random_vs_oracle():
    """A larger random window (5,000 landmarks, non-zero pose covariance) through the fused call, against the oracle's
    predict_projection + map matcher."""
    rng = np.random.default_rng(21)
    L, W, H = 5000, 1280, 720
    th = rng.normal(0, 0.05, 3)
    K = np.array([[0, -th[2], th[1]], [th[2], 0, -th[0]], [-th[1], th[0], 0]])
    Rwb = np.eye(3) + K + 0.5 * K @ K
    args = dict(Rwb_t=Rwb, pwb_t=rng.normal(0, 0.1, 3), Rbc=np.array([[0.0, 0.0, 1.0], [-1.0, 0.0, 0.0],
                                                                      [0.0, -1.0, 0.0]]),
                pbc=np.array([0.1, 0.0, 0.02]), Rwc_h=np.tile(np.array([[0.0, 0.0, 1.0], [-1.0, 0.0, 0.0],
                                                                        [0.0, -1.0, 0.0]]), (L, 1, 1)),
                pwc_h=rng.normal(0, 0.5, (L, 3)) - np.array([2.0, 0.0, 0.0]),
                lmp=np.stack([rng.uniform(-0.8, 0.8, L), rng.uniform(-0.5, 0.5, L), rng.uniform(0.05, 0.5, L)], 1),
                Spose=np.diag([1e-6, 1e-6, 1e-6, 1e-4, 1e-4, 1e-4]), Sl=np.tile(np.eye(3) * 1e-6, (L, 1, 1)),
                sig_px=1.5, fx=640.0, fy=640.0, cx=640.0, cy=360.0)
    order = ("Rwb_t", "pwb_t", "Rbc", "pbc", "Rwc_h", "pwc_h", "lmp", "Spose", "Sl", "sig_px", "fx", "fy", "cx", "cy")
    a = [args[k] for k in order]
    uv0, S0, ok0, dep0 = np.full((L, 2), np.nan), np.zeros((L, 2, 2)), np.zeros(L, np.bool_), np.zeros(L)
    O.predict_projection(*a, float(W), float(H), uv0, S0, ok0, dep0)
    sel = np.nonzero(ok0)[0]
    kp = np.concatenate([uv0[sel] + rng.normal(0, 1.0, (len(sel), 2)), rng.uniform(0, 700, (300, 2))])
    lmd = rng.integers(0, 256, (L, 3, 32), dtype=np.uint8)
    desc = np.concatenate([lmd[sel, 0], rng.integers(0, 256, (300, 32), dtype=np.uint8)])
    lnd = rng.integers(1, 4, L).astype(np.int64)
    mm = _mm(W, H)
    try:
        uv, S, ok, depth, k, d, d2 = mm.predict_match(*a, kp, desc, lmd, lnd)
    finally:
        mm.close()
    assert np.array_equal(ok, ok0) and np.array_equal(uv.view(np.uint64), uv0.view(np.uint64))
    assert np.array_equal(S.view(np.uint64), S0.view(np.uint64)) and np.array_equal(depth, dep0)
    want = O.mapmatch(kp, desc, uv0[sel], S0[sel], lmd[sel], lnd[sel], W, H)
    assert G.same_outputs((k[sel], d[sel], d2[sel]), want)
    assert len(sel) > 1000 and (want[0] >= 0).sum() > 500


@pytest.mark.parametrize("lanes", [1, 2, 4, 8])
def test_gate_lanes_give_identical_results(lanes):
    """The tuner's knob (lanes per landmark in the gate) changes only the time: bit-identical outputs for every value,
    on random frames with crowded cells and on the golden fixture's cases."""
    from xclean_b200 import _lib
    rng = np.random.default_rng(77)
    W, H, N, L, D = 1241, 376, 2000, 3000, 3
    kp, desc, uv, S, lmd, lnd = _random_case(rng, W, H, N, L, D)
    mm = _mm(W, H)
    try:
        mm.set_tuning(_lib.XCB_TUNE_MM_LANES, lanes)
        got = mm.match(kp, desc, uv, S, lmd, lnd, chi2=50.0)
        with pytest.raises(ValueError):                 # XCB_ERR_ARG, as every other bad argument
            mm.set_tuning(_lib.XCB_TUNE_MM_LANES, 3)
    finally:
        mm.close()
    assert G.same_outputs(got, O.mapmatch(kp, desc, uv, S, lmd, lnd, W, H, 50.0))
