"""The CPU oracle (oracle/front_oracle.c) against the reference's golden outputs: bit for bit.

This pins the oracle before it is used as the checker of the device path."""
import numpy as np
import pytest

from oracle import front_oracle as O
from tests import _golden as G


@pytest.fixture(scope="module", params=G.CASES)
def case(request):
    return request.param, G.load_case(request.param)


def test_detect_matches_reference(case):
    name, c = case
    cal = G.calib_of(c)
    for img, kp_ref, desc_ref in ((c["left0"], c["kp0"], c["desc0"]), (c["left1"], c["kp1"], c["desc1"])):
        kp = O.detect(img, int(c["budget"]), cal["q99"], cal["dy_vend"], cal["dx_vend"], cap=int(c["budget"]))
        assert G.same_bits(kp, kp_ref), name
        pat = G.pattern()
        desc = O.orb(O.blur(img, cal["kf"], cal["blur_vr"], cal["blur_vc"]), kp, pat)
        assert np.array_equal(desc, desc_ref), name


def test_noise_floor_matches_reference(case):
    name, c = case
    cal = G.calib_of(c)
    for img, ref in ((c["left0"], c["floor0"]), (c["left1"], c["floor1"])):
        fl, _ff = O.noise_floor(img, cal["q99"])
        assert np.isfinite(ref) and fl == float(ref), name


def test_stereo_matches_reference(case):
    name, c = case
    kp = c["kp0"].astype(np.float64)
    for tag, dlo, dhi, dy, band in G.stereo_variants(c):
        lo = None if dlo is None else np.full(len(kp), dlo, np.int64)
        hi = None if dhi is None else np.full(len(kp), dhi, np.int64)
        d, s, ok, zn, ody = O.stereo(c["left0"], c["right0"], kp, lo, hi, dy=dy, band=band, half=5)
        assert G.same_bits(d, c["st_%s_d" % tag]), (name, tag)
        assert G.same_bits(s, c["st_%s_sig" % tag]), (name, tag)
        assert np.array_equal(ok, c["st_%s_ok" % tag]), (name, tag)
        assert G.same_bits(zn, c["st_%s_zn" % tag]), (name, tag)
        assert G.same_bits(np.nan_to_num(ody, nan=-1e300), np.nan_to_num(c["st_%s_dy" % tag], nan=-1e300)), (name, tag)


def test_match_matches_reference(case):
    name, c = case
    i0, i1 = O.match_desc(c["desc0"], c["desc1"])
    assert np.array_equal(i0, c["m_i0"]) and np.array_equal(i1, c["m_i1"]), name


def test_lk_solver_matches_numba_lapack():
    z = np.load(G.GOLDEN + "/lk_solver.npz")
    X, Inv = O.lk_solve_inv(z["As"], z["gs"])
    assert G.same_bits(X, z["X"]) and G.same_bits(Inv, z["Inv"])


def test_edge_cases_oracle():
    """Empty inputs, off-image and non-finite keypoints, flat images (no positive response)."""
    flat = np.full((64, 80), 77, np.uint8)
    assert len(O.detect(flat, 50, 1.0, 64, 80)) == 0
    d, s, ok, zn, ody = O.stereo(flat, flat, np.zeros((0, 2)))
    assert len(d) == 0
    kp = np.array([[np.nan, 5.0], [np.inf, 3.0], [1e300, 2.0], [-3.0, 10.0], [40.0, 30.0]])
    d, s, ok, zn, ody = O.stereo(flat, flat, kp)
    assert not ok.any() and (zn == -2.0).all() and np.isinf(s).all()
    e0, e1 = O.match_desc(np.zeros((1, 32), np.uint8), np.zeros((5, 32), np.uint8))
    assert len(e0) == 0 and len(e1) == 0


@pytest.mark.parametrize("name", sorted(G.mapmatch_cases()))
def test_mapmatch_matches_reference(name):
    """The oracle's gated map matcher against xclean.front.mapmatch.MapMatcher's outputs (= mapmatch_fast's), bit for
    bit: realistic frames, an inflated re-search, degenerate inputs (non-finite keypoints and covariances, NaN d2 on
    accepted matches) and tie-heavy lattices."""
    c = G.mapmatch_cases()[name]
    with np.errstate(all="ignore"):
        got = O.mapmatch(c["kp"], c["desc"], c["uv"], c["S"], c["lmd"], c["lnd"], int(c["W"]), int(c["H"]),
                         float(c["chi2"]))
    assert G.same_outputs(got, (c["out_kp"], c["out_d"], c["out_d2"]))


def test_mapmatch_oracle_edges():
    """Empty landmark / keypoint sets return the defaults; more valid descriptors than slots is refused."""
    kp = np.array([[10.0, 10.0]])
    d = np.zeros((1, 32), np.uint8)
    out = O.mapmatch(np.zeros((0, 2)), np.zeros((0, 32), np.uint8), np.array([[10.0, 10.0]]), np.eye(2)[None],
                     np.zeros((1, 3, 32), np.uint8), np.array([1]), 64, 64)
    assert out[0].tolist() == [-1] and out[1].tolist() == [9999] and np.isinf(out[2]).all()
    out = O.mapmatch(kp, d, np.zeros((0, 2)), np.zeros((0, 2, 2)), np.zeros((0, 3, 32), np.uint8),
                     np.zeros(0, np.int64), 64, 64)
    assert all(len(o) == 0 for o in out)
    with pytest.raises(ValueError):
        O.mapmatch(kp, d, np.array([[10.0, 10.0]]), np.eye(2)[None], np.zeros((1, 2, 32), np.uint8), np.array([3]),
                   64, 64)


@pytest.mark.parametrize("name", sorted(G.predict_cases()))
def test_predict_projection_matches_reference(name):
    """The oracle's window.predict_projection against the reference's numba function, bit for bit, with the outputs
    pre-filled as the engine fills them (entries the reference leaves alone stay as they were); then the map matcher
    on the in-view landmarks."""
    c = G.predict_cases()[name]
    uv, S, ok, depth = c["uv0"].copy(), c["S0"].copy(), c["ok0"].copy(), c["depth0"].copy()
    with np.errstate(all="ignore"):
        O.predict_projection(*G.predict_args(c), uv, S, ok, depth)
    for got, k in ((uv, "uv"), (S, "S"), (depth, "depth")):
        assert np.array_equal(got.view(np.uint64), c[k].view(np.uint64)), k
    assert np.array_equal(ok, c["ok"])
    sel = np.nonzero(ok)[0]
    with np.errstate(all="ignore"):
        got = O.mapmatch(c["kp"], c["desc"], uv[sel], S[sel], c["lmd"][sel], c["lnd"][sel], int(c["W"]), int(c["H"]))
    assert G.same_outputs(got, (c["m_kp"], c["m_d"], c["m_d2"]))
