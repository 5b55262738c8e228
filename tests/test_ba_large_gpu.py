"""The large-window path of the batched window solve (xcb_ba_solve_windows_large_dev: the landmark passes of every
window in chunks on all SMs) against the persistent one-CTA-per-window kernel and the float64 oracle (the reference's
window.solve restated in C).

Tolerances as the other window tests: float64 - the first pose step to 1e-8 relative, the cost to 1e-10, the states to
1e-6 and the same accepted count (the chunks add their shares in another order); mixed precision - the first pose step
to 1e-6 relative against the float64 oracle."""
import numpy as np
import pytest

from oracle import ba_oracle as BO
from xclean_b200.backend import synth_ba as S

pytestmark = pytest.mark.gpu


def _windows():
    # 20-keyframe windows with 3-15 observing keyframes (the large configuration's shape), landmark counts that are
    # not multiples of the 256-landmark chunk, one window smaller than a chunk
    sizes = ((20, 1500), (20, 700), (16, 257), (12, 100))
    return [S.make_window(None, K=K, L=L, obs_min=3, obs_max=15, outlier_frac=0.10, step_m=0.15,
                          rng=np.random.default_rng([44, i])) for i, (K, L) in enumerate(sizes)]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_large_path_constant_landmarks_match_the_window_kernel():
    """The constant-landmark LM (the differentiable-BA forward: landmarks the Newton call flagged are held constant,
    their rows kept) on the large-window path against the one-CTA-per-window kernel, float64, the same flags."""
    import torch
    from xclean_b200.backend.ba import BatchSolver
    ws = _windows()
    a = BatchSolver(ws, "cuda", hold=0)
    b = BatchSolver(ws, "cuda", hold=0)
    for s in (a, b):
        s.solve(10, 1e-4, "fp64", path="window")
        s.newton(0)                                      # the flags
    assert torch.equal(a.frozen(), b.frozen()) and bool(a.frozen().any())
    held = b.t["lmp"][b.frozen()].clone()
    fa = a.solve_free(10, 1e-4, path="window").cpu().numpy()
    fb = b.solve_free(10, 1e-4, path="large").cpu().numpy()
    torch.cuda.synchronize()
    assert (fa[:, 4] == 0).all() and (fb[:, 4] == 0).all()
    assert np.array_equal(fa[:, 2], fb[:, 2])                               # accepted steps
    np.testing.assert_allclose(fb[:, 1], fa[:, 1], rtol=1e-9)               # final cost
    assert torch.equal(b.t["lmp"][b.frozen()], held)                         # the flagged landmarks did not move
    for k in ("Rwb", "pwb"):
        assert float((a.t[k] - b.t[k]).abs().max()) < 1e-6, k
    assert float((a.t["lmp"] - b.t["lmp"]).abs().max()) < 1e-5 * max(1.0, float(a.t["lmp"].abs().max()))


def test_large_path_matches_the_window_kernel_float64():
    import torch
    from xclean_b200.backend.ba import BatchSolver
    ws = _windows()
    a = BatchSolver(ws, "cuda", hold=0)
    b = BatchSolver(ws, "cuda", hold=0)
    a.solve(5, 1e-4, "fp64", path="window")
    b.solve(5, 1e-4, "fp64", path="large")
    torch.cuda.synchronize()
    ra, rb = a.results(), b.results()
    assert (ra["status"] == 0).all() and (rb["status"] == 0).all()
    assert np.array_equal(ra["accepted"], rb["accepted"])
    np.testing.assert_allclose(rb["cost0"], ra["cost0"], rtol=1e-10)
    np.testing.assert_allclose(rb["cost"], ra["cost"], rtol=1e-9)
    for i, w in enumerate(ws):
        n = 6 * w.Rwb.shape[0]
        assert _rel(rb["dx0"][i][:n], ra["dx0"][i][:n]) < 1e-8, i
    for k in ("Rwb", "pwb"):
        assert float((a.t[k] - b.t[k]).abs().max()) < 1e-6, k
    assert float((a.t["lmp"] - b.t["lmp"]).abs().max()) < 1e-5 * max(1.0, float(a.t["lmp"].abs().max()))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_large_path_against_the_oracle(precision, tol):
    from xclean_b200.backend.ba import solve_batch
    ws = _windows()[:3]
    ref = [w.copy() for w in ws]
    outs = [BO.solve(r, iters=5, lam0=1e-4, hold=0) for r in ref]
    res = solve_batch(ws, iters=5, lam0=1e-4, precision=precision, hold=0, path="large")
    for i, (w, r, o) in enumerate(zip(ws, ref, outs)):
        assert res["status"][i] == 0
        assert _rel(res["dx0_list"][i], o["dx0"]) < tol, (i, _rel(res["dx0_list"][i], o["dx0"]))
        assert abs(res["cost0"][i] - o["cost0"]) <= 1e-9 * abs(o["cost0"])
        assert res["accepted"][i] == o["accepted"], i
        assert np.abs(w.pwb - r.pwb).max() < 1e-6 and np.abs(w.Rwb - r.Rwb).max() < 1e-6


def test_large_path_refuses_a_short_scratch():
    import ctypes
    from xclean_b200 import _lib
    from xclean_b200.backend.ba import BatchSolver
    bs = BatchSolver(_windows()[2:], "cuda", hold=0)
    bs._large_setup()
    rc = _lib.lib().xcb_ba_solve_windows_large_dev(
        ctypes.byref(bs.desc), int(bs.host["Rwb"].shape[0]), int(bs.host["lmp"].shape[0]), bs.lchunks.data_ptr(),
        bs.nchunks, bs.max_slots, 5, 1e-4, _lib.XCB_BA_FP64, bs.stats.data_ptr(), None, 0, bs.lscratch.data_ptr(),
        bs.lscratch.numel() - 4096, None)
    assert rc == _lib.XCB_ERR_CAPACITY
