"""Batched window BA on the device (libxcb200 through the C ABI) against the float64 oracle (the reference's
window.solve restated in C).  Tolerances: FP64 mode - the first pose step to 1e-8 relative and the final states
to 1e-6 (atomics change the summation order); mixed mode - the first pose step to 1e-6 relative (the precision
target), the LM trajectory (accepted count) identical."""
import numpy as np
import pytest

from oracle import ba_oracle as BO
from xclean_b200.backend import synth_ba as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def windows_small(n=6, seed=0):
    rng = np.random.default_rng(seed)
    return [S.make_window(None, K=int(rng.integers(4, 12)), L=int(rng.integers(80, 400)), obs_min=2, obs_max=8,
                          rng=np.random.default_rng([seed, i])) for i in range(n)]


@pytest.mark.parametrize("precision,tol_dx", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_batch_matches_oracle(precision, tol_dx):
    from xclean_b200.backend.ba import solve_batch
    ws = windows_small()
    ref = [w.copy() for w in ws]
    outs = [BO.solve(r, iters=5, lam0=1e-4, hold=0) for r in ref]
    res = solve_batch(ws, iters=5, lam0=1e-4, precision=precision, hold=0)
    for i, (w, r, o) in enumerate(zip(ws, ref, outs)):
        assert res["status"][i] == 0
        assert rel(res["dx0_list"][i], o["dx0"]) < tol_dx, (i, rel(res["dx0_list"][i], o["dx0"]))
        assert abs(res["cost0"][i] - o["cost0"]) <= 1e-9 * abs(o["cost0"])
        assert res["accepted"][i] == o["accepted"], i
        assert np.abs(w.pwb - r.pwb).max() < 1e-6 and np.abs(w.Rwb - r.Rwb).max() < 1e-6
        assert np.abs(w.lmp - r.lmp).max() < 1e-5 * max(1.0, np.abs(r.lmp).max())


@pytest.mark.parametrize("precision,tol_dx", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_batch_with_extrinsic_and_depth_prior(precision, tol_dx):
    """Non-identity body-to-camera extrinsic and the inverse-depth prior (the paths the golden windows pin)."""
    from xclean_b200.backend.ba import solve_batch
    ext = dict(Rbc=S.so3_exp(np.array([0.02, -0.03, 0.01])), pbc=np.array([0.05, -0.02, 0.1]), depth_prior=0.05)
    ws = [S.make_window(None, K=k, L=l, obs_min=2, obs_max=8, rng=np.random.default_rng(100 + k), **ext)
          for k, l in ((5, 120), (9, 350), (14, 600))]
    ref = [w.copy() for w in ws]
    outs = [BO.solve(r, iters=5, lam0=1e-4, hold=0) for r in ref]
    res = solve_batch(ws, iters=5, lam0=1e-4, precision=precision, hold=0)
    for i, (w, r, o) in enumerate(zip(ws, ref, outs)):
        assert res["status"][i] == 0
        assert rel(res["dx0_list"][i], o["dx0"]) < tol_dx, (i, rel(res["dx0_list"][i], o["dx0"]))
        assert abs(res["cost0"][i] - o["cost0"]) <= 1e-9 * abs(o["cost0"])
        assert res["accepted"][i] == o["accepted"], i
        assert np.abs(w.pwb - r.pwb).max() < 1e-6 and np.abs(w.Rwb - r.Rwb).max() < 1e-6


def test_config0_window_mixed_step_error():
    from xclean_b200.backend.ba import solve_batch
    w = S.config0_window(1)
    r = w.copy()
    o = BO.solve(r, iters=5, lam0=1e-4, hold=0)
    res = solve_batch([w], iters=5, lam0=1e-4, precision="mixed", hold=0)
    assert rel(res["dx0_list"][0], o["dx0"]) <= 1e-6
    assert res["accepted"][0] == o["accepted"]


def test_limits():
    from xclean_b200.backend.ba import pack_windows
    w = S.make_window(0, K=21, L=50)
    with pytest.raises(ValueError):
        pack_windows([w])
