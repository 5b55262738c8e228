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


def test_short_scratch_is_refused_on_the_device():
    """A scratch that cannot hold the batch's per-landmark records: the kernels count the landmarks from the windows,
    write nothing past the scratch, leave the state unchanged and answer XCB_BA_STATUS_SCRATCH for every window."""
    import ctypes

    import torch
    from xclean_b200 import _lib
    from xclean_b200.backend.ba import BatchSolver, MAX_SLOTS
    bs = BatchSolver(windows_small(3, seed=5), "cuda", hold=0)
    Lt = int(bs.host["lmp"].shape[0])
    buf = torch.full((256 + 8 * 3 * Lt + 4096,), 0xA5, dtype=torch.uint8, device="cuda")
    short = 256 + 8 * 3 * (Lt - 1)                      # one landmark's trial state short
    before = {k: bs.t[k].clone() for k in ("Rwb", "pwb", "lmp")}
    bs.stats.zero_()
    for mode in (_lib.XCB_BA_FP64, _lib.XCB_BA_MIXED):
        rc = _lib.lib().xcb_ba_solve_windows_dev(ctypes.byref(bs.desc), bs.max_slots, 5, 1e-4, mode,
                                                 bs.stats.data_ptr(), bs.dx0.data_ptr(), 6 * MAX_SLOTS,
                                                 buf.data_ptr(), short, 0, None)
        assert rc == _lib.XCB_OK
        torch.cuda.synchronize()
        assert (bs.stats[:, 4].cpu().numpy() == _lib.XCB_BA_STATUS_SCRATCH).all()
        assert bool((buf[256:] == 0xA5).all()), "the kernel wrote into the scratch it refused"
        for k, v in before.items():
            assert torch.equal(bs.t[k], v), k
    # the Newton kernel: 19 doubles per landmark, then the reduced-system copies
    ncopy = int(_lib.lib().xcb_ba_newton_scratch_bytes(bs.nw, 0)) - 512
    nst = torch.zeros((bs.nw, 4), dtype=torch.float64, device="cuda")
    nbuf = torch.full((256 + 8 * 19 * Lt + ncopy + 4096,), 0xA5, dtype=torch.uint8, device="cuda")
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _lib.lib().xcb_ba_newton_windows_dev(ctypes.byref(bs.desc), bs.max_slots, _lib.XCB_BA_NEWTON_POLISH, 2, 10,
                                              1e-12, None, ctypes.c_void_p(z.data_ptr()), ctypes.c_void_p(z.data_ptr()),
                                              ctypes.c_void_p(z.data_ptr()), ctypes.c_void_p(nst.data_ptr()),
                                              ctypes.c_void_p(nbuf.data_ptr()), 256 + 8 * 19 * (Lt - 1) + ncopy, 0,
                                              None)
    assert rc == _lib.XCB_OK
    torch.cuda.synchronize()
    assert (nst[:, 3].cpu().numpy() == _lib.XCB_BA_STATUS_SCRATCH).all()
    assert bool((nbuf[256:] == 0xA5).all())
    for k, v in before.items():
        assert torch.equal(bs.t[k], v), k
