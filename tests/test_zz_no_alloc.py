"""The allocation-free batched window solve (xcb_ba_solve_windows_noalloc) through the C ABI.

It exists for callers that cannot call cudaMalloc while running (a real-time loop that must not risk an allocation's
device synchronisation and unbounded latency, a plugin whose host application owns the device memory).  Here it is
checked against the existing entry point (xcb_ba_solve_windows_dev with caller-provided scratch) on the same inputs,
twice in a row, in both precisions, within the tolerance of the other BA device tests (the first pose step to 1e-8
relative in float64 and 1e-6 in mixed precision, the states to 1e-6); the second call must leave the device's free
memory unchanged, and its size limit is checked.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from xclean_b200 import _lib
from xclean_b200.backend import synth_ba as S

pytestmark = pytest.mark.gpu


def _windows():
    rng = np.random.default_rng(42)
    return [S.make_window(None, K=int(rng.integers(4, 10)), L=int(rng.integers(60, 250)), obs_min=2, obs_max=6,
                          rng=np.random.default_rng([42, i])) for i in range(5)]


def _noalloc(bs, iters, lam0, prec, stream):
    Lt = int(bs.host["lmp"].shape[0])
    return _lib.lib().xcb_ba_solve_windows_noalloc(ctypes.byref(bs.desc), Lt, bs.max_slots, int(iters), float(lam0),
                                                   _lib.XCB_BA_FP64 if prec == "fp64" else _lib.XCB_BA_MIXED,
                                                   bs.stats.data_ptr(), bs.dx0.data_ptr(), bs.dx0.shape[1], 0,
                                                   ctypes.c_void_p(stream.cuda_stream or None))


@pytest.mark.parametrize("prec,tol_dx", [("fp64", 1e-8), ("mixed", 1e-6)])
def test_noalloc_matches_the_scratch_entry_point_twice(prec, tol_dx):
    import torch
    from xclean_b200.backend.ba import BatchSolver
    bs = BatchSolver(_windows(), "cuda", hold=0)
    stream = torch.cuda.current_stream()
    # the existing entry point: reference outputs
    bs.reset()
    bs.solve(5, 1e-4, prec)
    torch.cuda.synchronize()
    ref = bs.results()
    ref_state = {k: bs.t[k].clone() for k in ("Rwb", "pwb", "lmp")}
    for call in range(2):
        bs.reset()
        bs.stats.zero_()
        bs.dx0.zero_()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = _noalloc(bs, 5, 1e-4, prec, stream)
        assert rc == _lib.XCB_OK, _lib.lib().xcb_last_error()
        torch.cuda.synchronize()
        if call == 1:
            # after the first call (which looks up the array's address), a call takes no device memory at all
            assert torch.cuda.mem_get_info()[0] == free0
        got = bs.results()
        assert (got["status"] == 0).all()
        assert np.array_equal(got["accepted"], ref["accepted"])
        np.testing.assert_allclose(got["cost0"], ref["cost0"], rtol=1e-10)
        for i in range(bs.nw):
            n = 6 * int(bs.host["P"][i])
            a, b = got["dx0"][i][:n], ref["dx0"][i][:n]
            assert np.linalg.norm(a - b) <= tol_dx * np.linalg.norm(b)
        for k in ("Rwb", "pwb", "lmp"):
            assert float((bs.t[k] - ref_state[k]).abs().max()) < 1e-6


def test_noalloc_rejects_batches_beyond_its_scratch():
    from xclean_b200.backend.ba import BatchSolver
    import torch
    bs = BatchSolver(_windows()[:1], "cuda", hold=0)
    too_many = _lib.lib().xcb_ba_noalloc_max_landmarks() + 1
    rc = _lib.lib().xcb_ba_solve_windows_noalloc(ctypes.byref(bs.desc), too_many, bs.max_slots, 5, 1e-4,
                                                 _lib.XCB_BA_FP64, bs.stats.data_ptr(), bs.dx0.data_ptr(),
                                                 bs.dx0.shape[1], 0, None)
    assert rc == _lib.XCB_ERR_CAPACITY
    assert b"landmarks exceed the static scratch" in _lib.lib().xcb_last_error()
    torch.cuda.synchronize()
