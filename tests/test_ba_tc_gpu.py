"""The tensor-core Gram product (xcb_ba_gram_tc: D = U U^T through tcgen05 kind::tf32 MMAs with a TF32 hi / lo split,
FP32 accumulation in tensor memory) against a float64 torch reference of the same op.

Tolerance: float32 accuracy, |D - D64| <= 2e-6 sqrt(K / 32) max|D64| (the split carries about 22 bits per product; the
accumulation is float32)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,K", [(1, 1), (7, 0), (120, 32), (128, 33), (120, 1000), (96, 4099)])
def test_gram_matches_float64(n, K):
    import torch
    from xclean_b200 import _lib
    rng = np.random.default_rng(n * 131 + K)
    # Schur-like columns: a few nonzero 6-row blocks per column, magnitudes over several decades
    U = np.zeros((n, K), np.float32)
    for k in range(K):
        for s in rng.choice(max(n // 6, 1), size=min(3, max(n // 6, 1)), replace=False):
            U[6 * s:6 * s + 6, k] = (rng.normal(size=min(6, n - 6 * s)) * 10.0 ** rng.uniform(-3, 3)).astype(np.float32)
    Ud = torch.from_numpy(U).cuda()
    D = torch.full((n, n), np.nan, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _lib.lib().xcb_ba_gram_tc(ctypes.c_void_p(Ud.data_ptr()), n, K, ctypes.c_void_p(D.data_ptr()),
                                   ctypes.c_void_p(err.data_ptr()), None)
    assert rc == _lib.XCB_OK, _lib.lib().xcb_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = (torch.from_numpy(U.astype(np.float64)) @ torch.from_numpy(U.astype(np.float64)).T).numpy()
    got = D.cpu().numpy().astype(np.float64)
    assert np.isfinite(got).all()
    scale = max(np.abs(ref).max(), 1e-30)
    tol = 2e-6 * np.sqrt(max(K, 32) / 32.0)
    assert np.abs(got - ref).max() <= tol * scale, np.abs(got - ref).max() / scale
