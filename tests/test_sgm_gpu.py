"""The device SGM (xcb_sgm_*, csrc/stereo_sgm.cu) bit for bit against the reference's own SGM kernels
(oracle/_ref/libsgmref.so: the kernel source of src/xclean/stereo/sgm32.py compiled by oracle/build_ref_sgm.py with the
reference's launches) and against the CPU oracle (oracle/sgm_oracle.c): disparities, confidences, the cost volume and
the uint16 aggregated volume, on crops of a rendered driving pair, on a pair whose true shift is known, and on tiny
and odd image sizes."""
import numpy as np
import pytest

from oracle import sgm_oracle as SO

pytestmark = pytest.mark.gpu


def _pair(W, H, seed=2):
    from xclean_b200 import synth
    L, R = synth.sequence(synth.CAM_SMALL, 1, seed=seed)
    L, R = L.numpy()[0], R.numpy()[0]
    y0, x0 = (L.shape[0] - H) // 2, (L.shape[1] - W) // 2
    return np.ascontiguousarray(L[y0:y0 + H, x0:x0 + W]), np.ascontiguousarray(R[y0:y0 + H, x0:x0 + W])


@pytest.mark.parametrize("W,H", [(160, 120), (97, 61), (9, 5)])
def test_sgm_matches_the_oracle(W, H):
    from xclean_b200.stereo.sgm32 import SGM32
    L, R = _pair(W, H)
    s = SGM32(W, H)
    try:
        d, c = s.compute(L, R)
        C, S = s.cost_volume(), s.aggregated_volume()
    finally:
        s.close()
    od, oc, oC, oS = SO.sgm(L, R, volumes=True)
    assert np.array_equal(C, oC)
    assert np.array_equal(S, oS)
    assert np.array_equal(d.view(np.uint32), od.view(np.uint32))
    assert np.array_equal(c.view(np.uint32), oc.view(np.uint32))
    if W > 100:
        assert (d > 0).mean() > 0.3


def test_sgm_matches_the_reference_kernels_at_full_size():
    import torch
    from xclean_b200.stereo.sgm32 import SGM32
    if not SO.ref_available():
        pytest.skip("oracle/_ref/libsgmref.so not built (python oracle/build_ref_sgm.py <reference>/src)")
    L, R = _pair(752, 480)
    Lt, Rt = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    s = SGM32(752, 480)
    try:
        d, c = s.compute_gpu(Lt, Rt)
        torch.cuda.synchronize()
        d, c = d.cpu().numpy(), c.cpu().numpy()
        S = s.aggregated_volume()
    finally:
        s.close()
    rd, rc, rS = SO.ref_sgm(Lt, Rt)
    assert np.array_equal(S, rS)
    assert np.array_equal(d.view(np.uint32), rd.view(np.uint32))
    assert np.array_equal(c.view(np.uint32), rc.view(np.uint32))
    assert (d > 0).mean() > 0.3


def test_sgm_known_shift_and_errors():
    from xclean_b200.stereo.sgm32 import SGM32
    rng = np.random.default_rng(3)
    H, W, shift = 64, 200, 11
    base = (rng.random((H, W + shift)) * 255).astype(np.uint8)
    L, R = np.ascontiguousarray(base[:, :W]), np.ascontiguousarray(base[:, shift:])
    s = SGM32(W, H)
    try:
        d, c = s.compute(L, R)
        with pytest.raises(ValueError):
            import torch
            s.compute_gpu(torch.zeros((H, W + 1), dtype=torch.uint8, device="cuda"),
                          torch.zeros((H, W + 1), dtype=torch.uint8, device="cuda"))
    finally:
        s.close()
    inner = d[:, 24:-8]
    assert ((inner > 0) & (np.abs(inner - shift) < 0.6)).mean() > 0.8
    od, oc = SO.sgm(L, R)
    assert np.array_equal(d.view(np.uint32), od.view(np.uint32))
    with pytest.raises(RuntimeError):
        SGM32(4096, 16)
