"""The float64 autodiff reference of the implicit adjoint (oracle/ba_adjoint_ref.py) checked on the CPU, without the
device: the Schur-complement form that the GPU tests of the 2,000-landmark windows use (`implicit_grad_schur`) equals
the dense-Hessian form (`implicit_grad`), with and without landmarks held constant, and both equal central finite
differences of the re-converged window solve.

Windows: 4 keyframes, 30 landmarks seen by 2-4 keyframes, a non-identity body-to-camera extrinsic, an inverse-depth
prior and 5 % outliers (Huber weights active), solved by Newton from the synthetic truth.  Tolerances: 1e-9 relative
between the two exact forms (the same quantities, summed in another order); 1e-5 relative, group-wise (max-norm of
the error over max-norm of the reference gradient), against finite differences with steps 1e-3 px (fx, fy, cx, cy)
and 1e-5 m (the baseline)."""
import copy

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _window(seed, const_every=0):
    from oracle import ba_adjoint_ref as AR
    from xclean_b200.backend import synth_ba as S
    w = S.make_window(None, K=4, L=30, obs_min=2, obs_max=4, rng=np.random.default_rng(seed),
                      Rbc=S.so3_exp(np.array([0.02, -0.03, 0.01])), pbc=np.array([0.05, -0.02, 0.1]),
                      depth_prior=0.05)
    c = w.copy()
    c.Rwb, c.pwb, c.lmp = w.Rwb_true.copy(), w.pwb_true.copy(), w.lmp_true.copy()
    const = None
    if const_every:
        const = np.zeros(w.lmp.shape[0], bool)
        const[::const_every] = True
    W = AR.Window(c, hold=0, const=const)
    AR.solve(W, W.theta0, W.isig0, W.z0)
    return w, W


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("const_every", [0, 4])
def test_schur_form_equals_the_dense_form(const_every):
    from oracle import ba_adjoint_ref as AR
    w, W = _window(9, const_every)
    dLdp = 2 * (W.p0.numpy() - w.pwb_true)
    dense = AR.implicit_grad(W, W.theta0, W.isig0, W.z0, dLdp)
    gt, gs, gz, gmax = AR.implicit_grad_schur(W, W.theta0, W.isig0, W.z0, dLdp)
    assert gmax < 1e-8
    for a, b in zip((gt, gs, gz), dense):
        assert _rel(a, b) < 1e-9


def test_dense_form_equals_central_differences():
    from oracle import ba_adjoint_ref as AR
    w, W = _window(8)
    ptrue = torch.as_tensor(w.pwb_true)
    dLdp = 2 * (W.p0.numpy() - w.pwb_true)
    gt, _gs, _gz = AR.implicit_grad(W, W.theta0, W.isig0, W.z0, dLdp)

    def loss(theta):
        s = AR.solve(copy.deepcopy(W), theta, W.isig0, W.z0)
        return float(((s.p0 - ptrue) ** 2).sum())

    fd = np.zeros(5)
    for j, h in ((0, 1e-3), (1, 1e-3), (2, 1e-3), (3, 1e-3), (4, 1e-5)):
        tp, tm = W.theta0.clone(), W.theta0.clone()
        tp[j] += h
        tm[j] -= h
        fd[j] = (loss(tp) - loss(tm)) / (2 * h)
    assert _rel(gt[:4], fd[:4]) < 1e-5, (gt[:4], fd[:4])
    assert abs(gt[4] - fd[4]) < 1e-5 * abs(fd[4]), (gt[4], fd[4])
