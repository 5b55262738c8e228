"""The implicit adjoint on windows of the differentiable-BA shape: 4 windows of 10 keyframes and 2,000 landmarks seen by
2-6 keyframes, 1 px noise, 5 % outliers (synth_ba.config3_windows).

- The forward ends at a stationary point of the float64 cost: the gradient of oracle/ba_adjoint_ref.py's restatement
  of the window cost at the device state, over the variables (the landmarks the forward flagged constant excluded, their
  rows kept), is below 1e-6.
- The adjoint matches that restatement's autodiff implicit gradient (solved through the Schur complement on the poses,
  `implicit_grad_schur`) to 1e-5 relative, group-wise (max-norm of the error over max-norm of the reference), on the 11
  window parameters, every row's weight and every row's pixels.
- It matches central finite differences of the device forward (re-converged from the solved state with the same
  constant landmarks, `newton(flag=False)`) on fx, fy, cx, cy (step 1e-3 px), the baseline (step 1e-5 m) and, per
  window, the two pixel rows and the weight row with the largest gradients (steps 1e-3 px and 1e-4), to 1e-5 of the
  group's largest gradient.  The rectified rig's extrinsic gradient has no finite-difference counterpart here (the
  device forward is the rectified model), so it is checked against the autodiff reference only."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5
NW = 4


@pytest.fixture(scope="module")
def c3():
    import torch
    from xclean_b200.backend import synth_ba as S
    from xclean_b200.backend.adjoint import BAAdjoint, inputs_of
    from xclean_b200.backend.ba import BatchSolver
    ws = S.config3_windows(NW, seed=11)
    solver = BatchSolver(ws, "cuda", hold=0)
    inp = inputs_of(solver)
    p = BAAdjoint.apply(*inp, solver, 20, 30)
    ptrue = torch.as_tensor(np.concatenate([w.pwb_true for w in ws]), device="cuda")
    ((p - ptrue) ** 2).sum().backward()
    torch.cuda.synchronize()
    grads = [x.grad.detach().cpu().numpy() for x in inp]
    state = {k: solver.t[k].clone() for k in ("Rwb", "pwb", "lmp")}
    ro = np.concatenate([[0], np.cumsum([w.ob_pose.shape[0] for w in ws])])
    return dict(ws=ws, solver=solver, grads=grads, state=state, scratch=solver.nscratch.clone(),
                frozen=solver.frozen().cpu().numpy(), ro=ro)


def _ref_window(c3, i):
    from oracle import ba_adjoint_ref as AR
    w, s = c3["ws"][i], c3["solver"]
    so, lo = s.host["slot_off"], s.host["lm_off"]
    P, L = w.Rwb.shape[0], w.lmp.shape[0]
    c = w.copy()
    c.Rwb = c3["state"]["Rwb"].cpu().numpy().reshape(-1, 3, 3)[so[i]:so[i] + P].copy()
    c.pwb = c3["state"]["pwb"].cpu().numpy()[so[i]:so[i] + P].copy()
    c.lmp = c3["state"]["lmp"].cpu().numpy()[lo[i]:lo[i] + L].copy()
    return AR.Window(c, hold=0, const=c3["frozen"][lo[i]:lo[i] + L])


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_config3_adjoint_matches_the_autodiff_reference_at_a_stationary_point(c3):
    from oracle import ba_adjoint_ref as AR
    gi, gb, ge, gw, gp = c3["grads"]
    for i, w in enumerate(c3["ws"]):
        W = _ref_window(c3, i)
        gth, gis, gz, gmax = AR.implicit_grad_schur(W, W.theta0, W.isig0, W.z0, 2 * (W.p0.numpy() - w.pwb_true))
        assert gmax < 1e-6, (i, gmax)
        r0, r1 = c3["ro"][i], c3["ro"][i + 1]
        dev_theta = np.concatenate([gi[i], [gb[i]], ge[i]])
        assert _rel(dev_theta, gth) < TOL, (i, dev_theta, gth)
        assert _rel(gw[r0:r1], gis) < TOL, i
        assert _rel(gp[r0:r1], gz) < TOL, i


def test_config3_adjoint_matches_central_finite_differences(c3):
    s, ws, ro = c3["solver"], c3["ws"], c3["ro"]
    gi, gb, _ge, gw, gp = c3["grads"]
    so = s.host["slot_off"]

    def losses():
        # from the solved state, with the same constant landmarks; per-window loss sum |t - t_gt|^2
        for k, v in c3["state"].items():
            s.t[k].copy_(v)
        s.nscratch.copy_(c3["scratch"])
        st = s.newton(30, flag=False).cpu().numpy()
        assert float(st[:, 2].max()) < 1e-6, st
        pw = s.t["pwb"].cpu().numpy()
        return np.array([((pw[so[i]:so[i] + w.Rwb.shape[0]] - w.pwb_true) ** 2).sum() for i, w in enumerate(ws)])

    def central(field, index, h):
        base = s.t[field].clone()
        out = []
        for sg in (1.0, -1.0):
            s.t[field].copy_(base)
            s.t[field][index] += sg * h
            out.append(losses())
        s.t[field].copy_(base)
        return (out[0] - out[1]) / (2.0 * h)

    import torch
    rows = torch.arange(NW, device="cuda")
    for j, h in ((0, 1e-3), (1, 1e-3), (2, 1e-3), (3, 1e-3), (4, 1e-5)):
        fd = central("cam", (rows, torch.full_like(rows, j)), h)
        dev = gi[:, j] if j < 4 else gb
        assert _rel(dev, fd) < TOL, (j, dev, fd)
    # per window the two pixel rows and the weight row with the largest gradients, one row of every window per solve
    zrows = np.stack([ro[i] + np.argsort(-np.abs(gp[ro[i]:ro[i + 1], 0]))[:2] for i in range(NW)])
    wrows = np.array([ro[i] + int(np.argmax(np.abs(gw[ro[i]:ro[i + 1]]))) for i in range(NW)])
    for k in range(2):
        idx = torch.as_tensor(zrows[:, k], device="cuda")
        fd = central("ob_z", (idx, torch.zeros_like(idx)), 1e-3)
        for i in range(NW):
            assert abs(fd[i] - gp[zrows[i, k], 0]) < TOL * np.abs(gp[ro[i]:ro[i + 1]]).max(), (i, k)
    fd = central("ob_isig", torch.as_tensor(wrows, device="cuda"), 1e-4)
    for i in range(NW):
        assert abs(fd[i] - gw[wrows[i]]) < TOL * np.abs(gw[ro[i]:ro[i + 1]]).max(), i


def test_config3_clusters_and_one_cta_per_window_agree(c3):
    """The Newton kernel gives a window a thread-block cluster of up to four CTAs when there are fewer windows than SMs
    (here 4 CTAs each) and reduces across them in rank order; with `grid` equal to the window count it runs one CTA
    per window.  Both forward states and adjoints agree to rounding (the sums run in another order)."""
    import torch
    from xclean_b200.backend.ba import BatchSolver
    s1, ws = c3["solver"], c3["ws"]
    s2 = BatchSolver(ws, "cuda", hold=0)
    for k in ("cam", "ob_isig", "ob_z"):
        s2.t[k].copy_(s1.t[k])
    s2.reset()
    s2.solve(20, 1e-4, "fp64", path="auto")
    s2.newton(0, grid=NW)
    s2.solve_free(20, 1e-4)
    st = s2.newton(40, grid=NW).cpu().numpy()
    assert float(st[:, 2].max()) < 1e-6, st
    for k in ("Rwb", "pwb", "lmp"):
        a, b = c3["state"][k].cpu().numpy(), s2.t[k].cpu().numpy()
        assert np.abs(a - b).max() < 1e-9 * max(1.0, np.abs(a).max()), k
    ptrue = torch.as_tensor(np.concatenate([w.pwb_true for w in ws]), device="cuda")
    gpose = torch.zeros((s2.t["pwb"].shape[0], 6), dtype=torch.float64, device="cuda")
    gpose[:, 3:] = 2 * (s2.t["pwb"] - ptrue)
    _st, gth, gis, gz = s2.adjoint(gpose, grid=NW)
    gi, gb, ge, gw, gp = c3["grads"]
    dev_theta = np.concatenate([gi, gb[:, None], ge], axis=1)
    assert _rel(gth.cpu().numpy(), dev_theta) < 1e-7
    assert _rel(gis.cpu().numpy(), gw) < 1e-7
    assert _rel(gz.cpu().numpy(), gp) < 1e-7
