"""BAAdjoint's host logic on the CPU, with a stand-in for the device solver (the kernels are covered by the GPU tests):
the forward's call sequence (LM, constant-landmark flags, LM with them held, Newton polish), the parameters it loads
into the packed batch, the backward's pose cotangent (rotation part zero, translation part dL/dp) and the routing of
the adjoint's outputs to the five inputs in their own dtypes, the argument checks, and the refusal to run backward
after the solver's state changed."""
import pytest

torch = pytest.importorskip("torch")

NW, S, M = 2, 5, 7


class FakeSolver:
    """The BatchSolver surface BAAdjoint uses, on CPU tensors: every state-changing call bumps `generation`."""

    def __init__(self):
        f = torch.float64
        self.nw = NW
        self.generation = 0
        self.calls = []
        self.t = {"cam": torch.zeros((NW, 6), dtype=f), "ob_isig": torch.zeros(M, dtype=f),
                  "ob_z": torch.zeros((M, 2), dtype=f), "pwb": torch.zeros((S, 3), dtype=f)}
        self.gpose = None

    def _step(self, name, *a, **k):
        self.generation += 1
        self.calls.append((name, a, k))
        # a converged translation that depends on the loaded parameters
        self.t["pwb"].copy_(torch.arange(S * 3, dtype=torch.float64).view(S, 3) * self.t["cam"][0, 0])

    def reset(self):
        self._step("reset")

    def solve(self, *a, **k):
        self._step("solve", *a, **k)

    def solve_free(self, *a, **k):
        self._step("solve_free", *a, **k)

    def newton(self, *a, **k):
        self._step("newton", *a, **k)
        return torch.zeros((NW, 4), dtype=torch.float64)

    def adjoint(self, gpose, tol=1e-12):
        self.gpose = gpose.clone()
        f = torch.float64
        gth = torch.arange(NW * 11, dtype=f).view(NW, 11) + 1.0
        return torch.zeros((NW, 4), dtype=f), gth, torch.full((M,), 2.0, dtype=f), torch.full((M, 2), 3.0, dtype=f)


def _inputs(dtype=torch.float64):
    mk = lambda x: x.to(dtype).requires_grad_(True)
    return (mk(torch.tensor([[458.0, 457.0, 367.0, 248.0]] * NW)), mk(torch.full((NW,), 0.11)),
            mk(torch.zeros((NW, 6))), mk(torch.ones(M)), mk(torch.rand(M, 2)))


def test_forward_sequence_and_backward_routing():
    from xclean_b200.backend.adjoint import BAAdjoint
    s = FakeSolver()
    inp = _inputs(torch.float32)
    p = BAAdjoint.apply(*inp, s, 20, 30)
    assert [c[0] for c in s.calls] == ["reset", "solve", "newton", "solve_free", "newton"]
    assert s.calls[1][1][:3] == (20, 1e-4, "fp64") and s.calls[1][2] == {"path": "auto"}
    assert s.calls[2][1] == (0,)
    assert s.calls[3][1] == (20, 1e-4) and s.calls[3][2] == {"path": "auto"}
    assert s.calls[4][1] == (30,)
    assert torch.equal(s.t["cam"][:, 0:4], inp[0].detach().double())
    assert torch.equal(s.t["cam"][:, 4], inp[1].detach().double())
    assert torch.equal(s.t["ob_isig"], inp[3].detach().double())
    assert torch.equal(s.t["ob_z"], inp[4].detach().double())
    gp = torch.randn(S, 3, dtype=torch.float64)
    (p * gp).sum().backward()
    assert torch.equal(s.gpose[:, :3], torch.zeros(S, 3, dtype=torch.float64))
    assert torch.equal(s.gpose[:, 3:], gp)
    gth = torch.arange(NW * 11, dtype=torch.float64).view(NW, 11) + 1.0
    for x in inp:
        assert x.grad is not None and x.grad.dtype == torch.float32 and x.grad.shape == x.shape
    assert torch.equal(inp[0].grad, gth[:, 0:4].float())
    assert torch.equal(inp[1].grad, gth[:, 4].float())
    assert torch.equal(inp[2].grad, gth[:, 5:11].float())
    assert torch.equal(inp[3].grad, torch.full((M,), 2.0))
    assert torch.equal(inp[4].grad, torch.full((M, 2), 3.0))


def test_backward_after_the_state_changed_raises():
    from xclean_b200.backend.adjoint import BAAdjoint
    s = FakeSolver()
    p = BAAdjoint.apply(*_inputs(), s, 20, 30)
    s.solve(5)
    with pytest.raises(RuntimeError, match="changed between forward and backward"):
        p.sum().backward()
    # a second forward on the same solver invalidates the first graph but not its own
    s2 = FakeSolver()
    p1 = BAAdjoint.apply(*_inputs(), s2, 20, 30)
    p2 = BAAdjoint.apply(*_inputs(), s2, 20, 30)
    p2.sum().backward()
    with pytest.raises(RuntimeError):
        p1.sum().backward()


def test_argument_checks():
    from xclean_b200.backend.adjoint import BAAdjoint
    s = FakeSolver()
    i, b, e, w, z = _inputs()
    with pytest.raises(ValueError, match="rectified rig"):
        BAAdjoint.apply(i, b, e.detach() + 1e-3, w, z, s)
    with pytest.raises(ValueError):
        BAAdjoint.apply(i[:1], b, e, w, z, s)
    with pytest.raises(ValueError):
        BAAdjoint.apply(i, b, e, w[:-1], z, s)
    with pytest.raises(ValueError):
        BAAdjoint.apply(i, b, e, w, z[:, :1], s)
    assert s.calls == []
