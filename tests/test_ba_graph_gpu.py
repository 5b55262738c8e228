"""The batched window solve inside a captured CUDA graph: the reset (state copies) and the one persistent launch are
captured once and replayed; each replay gives the results of a direct call on the same windows (to 1e-9 relative:
the shared-memory atomics of the reduced system sum in a different order each run)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_window_solve_replays_from_a_cuda_graph():
    import torch
    from xclean_b200.backend import synth_ba as S
    from xclean_b200.backend.ba import BatchSolver
    ws = [S.make_window(None, K=int(k), L=int(l), obs_min=2, obs_max=8, rng=np.random.default_rng([5, i]))
          for i, (k, l) in enumerate(((6, 300), (11, 900), (4, 120), (16, 1500)))]
    bs = BatchSolver(ws, "cuda", hold=0)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        bs.reset()
        bs.solve(5, 1e-4, "fp64", stream=s)           # direct call (also sets the kernel's attributes before capture)
    s.synchronize()
    want = {k: bs.t[k].clone() for k in ("Rwb", "pwb", "lmp")}
    want_stats = bs.stats.clone()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        bs.reset()
        bs.solve(5, 1e-4, "fp64", stream=s)
    for _ in range(2):
        for k in ("Rwb", "pwb", "lmp"):
            bs.t[k].zero_()
        g.replay()
        torch.cuda.synchronize()
        for k in ("Rwb", "pwb", "lmp"):
            a, b = bs.t[k].double(), want[k].double()
            assert float((a - b).abs().max()) <= 1e-9 * max(1.0, float(b.abs().max())), k
        st, wst = bs.stats.cpu().numpy(), want_stats.cpu().numpy()
        assert np.array_equal(st[:, 2], wst[:, 2])                  # accepted LM steps
        assert np.allclose(st[:, 1], wst[:, 1], rtol=1e-9, atol=0)  # final costs
