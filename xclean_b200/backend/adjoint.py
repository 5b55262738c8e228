"""Differentiable window BA: the implicit adjoint of the converged solve behind a torch.autograd.Function.

    solver = BatchSolver(windows, "cuda", hold=0)             # packed once, resident on the device
    p = BAAdjoint.apply(intrinsics, baseline, extrinsic, weights, pixels, solver)
    loss = ((p - p_true) ** 2).sum()                            # e.g. translation error of the converged poses
    loss.backward()                                             # -> .grad of the five tensors

Inputs (CUDA tensors): intrinsics [nw, 4] (fx, fy, cx, cy per window), baseline [nw], extrinsic [nw, 6] (the
left-to-right extrinsic (omega, t) at the rectified rig: must be zero; its gradient is the sensitivity of the
converged poses to de-rectifying it), weights [M] (the per-row weight 1/sigma inside the Huber kernel), pixels
[M, 2] (observed pixels per row; the right rows use column 0).  Output: the converged body translations [slots, 3]
(float64; the batch's slots in window order).

Forward: `iters` LM iterations of window.solve (float64, batched: one launch, or the large-window path when the
batch holds few large windows); then the landmarks whose Gauss-Newton step would take the inverse depth to <= 1e-9
(window.solve keeps them where they are, while its Schur complement assumes they move, so its fixed point is not
stationary) are flagged constant and `free_iters` LM iterations run with them held; then at most `newton_steps`
landmark-eliminated Newton steps on the exact Hessian (the LM converges only linearly where Huber weights are active,
and the adjoint is exact only at a stationary point): each moves every landmark to the minimum of its own cost with
the poses fixed, then solves the exact reduced pose system; landmarks whose minimum lies at infinity (rho < 1e-7) are
flagged constant on the way.  Backward: one solve H x = dL/dstate with the exact reduced system (its Cholesky factor
for the poses, the landmarks by back-substitution, at most two refinement steps on the exact residual; H applied
through dual numbers, Jacobians recomputed from the state rather than stored; conjugate gradients preconditioned with
the Gauss-Newton system where the reduced system is not positive definite), then dL/dtheta = -(d2C / dtheta dstate) x,
scattered to the window parameters and to every observation row.
The solver keeps the converged state between forward and backward: backward raises RuntimeError when a solver call
changed it in between (another forward, solve, solve_free, newton, reset; the solver's `generation` counts them;
writes into solver.t are the caller's to avoid).  ctx.newton_stats / ctx.adjoint_stats keep the per-window stats
(column 2: the gradient max-norm at the returned state; a window that did not reach a stationary point within
`newton_steps` has an approximate gradient).  The flagged landmarks are constants of the forward and of the adjoint.
"""
from __future__ import annotations

import torch


class BAAdjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, intrinsics, baseline, extrinsic, weights, pixels, solver, iters=20, newton_steps=40,
                lam0=1e-4, tol=1e-12, free_iters=20):
        if float(extrinsic.detach().abs().max()) != 0.0:
            raise ValueError("BAAdjoint: the left-to-right extrinsic is the rectified rig (zero); only its gradient "
                             "is returned")
        t = solver.t
        nw = solver.nw
        if tuple(intrinsics.shape) != (nw, 4) or tuple(baseline.shape) != (nw,) or tuple(extrinsic.shape) != (nw, 6):
            raise ValueError("BAAdjoint: intrinsics [nw,4], baseline [nw], extrinsic [nw,6]")
        if weights.shape != t["ob_isig"].shape or pixels.shape != t["ob_z"].shape:
            raise ValueError("BAAdjoint: weights [M], pixels [M,2] of the packed batch")
        with torch.no_grad():
            t["cam"][:, 0:4].copy_(intrinsics.detach().to(torch.float64))
            t["cam"][:, 4].copy_(baseline.detach().to(torch.float64))
            t["ob_isig"].copy_(weights.detach().to(torch.float64))
            t["ob_z"].copy_(pixels.detach().to(torch.float64))
            solver.reset()
            solver.solve(int(iters), float(lam0), "fp64", path="auto")    # the large-window path for few large windows
            solver.newton(0)                                        # flag the landmarks the LM cannot move
            solver.solve_free(int(free_iters), float(lam0), path="auto")
            st = solver.newton(int(newton_steps), tol=float(tol))
        ctx.solver = solver
        ctx.generation = solver.generation
        ctx.tol = float(tol)
        ctx.dtypes = (intrinsics.dtype, baseline.dtype, extrinsic.dtype, weights.dtype, pixels.dtype)
        ctx.newton_stats = st
        return t["pwb"].clone()

    @staticmethod
    def backward(ctx, grad_p):
        solver = ctx.solver
        if solver.generation != ctx.generation:
            raise RuntimeError("BAAdjoint: the solver's state changed between forward and backward (a solve, newton, "
                               "reset or another forward on the same solver); run backward first")
        gpose = torch.zeros((grad_p.shape[0], 6), dtype=torch.float64, device=grad_p.device)
        gpose[:, 3:] = grad_p.to(torch.float64)
        stats, gtheta, gisig, gz = solver.adjoint(gpose, tol=ctx.tol)
        ctx.adjoint_stats = stats
        di, db, de, dw, dp = ctx.dtypes
        return (gtheta[:, 0:4].to(di), gtheta[:, 4].to(db), gtheta[:, 5:11].to(de), gisig.to(dw), gz.to(dp),
                None, None, None, None, None, None)


def inputs_of(solver, requires_grad=True):
    """The solver's current parameters as leaf tensors (intrinsics, baseline, extrinsic = 0, weights, pixels)."""
    t = solver.t
    mk = lambda x: x.detach().clone().requires_grad_(requires_grad)
    return (mk(t["cam"][:, 0:4]), mk(t["cam"][:, 4]),
            mk(torch.zeros((solver.nw, 6), dtype=torch.float64, device=t["cam"].device)),
            mk(t["ob_isig"]), mk(t["ob_z"]))
