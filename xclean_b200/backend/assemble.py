"""The window Problem assembled on the device from the engine's state (the drop-in for P1Engine._problem's host work,
src/xclean/vio/engine_live.py:407-530, visual part), and solved there without a host round trip.

    asm = DeviceAssembler(P=10, n_lm=20000, M=60000)          # capacities; device buffers allocated once
    out = asm.run(state)                                      # state: dict of torch CUDA tensors (see run())
    win = asm.window(Rwb, pwb, Rbc, pbc, cam)                 # the assembled arrays as one window of the batched solve
    win.solve(iters=5, lam0=1e-4, precision="fp64")           # xcb_ba_solve_windows_dev on them, asynchronous
    host = asm.to_host()                                      # the Problem's arrays as numpy (tests, write-back)

The reference builds the Problem with numpy on the host every keyframe and copies it to the solver; here the
alive-landmark scan, the stable sort of the observations by landmark, the gathers and the weights are seven launches
on the caller's stream (xcb_ba_assemble_dev), and their outputs are already the solve's inputs.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib
from .ba import MAX_SLOTS

_STATE = ("sids", "slot_n", "lid", "uv", "cam", "valid", "sig", "lm_alive", "lm_host", "lm_p", "lm_rho_meas",
          "lm_sig_lk", "lm_span")
_DT = {"sids": "int64", "slot_n": "int64", "lid": "int64", "uv": "float64", "cam": "int64", "valid": "uint8",
       "sig": "float64", "lm_alive": "uint8", "lm_host": "int64", "lm_p": "float64", "lm_rho_meas": "float64",
       "lm_sig_lk": "float64", "lm_span": "float64", "select": "uint8"}


class DeviceAssembler:
    def __init__(self, P, n_lm, M, device="cuda"):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.P, self.n_lm, self.M = int(P), int(n_lm), int(M)
        if not 1 <= self.P <= MAX_SLOTS:
            raise ValueError("DeviceAssembler: 1..%d slots" % MAX_SLOTS)
        z = lambda shape, dt: torch.zeros(shape, dtype=dt, device=self.dev)
        nl, m = max(self.n_lm, 1), max(self.M, 1)
        self.out = dict(counts=z(3, torch.int32), alive=z(nl, torch.int64), src=z((m, 2), torch.int32),
                        lmp=z((nl, 3), torch.float64), lm_host=z(nl, torch.int32), lm_mask=z(nl, torch.uint8),
                        rho_meas=z(nl, torch.float64), rho_isig=z(nl, torch.float64), lm_ob=z(nl + 1, torch.int32),
                        ob_pose=z(m, torch.int32), ob_cam=z(m, torch.uint8), ob_z=z((m, 2), torch.float64),
                        ob_isig=z(m, torch.float64), ob_valid=z(m, torch.uint8))
        nb = int(_lib.lib().xcb_ba_assemble_scratch_bytes(self.n_lm, self.M, self.P))
        self.scratch = z(nb, torch.uint8)
        self.desc = _lib.BaAssembled()
        for k, t in self.out.items():
            setattr(self.desc, k, t.data_ptr())

    def run(self, state, prior_mode=True, kappa_d=1.0, fB=1.0, sig_px=1.0, select=None, stream=None):
        """state: dict of CUDA tensors - sids [P], slot_n [P] (the slots' observation lists concatenated in slot order),
        lid [M], uv [M,2], cam [M], valid [M] (uint8), sig [M], lm_alive [n_lm] (uint8), lm_host [n_lm] (host slot
        id), lm_p [n_lm,3], lm_rho_meas / lm_sig_lk / lm_span [n_lm]; select [n_lm] (uint8) or None.  Launches only."""
        torch = self.torch
        t = {}
        for k in _STATE:
            v = state[k]
            if not (isinstance(v, torch.Tensor) and v.is_cuda and v.is_contiguous() and str(v.dtype) == "torch." + _DT[k]):
                raise ValueError("DeviceAssembler.run: %s must be a contiguous CUDA %s tensor" % (k, _DT[k]))
            t[k] = v
        P, M, n_lm = int(t["sids"].numel()), int(t["lid"].numel()), int(t["lm_alive"].numel())
        if P != self.P or M > self.M or n_lm > self.n_lm:
            raise ValueError("DeviceAssembler.run: %d slots, %d observations, %d landmark ids exceed the capacities "
                             "(%d, %d, %d)" % (P, M, n_lm, self.P, self.M, self.n_lm))
        e = _lib.BaEngine()
        e.P, e.M, e.n_lm = P, M, n_lm
        for k, v in t.items():
            setattr(e, k, v.data_ptr())
        if select is not None:
            if not (select.is_cuda and select.dtype == torch.uint8 and select.numel() >= n_lm):
                raise ValueError("DeviceAssembler.run: select must be a CUDA uint8 tensor over the landmark ids")
            e.select = select.data_ptr()
        e.prior_mode, e.kappa_d, e.fB, e.sig_px = int(bool(prior_mode)), float(kappa_d), float(fB), float(sig_px)
        s = stream if stream is not None else torch.cuda.current_stream(self.dev)
        self._keep = (t, select)
        rc = _lib.lib().xcb_ba_assemble_dev(ctypes.byref(e), ctypes.byref(self.desc), self.scratch.data_ptr(),
                                            self.scratch.numel(), ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_assemble_dev")
        return self.out

    def to_host(self):
        """The assembled Problem's arrays as numpy (synchronises): the oracle's keys."""
        c = self.out["counts"].cpu().numpy()
        if c[2]:
            raise RuntimeError("assemble: a landmark's host slot is not in the window")
        L, M = int(c[0]), int(c[1])
        g = lambda k, n: self.out[k][:n].cpu().numpy()
        return dict(alive=g("alive", L), lmp=g("lmp", L), lm_host=g("lm_host", L).astype(np.int64),
                    lm_mask=g("lm_mask", L).astype(np.bool_), rho_meas=g("rho_meas", L), rho_isig=g("rho_isig", L),
                    ob_start=g("lm_ob", L + 1).astype(np.int64), ob_pose=g("ob_pose", M).astype(np.int64),
                    ob_cam=g("ob_cam", M).astype(np.int64), ob_z=g("ob_z", M), ob_isig=g("ob_isig", M),
                    ob_valid=g("ob_valid", M).astype(np.bool_), src=g("src", M).astype(np.int64))

    def window(self, Rwb, pwb, Rbc, pbc, cam, hold=-1):
        return AssembledWindow(self, Rwb, pwb, Rbc, pbc, cam, hold)


class AssembledWindow:
    """The assembler's outputs as the one window of an xcb_ba_windows batch (no host round trip): the slot poses
    (Rwb [P,3,3], pwb [P,3] CUDA float64, updated in place by solve), the extrinsic and the camera
    (fx, fy, cx, cy, B, huber_k)."""

    def __init__(self, asm, Rwb, pwb, Rbc, pbc, cam, hold=-1):
        torch = asm.torch
        dev = asm.dev
        f64 = lambda a, shape: torch.as_tensor(np.asarray(a, np.float64).reshape(shape), device=dev).contiguous()
        self.asm = asm
        self.Rwb = Rwb if isinstance(Rwb, torch.Tensor) else f64(Rwb, (-1, 9))
        self.pwb = pwb if isinstance(pwb, torch.Tensor) else f64(pwb, (-1, 3))
        P = asm.P
        i32 = lambda v: torch.tensor(v, dtype=torch.int32, device=dev)
        self.t = dict(P=i32([P]), slot_off=i32([0]), lm_off=i32([0]), hold=i32([int(hold)]),
                      cam=f64(cam, (1, 6)),
                      ext=f64(np.concatenate([np.asarray(Rbc, np.float64).ravel(), np.asarray(pbc, np.float64).ravel()]),
                              (1, 12)))
        d = _lib.BaWindows()
        d.nw = 1
        o = asm.out
        for k, v in (("P", self.t["P"]), ("L", o["counts"]), ("slot_off", self.t["slot_off"]),
                     ("lm_off", self.t["lm_off"]), ("hold", self.t["hold"]), ("cam", self.t["cam"]),
                     ("ext", self.t["ext"]), ("Rwb", self.Rwb), ("pwb", self.pwb), ("lmp", o["lmp"]),
                     ("lm_host", o["lm_host"]), ("lm_mask", o["lm_mask"]), ("rho_meas", o["rho_meas"]),
                     ("rho_isig", o["rho_isig"]), ("lm_ob", o["lm_ob"]), ("ob_pose", o["ob_pose"]),
                     ("ob_cam", o["ob_cam"]), ("ob_z", o["ob_z"]), ("ob_isig", o["ob_isig"]),
                     ("ob_valid", o["ob_valid"])):
            setattr(d, k, v.data_ptr())
        self.desc = d
        self.stats = torch.zeros((1, 8), dtype=torch.float64, device=dev)
        self.dx0 = torch.zeros((1, 6 * MAX_SLOTS), dtype=torch.float64, device=dev)
        nb = int(_lib.lib().xcb_ba_scratch_bytes(1, max(asm.n_lm, 1)))
        self.scratch = torch.zeros(nb, dtype=torch.uint8, device=dev)

    def solve(self, iters=5, lam0=1e-4, precision="fp64", stream=None):
        """window.solve on the assembled window (asynchronous); the state (Rwb, pwb and the assembled lmp) is updated
        in place."""
        from .ba import PRECISIONS
        torch = self.asm.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.asm.dev)
        rc = _lib.lib().xcb_ba_solve_windows_dev(ctypes.byref(self.desc), self.asm.P, int(iters), float(lam0),
                                                 PRECISIONS[precision], self.stats.data_ptr(), self.dx0.data_ptr(),
                                                 6 * MAX_SLOTS, self.scratch.data_ptr(), self.scratch.numel(), 0,
                                                 ctypes.c_void_p(s.cuda_stream or None))
        _lib.check(rc, None, "xcb_ba_solve_windows_dev")
