"""CPU oracle of the dense 32-direction SGM (test infrastructure; never the product path): oracle/sgm_oracle.c, the
reference's src/xclean/stereo/sgm32.py restated in C, and the reference's own SGM kernels where they were compiled
(oracle/_ref/libsgmref.so, made by oracle/build_ref_sgm.py; it needs a GPU to run).

Only tests/ and bench.py's CPU-baseline leg import this module."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import front_oracle as _fo

REF_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libsgmref.so")
P1, P2, UNIQ, LR, DMIN = 13, 152, 0.05, 1.0, 0.5          # sgm32.py:68-82


def sgm(left, right, p1=P1, p2=P2, uniq=UNIQ, lr=LR, dmin=DMIN, volumes=False):
    """-> (disp, conf) float32 (H, W) [, cost (H, W, 128) u8, sum (H, W, 128) u16]."""
    L = np.ascontiguousarray(left, np.uint8)
    R = np.ascontiguousarray(right, np.uint8)
    H, W = L.shape
    disp = np.zeros((H, W), np.float32)
    conf = np.zeros((H, W), np.float32)
    C = np.zeros((H, W, 128), np.uint8) if volumes else None
    S = np.zeros((H, W, 128), np.uint16) if volumes else None
    p = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)
    _fo.lib().xo_sgm(p(L), p(R), H, W, int(p1), int(p2), ctypes.c_float(uniq), ctypes.c_float(lr),
                     ctypes.c_float(dmin), p(disp), p(conf), p(C), p(S))
    return (disp, conf, C, S) if volumes else (disp, conf)


def ref_available():
    return os.path.exists(REF_LIB)


def ref_sgm(left_t, right_t, p1=P1, p2=P2, uniq=UNIQ, lr=LR, dmin=DMIN):
    """The reference's own kernels on device tensors (torch CUDA uint8 (H, W)) -> (disp, conf, sum) host arrays."""
    import torch
    lib = ctypes.CDLL(REF_LIB)
    H, W = left_t.shape
    disp = torch.zeros((H, W), dtype=torch.float32, device=left_t.device)
    conf = torch.zeros((H, W), dtype=torch.float32, device=left_t.device)
    S = torch.zeros((H, W, 128), dtype=torch.int16, device=left_t.device)
    v = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.xr_sgm(v(left_t), v(right_t), H, W, int(p1), int(p2), ctypes.c_float(uniq), ctypes.c_float(lr),
                    ctypes.c_float(dmin), v(disp), v(conf), v(S))
    if rc != 0:
        raise RuntimeError("reference SGM kernels failed (%d)" % rc)
    return disp.cpu().numpy(), conf.cpu().numpy(), S.cpu().numpy().view(np.uint16)


def ref_sgm_time(left_t, right_t, passes=3, p1=P1, p2=P2, uniq=UNIQ, lr=LR, dmin=DMIN):
    """The reference's own kernels timed on F pairs in device memory (torch CUDA uint8 (F, H, W)), buffers allocated
    once as SGM32 does; one untimed pass, then `passes` passes between CUDA events -> ms per frame."""
    import torch
    lib = ctypes.CDLL(REF_LIB)
    F, H, W = left_t.shape
    disp = torch.zeros((H, W), dtype=torch.float32, device=left_t.device)
    conf = torch.zeros((H, W), dtype=torch.float32, device=left_t.device)
    ms = ctypes.c_float(0.0)
    v = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.xr_sgm_time(v(left_t), v(right_t), F, H, W, int(p1), int(p2), ctypes.c_float(uniq), ctypes.c_float(lr),
                         ctypes.c_float(dmin), v(disp), v(conf), int(passes), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError("reference SGM kernels failed (%d)" % rc)
    return float(ms.value)
