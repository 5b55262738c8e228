"""Drop-in of src/xclean/backend/kernels.py: the local-BA stage kernels, same names and argument order.

The reference's wrappers take CuPy device arrays; these take torch CUDA tensors (float32 / int32, C-contiguous, the
reference's layouts) or raw device pointers (int), and launch the sm_100a kernels of libxcb200.so on the current
torch stream.  Accumulated outputs (Hll, bl, Hred, g) are added to, as in the reference: the caller zeroes them.
There is no CPU fallback: without the library or a CUDA device every call raises.

    build_blocks(Tcw, pts, okf, olm, ouv, Jpose, Jlm, resw, Hll, bl, Hpl, N, fx, cx, cy, huber)   kernels.py:794-800
    depth_prior(pts, chost, rho0, invsig, valid, Hll, bl, nl, huber)                            kernels.py:803-807
    inv3_damped(Hll, Hlli, nl, lam)                                                              kernels.py:810-813
    schur_pairs(Hpl, Hlli, okf, olm, pa, pb, Hred, npair, d, n)                                  kernels.py:816-819
    schur_grad(Hpl, Hlli, bl, okf, olm, g_, N, d)                                                kernels.py:822-825
    pose_blocks(Jp, res, kf, Hred, grad, N, r, d, n)                                             kernels.py:828-831
    chol_solve(H, b, x, n, nthreads=256) -> status (int32 device tensor: 0, or k+1 at a
                                            non-positive pivot k)                                kernels.py:837-850
    backsub(Hpl, Hlli, bl, dxp, okf, offs, dxl, nl, d)                                           kernels.py:853-856
    build_blocks_id(Tcw, hpose, hidx, mbear, rhov, okf, olm, ouv, Jp, resw, kslot, Hll, bl, Hpl,
                    N, fx, cx, cy, huber)                                                        kernels.py:866-872
    landmark_prior_id(mb, rhov, m0, rho0, invsig, wbear, valid, Hll, bl, nl, huber)             kernels.py:875-880
    pose_blocks_id(Jp, res, kslot, Hred, grad, N, d, n)                                          kernels.py:883-886
    schur_pairs_id(Hpl, Hlli, kslot, olm, pa, pb, Hred, npair, d, n)                            kernels.py:889-892
    schur_grad_id(Hpl, Hlli, bl, kslot, olm, g_, N, d)                                           kernels.py:895-898
    backsub_id(Hpl, Hlli, bl, dxp, kslot, offs, dxl, nl, d)                                      kernels.py:901-904

One difference: chol_solve's status buffer is cleared by every call (the reference's is set on failure and never
cleared, so one non-positive-definite system marks every later call).
"""
from __future__ import annotations

import ctypes

from .. import _lib

F32, I32 = "float32", "int32"


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream or None)


def _p(x, dtype, name):
    """Device pointer of a torch CUDA tensor of `dtype` (or a raw pointer given as int)."""
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    import torch
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError("%s: a CUDA torch tensor (or a device pointer) is required" % name)
    if str(x.dtype) != "torch." + dtype:
        raise TypeError("%s: dtype %s, expected %s" % (name, x.dtype, dtype))
    if not x.is_contiguous():
        raise ValueError("%s: tensor must be contiguous" % name)
    return ctypes.c_void_p(x.data_ptr())


def _call(fn, *args):
    _lib.check(getattr(_lib.lib(), fn)(*args), what=fn)


def build_blocks(Tcw, pts, okf, olm, ouv, Jpose, Jlm, resw, Hll, bl, Hpl, N, fx, cx, cy, huber):
    _call("xcb_bk_build_blocks", _p(Tcw, F32, "Tcw"), _p(pts, F32, "pts"), _p(okf, I32, "okf"), _p(olm, I32, "olm"),
          _p(ouv, F32, "ouv"), _p(Jpose, F32, "Jpose"), _p(Jlm, F32, "Jlm"), _p(resw, F32, "resw"),
          _p(Hll, F32, "Hll"), _p(bl, F32, "bl"), _p(Hpl, F32, "Hpl"), int(N), float(fx), float(cx), float(cy),
          float(huber), _stream())


def depth_prior(pts, chost, rho0, invsig, valid, Hll, bl, nl, huber):
    _call("xcb_bk_depth_prior", _p(pts, F32, "pts"), _p(chost, F32, "chost"), _p(rho0, F32, "rho0"),
          _p(invsig, F32, "invsig"), _p(valid, F32, "valid"), _p(Hll, F32, "Hll"), _p(bl, F32, "bl"), int(nl),
          float(huber), _stream())


def inv3_damped(Hll, Hlli, nl, lam):
    _call("xcb_bk_inv3_damped", _p(Hll, F32, "Hll"), _p(Hlli, F32, "Hlli"), int(nl), float(lam), _stream())


def schur_pairs(Hpl, Hlli, okf, olm, pa, pb, Hred, npair, d, n):
    _call("xcb_bk_schur_pairs", _p(Hpl, F32, "Hpl"), _p(Hlli, F32, "Hlli"), _p(okf, I32, "okf"), _p(olm, I32, "olm"),
          _p(pa, I32, "pa"), _p(pb, I32, "pb"), _p(Hred, F32, "Hred"), int(npair), int(d), int(n), _stream())


def schur_grad(Hpl, Hlli, bl, okf, olm, g_, N, d):
    _call("xcb_bk_schur_grad", _p(Hpl, F32, "Hpl"), _p(Hlli, F32, "Hlli"), _p(bl, F32, "bl"), _p(okf, I32, "okf"),
          _p(olm, I32, "olm"), _p(g_, F32, "g"), int(N), int(d), _stream())


def pose_blocks(Jp, res, kf, Hred, grad, N, r, d, n):
    _call("xcb_bk_pose_blocks", _p(Jp, F32, "Jp"), _p(res, F32, "res"), _p(kf, I32, "kf"), _p(Hred, F32, "Hred"),
          _p(grad, F32, "grad"), int(N), int(r), int(d), int(n), _stream())


_STATUS = {}


def chol_solve(H, b, x, n, nthreads=256):
    """Factor and solve in one launch (H is overwritten by its lower Cholesky factor) -> the status tensor."""
    import torch
    dev = H.device if isinstance(H, torch.Tensor) else torch.device("cuda", torch.cuda.current_device())
    st = _STATUS.get(dev)
    if st is None:
        st = _STATUS[dev] = torch.zeros(1, dtype=torch.int32, device=dev)
    _call("xcb_bk_chol_solve", _p(H, F32, "H"), _p(b, F32, "b"), _p(x, F32, "x"), int(n), _p(st, I32, "status"),
          int(nthreads), _stream())
    return st


def backsub(Hpl, Hlli, bl, dxp, okf, offs, dxl, nl, d):
    _call("xcb_bk_backsub", _p(Hpl, F32, "Hpl"), _p(Hlli, F32, "Hlli"), _p(bl, F32, "bl"), _p(dxp, F32, "dxp"),
          _p(okf, I32, "okf"), _p(offs, I32, "offs"), _p(dxl, F32, "dxl"), int(nl), int(d), _stream())


def build_blocks_id(Tcw, hpose, hidx, mbear, rhov, okf, olm, ouv, Jp, resw, kslot, Hll, bl, Hpl, N, fx, cx, cy,
                    huber):
    _call("xcb_bk_build_blocks_id", _p(Tcw, F32, "Tcw"), _p(hpose, F32, "hpose"), _p(hidx, I32, "hidx"),
          _p(mbear, F32, "mbear"), _p(rhov, F32, "rhov"), _p(okf, I32, "okf"), _p(olm, I32, "olm"),
          _p(ouv, F32, "ouv"), _p(Jp, F32, "Jp"), _p(resw, F32, "resw"), _p(kslot, I32, "kslot"),
          _p(Hll, F32, "Hll"), _p(bl, F32, "bl"), _p(Hpl, F32, "Hpl"), int(N), float(fx), float(cx), float(cy),
          float(huber), _stream())


def landmark_prior_id(mb, rhov, m0, rho0, invsig, wbear, valid, Hll, bl, nl, huber):
    _call("xcb_bk_landmark_prior_id", _p(mb, F32, "mb"), _p(rhov, F32, "rhov"), _p(m0, F32, "m0"),
          _p(rho0, F32, "rho0"), _p(invsig, F32, "invsig"), _p(wbear, F32, "wbear"), _p(valid, F32, "valid"),
          _p(Hll, F32, "Hll"), _p(bl, F32, "bl"), int(nl), float(huber), _stream())


def pose_blocks_id(Jp, res, kslot, Hred, grad, N, d, n):
    _call("xcb_bk_pose_blocks_id", _p(Jp, F32, "Jp"), _p(res, F32, "res"), _p(kslot, I32, "kslot"),
          _p(Hred, F32, "Hred"), _p(grad, F32, "grad"), int(N), int(d), int(n), _stream())


def schur_pairs_id(Hpl, Hlli, kslot, olm, pa, pb, Hred, npair, d, n):
    _call("xcb_bk_schur_pairs_id", _p(Hpl, F32, "Hpl"), _p(Hlli, F32, "Hlli"), _p(kslot, I32, "kslot"),
          _p(olm, I32, "olm"), _p(pa, I32, "pa"), _p(pb, I32, "pb"), _p(Hred, F32, "Hred"), int(npair), int(d),
          int(n), _stream())


def schur_grad_id(Hpl, Hlli, bl, kslot, olm, g_, N, d):
    _call("xcb_bk_schur_grad_id", _p(Hpl, F32, "Hpl"), _p(Hlli, F32, "Hlli"), _p(bl, F32, "bl"),
          _p(kslot, I32, "kslot"), _p(olm, I32, "olm"), _p(g_, F32, "g"), int(N), int(d), _stream())


def backsub_id(Hpl, Hlli, bl, dxp, kslot, offs, dxl, nl, d):
    _call("xcb_bk_backsub_id", _p(Hpl, F32, "Hpl"), _p(Hlli, F32, "Hlli"), _p(bl, F32, "bl"), _p(dxp, F32, "dxp"),
          _p(kslot, I32, "kslot"), _p(offs, I32, "offs"), _p(dxl, F32, "dxl"), int(nl), int(d), _stream())
