"""xclean_b200: the per-frame hot path of xclean (stereo frontend + sliding-window BA linear solve) on B200.

Subpackages mirror the reference modules they replace:
    xclean_b200.front.gpu_front   <- xclean.front.gpu_front
    xclean_b200.backend.kernels   <- xclean.backend.kernels (the local-BA stage kernels)
    xclean_b200.backend.local_ba  <- xclean.backend.ba (_solve_gpu, _solve_gpu_id, build_pairs, warmup)
    xclean_b200.backend.ba        <- xclean.vio.window.solve, batched over many windows in one launch
The device code is libxcb200.so (xclean_b200/csrc, include/xcb200.h), called through ctypes."""

__version__ = "0.1.0"
