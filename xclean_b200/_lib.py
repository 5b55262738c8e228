"""ctypes binding of libxcb200.so (the sm_100a kernels behind include/xcb200.h).

The library is built in-tree (xclean_b200/build.py).  There is no fallback: if it is missing, or no CUDA device is
visible, every entry point that needs it raises RuntimeError."""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxcb200.so")

XCB_OK = 0
XCB_ERR_ARG = -1
XCB_ERR_CUDA = -2
XCB_ERR_CAPACITY = -3
XCB_ERR_NOT_CALIBRATED = -4
XCB_ERR_DEVICE = -5

_lock = threading.Lock()
_LIB = None

c_int, c_double, c_float, c_void_p, c_size_t = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, \
    ctypes.c_size_t
P = c_void_p


class FrontBufs(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("counts", "kp", "desc", "d", "sig", "ok", "zn", "dy", "m0", "m1", "nmatch",
                                         "floor", "anypos")]


# name -> (restype, argtypes)
_SIGS = {
    "xcb_last_error": (ctypes.c_char_p, []),
    "xcb_version": (c_int, []),
    "xcb_peak_fma": (c_int, [c_int, c_int, P, P]),
    "xcb_front_create": (c_int, [c_int, c_int, c_int, c_int, ctypes.POINTER(c_void_p)]),
    "xcb_front_destroy": (None, [P]),
    "xcb_front_last_error": (ctypes.c_char_p, [P]),
    "xcb_front_device_bytes": (c_size_t, [P]),
    "xcb_front_set_calibration": (c_int, [P, c_int, c_int, c_int, c_int, P, P, c_double]),
    "xcb_front_response_host": (c_int, [P, P, c_int, c_int, P]),
    "xcb_front_noise_floor_host": (c_int, [P, P, P]),
    "xcb_front_blur_host": (c_int, [P, P, c_int, c_int, P]),
    "xcb_front_detect_host": (c_int, [P, P, c_int, c_int, P, P, P, P, P]),
    "xcb_front_describe_host": (c_int, [P, P, P, c_int, P]),
    "xcb_front_stereo_host": (c_int, [P, P, P, P, P, P, c_int, c_double, c_int, c_int, P, P, P, P, P]),
    "xcb_front_hamming_host": (c_int, [P, P, c_int, P, c_int, P, P, P, P]),
    "xcb_front_match_host": (c_int, [P, P, c_int, P, c_int, c_int, c_double, P, P, P]),
    "xcb_front_lk_check_host": (c_int, [P, P, P, c_int, P, P]),
    "xcb_front_pipeline_dev": (c_int, [P, P, P, c_int, c_int, c_int, c_int, c_int, c_int, P]),
    "xcb_front_buffers": (c_int, [P, ctypes.POINTER(FrontBufs)]),
    "xcb_front_pipeline_host": (c_int, [P, P, P, c_int, c_int, c_int, c_int, c_int, c_int, ctypes.POINTER(FrontBufs), P]),
    "xcb_front_pipeline_host_batches": (c_int, [P, P, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                                                ctypes.POINTER(FrontBufs), P]),
    "xcb_front_last_launches": (c_int, [P]),
    "xcb_front_set_tuning": (c_int, [P, c_int, c_int]),
    "xcb_front_sync_check": (c_int, [P, P]),
    "xcb_front_set_stage_timing": (c_int, [P, c_int]),
    "xcb_front_stage_times": (c_int, [P, P, P]),
}

FRONT_STAGES = ("response", "noise_floor", "candidates", "greedy", "orb", "stereo", "match")


class BaEngine(ctypes.Structure):
    _fields_ = [("P", c_int), ("sids", c_void_p), ("slot_n", c_void_p), ("M", ctypes.c_longlong), ("lid", c_void_p),
                ("uv", c_void_p), ("cam", c_void_p), ("valid", c_void_p), ("sig", c_void_p), ("n_lm", c_int),
                ("lm_alive", c_void_p), ("select", c_void_p), ("lm_host", c_void_p), ("lm_p", c_void_p),
                ("lm_rho_meas", c_void_p), ("lm_sig_lk", c_void_p), ("lm_span", c_void_p), ("prior_mode", c_int),
                ("kappa_d", c_double), ("fB", c_double), ("sig_px", c_double)]


class BaAssembled(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("counts", "alive", "src", "lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig",
                                         "lm_ob", "ob_pose", "ob_cam", "ob_z", "ob_isig", "ob_valid")]


class BaWindows(ctypes.Structure):
    _fields_ = [("nw", c_int)] + [(n, c_void_p) for n in (
        "P", "L", "slot_off", "lm_off", "hold", "order", "cam", "ext", "Rwb", "pwb", "lmp", "lm_host", "lm_mask",
        "rho_meas", "rho_isig", "lm_ob", "ob_pose", "ob_cam", "ob_z", "ob_isig", "ob_valid",
        "pr_m", "pr_nb", "pr_boff", "pr_soff", "pr_roff", "pr_blk", "pr_x0", "pr_S", "pr_r")]


XCB_TUNE_MM_LANES = 1
XCB_TUNE_STEREO_WARPS = 2
XCB_TUNE_STEREO_GROUP = 3
XCB_BA_FP64 = 0
XCB_BA_MIXED = 1
XCB_BA_NEWTON_POLISH = 0
XCB_BA_NEWTON_ADJOINT = 1
XCB_BA_NEWTON_POLISH_FIXED = 2
XCB_BA_STATUS_SCRATCH = -3
XCB_BA_STATUS_PRIOR = -4
_SIGS.update({
    "xcb_ba_scratch_bytes": (c_size_t, [c_int, c_int]),
    "xcb_ba_large_scratch_bytes": (c_size_t, [c_int, c_int, c_int]),
    "xcb_ba_gram_tc": (c_int, [P, c_int, c_int, P, P, P]),
    "xcb_ba_assemble_scratch_bytes": (c_size_t, [c_int, c_int, c_int]),
    "xcb_ba_assemble_dev": (c_int, [ctypes.POINTER(BaEngine), ctypes.POINTER(BaAssembled), P, c_size_t, P]),
    "xcb_ba_solve_windows_large_dev": (c_int, [ctypes.POINTER(BaWindows), c_int, c_int, P, c_int, c_int, c_int,
                                               c_double, c_int, P, P, c_int, P, c_size_t, P]),
    "xcb_ba_solve_windows_large_free_dev": (c_int, [ctypes.POINTER(BaWindows), c_int, c_int, P, c_int, c_int, c_int,
                                                    c_double, P, P, c_size_t, P, c_size_t, P]),
    "xcb_ba_solve_windows_dev": (c_int, [ctypes.POINTER(BaWindows), c_int, c_int, c_double, c_int, P, P, c_int, P,
                                         c_size_t, c_int, P]),
    "xcb_ba_newton_scratch_bytes": (c_size_t, [c_int, c_int]),
    "xcb_ba_newton_windows_dev": (c_int, [ctypes.POINTER(BaWindows), c_int, c_int, c_int, c_int, c_double, P, P, P,
                                          P, P, P, c_size_t, c_int, P]),
    "xcb_ba_solve_windows_free_dev": (c_int, [ctypes.POINTER(BaWindows), c_int, c_int, c_int, c_double, P, P,
                                              c_size_t, c_int, P]),
    "xcb_ba_noalloc_max_landmarks": (c_int, []),
    "xcb_ba_solve_windows_noalloc": (c_int, [ctypes.POINTER(BaWindows), c_int, c_int, c_int, c_double, c_int, P, P,
                                             c_int, c_int, P]),
})

# local-BA stage kernels (src/xclean/backend/kernels.py): device pointers, float32 scalars, stream last
c_ll = ctypes.c_longlong
_SIGS.update({
    "xcb_bk_build_blocks": (c_int, [P] * 11 + [c_int, c_float, c_float, c_float, c_float, P]),
    "xcb_bk_depth_prior": (c_int, [P] * 7 + [c_int, c_float, P]),
    "xcb_bk_inv3_damped": (c_int, [P, P, c_int, c_float, P]),
    "xcb_bk_schur_pairs": (c_int, [P] * 7 + [c_ll, c_int, c_int, P]),
    "xcb_bk_schur_grad": (c_int, [P] * 6 + [c_int, c_int, P]),
    "xcb_bk_pose_blocks": (c_int, [P] * 5 + [c_int, c_int, c_int, c_int, P]),
    "xcb_bk_chol_solve": (c_int, [P, P, P, c_int, P, c_int, P]),
    "xcb_bk_backsub": (c_int, [P] * 7 + [c_int, c_int, P]),
    "xcb_bk_build_blocks_id": (c_int, [P] * 14 + [c_int, c_float, c_float, c_float, c_float, P]),
    "xcb_bk_landmark_prior_id": (c_int, [P] * 9 + [c_int, c_float, P]),
    "xcb_bk_pose_blocks_id": (c_int, [P] * 5 + [c_int, c_int, c_int, P]),
    "xcb_bk_schur_pairs_id": (c_int, [P] * 7 + [c_ll, c_int, c_int, P]),
    "xcb_bk_schur_grad_id": (c_int, [P] * 6 + [c_int, c_int, P]),
    "xcb_bk_backsub_id": (c_int, [P] * 7 + [c_int, c_int, P]),
})

XCB_LBA_EUCLID = 0
XCB_LBA_INVDEPTH = 1
XCB_LBA_MAX_SLOTS = 64
XCB_LBA_MAX_TOUCHED = 32
LBA_STATS = 10


class LbaProblem(ctypes.Structure):
    _fields_ = ([("model", c_int), ("nk", c_int), ("nl", c_int), ("N", c_int)]
                + [(k, c_double) for k in ("fx", "cx", "cy", "huber", "rho_floor")]
                + [(k, c_void_p) for k in ("Tcw", "lm", "rho", "okf", "olm", "ouv", "offs", "hidx", "hpose",
                                           "free_mask", "p0", "p1", "p2", "p3", "p4")]
                + [("nrot", c_int)] + [(k, c_void_p) for k in ("rot_a", "rot_b", "rot_M", "rot_sig")])


_SIGS.update({
    "xcb_mm_create": (c_int, [c_int, c_int, c_int, c_int, c_int, P]),
    "xcb_mm_set_tuning": (c_int, [P, c_int, c_int]),
    "xcb_sgm_create": (c_int, [c_int, c_int, c_int, c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, P]),
    "xcb_sgm_destroy": (None, [P]),
    "xcb_sgm_last_error": (ctypes.c_char_p, [P]),
    "xcb_sgm_compute_dev": (c_int, [P, P, P, P, P, P]),
    "xcb_sgm_compute_host": (c_int, [P, P, P, P, P]),
    "xcb_sgm_buffers": (c_int, [P, P, P, P]),
    "xcb_sgm_read_volumes": (c_int, [P, P, P]),
    "xcb_sgm_set_stage_timing": (c_int, [P, c_int]),
    "xcb_sgm_stage_times": (c_int, [P, P, P]),
    "xcb_fast_scratch_bytes": (c_size_t, [c_int, c_int]),
    "xcb_fast_dev": (c_int, [P, c_int, c_int, c_int, c_int, c_int, P, P, P, P, c_size_t, P]),
    "xcb_fast_select_dev": (c_int, [P, P, P, c_int, c_int, c_int, c_int, c_int, P, P, P, P]),
    "xcb_pyr_tables": (c_int, [c_int, c_int, P, P]),
    "xcb_pyr_down_dev": (c_int, [P, c_int, c_int, P, c_int, c_int, P, P, P, P, P]),
    "xcb_orient_tables": (c_int, [P, P, P]),
    "xcb_ic_bins_dev": (c_int, [P, c_int, c_int, P, c_int, P, P, P, P, P, P, P]),
    "xcb_orb_steered_dev": (c_int, [P, c_int, c_int, c_int, P, c_int, P, P, P, P, P]),
    "xcb_blur_dev": (c_int, [P, c_int, c_int, P, c_int, c_int, P, P]),
    "xcb_orbx_create": (c_int, [c_int, c_int, c_int, c_double, c_int, c_int, c_int, c_int, P]),
    "xcb_orbx_destroy": (None, [P]),
    "xcb_orbx_last_error": (ctypes.c_char_p, [P]),
    "xcb_orbx_level": (c_int, [P, c_int, P, P, P, P, P]),
    "xcb_orbx_set_blur": (c_int, [P, c_int, c_int, c_int, P]),
    "xcb_orbx_set_patterns": (c_int, [P, P]),
    "xcb_orbx_detect_dev": (c_int, [P, P, P]),
    "xcb_orbx_launches": (c_int, [P]),
    "xcb_orbx_outputs": (c_int, [P, P, P, P, P, P, P, P]),
    "xcb_orbx_detect_host": (c_int, [P, P, P, P, P, P, P, P, P]),
    "xcb_orbx_read": (c_int, [P, P, P, P, P, P, P, P]),
    "xcb_orbx_read_level": (c_int, [P, c_int, P]),
    "xcb_mm_destroy": (c_int, [P]),
    "xcb_mm_last_error": (ctypes.c_char_p, [P]),
    "xcb_mm_grid_dims": (c_int, [P, P, P]),
    "xcb_mm_match_host": (c_int, [P, P, c_int, P, P, P, P, c_int, P, c_int, c_double, P, P, P, P]),
    "xcb_mm_match_dev": (c_int, [P, c_int, P, P, c_int, P, P, P, P, c_int, P, P, c_int, c_double, P, P, P, P]),
    "xcb_mm_sync": (c_int, [P, P]),
    "xcb_mm_predict_host": (c_int, [P, P, P, P, P, P, P, P, P, P] + [c_double] * 7 + [c_int, P, P, P, P, P]),
    "xcb_mm_predict_match_host": (c_int, [P, P, P, P, P, P, P, P, P, P] + [c_double] * 5
                                  + [c_int, P, c_int, P, P, c_int, P, c_double, P, P, P, P, P, P, P, P]),
})

_SIGS.update({
    "xcb_ba_linearise_windows_dev": (c_int, [ctypes.POINTER(BaWindows), c_int, P, c_int, P, P, c_size_t, c_int, P]),
    "xcb_ba_posefree_host": (c_int, [c_int, P, P, P, P, c_int, P, P, P, P, P] + [c_double] * 6
                             + [c_int, c_double, P, P, P, P, P]),
})

_SIGS.update({
    "xcb_lba_workspace_bytes": (c_size_t, [ctypes.POINTER(LbaProblem)]),
    "xcb_lba_solve": (c_int, [ctypes.POINTER(LbaProblem), c_int, c_double, P, P, c_size_t, P]),
})


def declared_symbols():
    """Every entry point the header declares (the loader binds exactly these)."""
    return sorted(_SIGS)


def lib():
    """The loaded library; RuntimeError when it is not built."""
    global _LIB
    with _lock:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError("xclean_b200: %s is not built (run python -m xclean_b200.build or "
                                   "__graft_entry__.build())" % LIB_PATH)
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _LIB = L
    return _LIB


def check(rc, handle=None, what="xcb"):
    if rc == XCB_OK:
        return
    L = lib()
    msg = (L.xcb_front_last_error(handle) if handle else L.xcb_last_error()) or b""
    msg = msg.decode(errors="replace")
    if rc == XCB_ERR_CAPACITY:
        raise ValueError("%s: %s" % (what, msg))
    raise RuntimeError("%s failed (%d): %s" % (what, rc, msg))


def ptr(a):
    """Data pointer of a numpy array (or None)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)
