"""The C-ABI library loads and exports every entry point include/xcb200.h declares (no GPU call)."""
import ctypes
import os
import re

from xclean_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "xcb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(xcb_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_function():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert set(header_functions()) == set(_lib.declared_symbols())


def test_loader_binds_without_a_device():
    L = _lib.lib()
    assert L.xcb_version() >= 1


def test_host_side_size_rules_without_a_device():
    """Scratch sizes and argument checks that run on the host before any device call."""
    L = _lib.lib()
    for nw, Lt in ((1, 1), (4, 1000), (256, 412517)):
        need = ((3 * Lt + 31) // 32 * 32 + 118 * Lt) * 8 + 256        # counter, trial states, back-substitution records
        assert int(L.xcb_ba_scratch_bytes(nw, Lt)) >= need
        assert int(L.xcb_ba_newton_scratch_bytes(nw, Lt)) >= 22 * 8 * Lt + 256
    h = ctypes.c_void_p()
    for w, hgt in ((8193, 376), (47, 376), (1241, 47)):      # outside 48 <= width <= 8192, 48 <= height
        rc = L.xcb_front_create(w, hgt, 2048, 4, ctypes.byref(h))
        assert rc == _lib.XCB_ERR_ARG and not h.value
        assert b"bad size" in L.xcb_last_error()


def test_map_matcher_argument_checks_without_a_device():
    """xcb_mm_create refuses bad sizes and grids larger than one CTA's shared memory before any device call."""
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.xcb_mm_create(0, 48, 1, 16, 16, ctypes.byref(h)) == _lib.XCB_ERR_ARG and not h.value
    assert L.xcb_mm_create(64, 48, 0, 16, 16, ctypes.byref(h)) == _lib.XCB_ERR_ARG
    assert L.xcb_mm_create(8192, 8192, 1, 16, 16, ctypes.byref(h)) == _lib.XCB_ERR_ARG
    assert b"49152" in L.xcb_last_error()
    assert L.xcb_mm_match_host(None, None, 0, None, None, None, None, 0, None, 0, 1.0, None, None, None,
                               None) == _lib.XCB_ERR_ARG


def test_new_entry_points_refuse_bad_arguments_without_a_device():
    """The prediction, pose-free, linearisation and batched-pipeline entries check their arguments on the host
    before any device call."""
    L = _lib.lib()
    z = [None] * 9
    assert L.xcb_mm_predict_host(None, *z, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0, None, None, None, None,
                                 None) == _lib.XCB_ERR_ARG
    assert L.xcb_mm_predict_match_host(None, *z, 1.0, 1.0, 1.0, 1.0, 1.0, 0, None, 0, None, None, 0, None, 1.0,
                                       None, None, None, None, None, None, None, None) == _lib.XCB_ERR_ARG
    assert L.xcb_mm_match_dev(None, 1, None, None, 0, None, None, None, None, 1, None, None, 0, 1.0, None, None,
                              None, None) == _lib.XCB_ERR_ARG
    assert L.xcb_ba_linearise_windows_dev(None, 1, None, 0, None, None, 0, 0, None) == _lib.XCB_ERR_ARG
    assert L.xcb_ba_posefree_host(0, None, None, None, None, 0, None, None, None, None, None, 1.0, 1.0, 1.0, 1.0, 1.0,
                                  1.345, 0, 0.0, None, None, None, None, None) == _lib.XCB_ERR_ARG
    assert b"bad window" in L.xcb_last_error()
    assert L.xcb_front_pipeline_host_batches(None, None, None, 1, 1, 100, 4, 0, 96, 0, None,
                                             None) == _lib.XCB_ERR_ARG


def test_newton_and_constant_landmark_entries_refuse_bad_arguments_without_a_device():
    """xcb_ba_newton_windows_dev and xcb_ba_solve_windows_large_free_dev check their arguments and scratch sizes on
    the host before any device call.  Every call below fails one of those checks (or has no window), so none reaches
    the device and the placeholder pointers are never dereferenced."""
    L = _lib.lib()
    E, C, OK = _lib.XCB_ERR_ARG, _lib.XCB_ERR_CAPACITY, _lib.XCB_OK
    w = _lib.BaWindows()
    w.nw = 4
    fake = ctypes.c_void_p(4096)
    need = int(L.xcb_ba_newton_scratch_bytes(4, 0))

    def nt(wp=ctypes.byref(w), max_slots=10, mode=_lib.XCB_BA_NEWTON_POLISH, steps=3, maxit=60, gpose=None,
           gtheta=None, scratch=fake, nbytes=need):
        return L.xcb_ba_newton_windows_dev(wp, max_slots, mode, steps, maxit, 1e-12, gpose, gtheta, None, None, fake,
                                           scratch, nbytes, 0, None)

    assert nt(wp=None) == E
    assert nt(scratch=None) == E
    assert nt(max_slots=0) == C and nt(max_slots=21) == C
    assert nt(mode=7) == E
    assert nt(mode=_lib.XCB_BA_NEWTON_ADJOINT) == E and b"adjoint outputs" in L.xcb_last_error()
    assert nt(steps=-1) == E and nt(maxit=0) == E
    assert nt(nbytes=256) == C and b"xcb_ba_newton_scratch_bytes" in L.xcb_last_error()   # below the copies' region
    w0 = _lib.BaWindows()
    w0.nw = 0
    assert nt(wp=ctypes.byref(w0)) == OK                              # nothing to do: no device call

    Lt, slots = 1000, 40
    big = int(L.xcb_ba_large_scratch_bytes(4, slots, Lt))
    nbig = 256 + 19 * Lt * 8

    def lf(wp=ctypes.byref(w), chunks=fake, nchunks=8, max_slots=10, iters=20, sl=slots, lt=Lt, scratch=fake,
           nbytes=big, nscr=fake, nnbytes=nbig):
        return L.xcb_ba_solve_windows_large_free_dev(wp, sl, lt, chunks, nchunks, max_slots, iters, 1e-4, fake,
                                                     scratch, nbytes, nscr, nnbytes, None)

    assert lf(wp=None) == E and lf(nscr=None) == E and lf(scratch=None) == E
    assert lf(chunks=None) == E
    assert lf(max_slots=21) == C
    assert lf(sl=-1) == E and lf(lt=-1) == E and lf(nchunks=-1) == E and lf(iters=-1) == E
    assert lf(nbytes=big - 1) == C
    assert lf(nnbytes=nbig - 8) == C and b"19 doubles per landmark" in L.xcb_last_error()
    wp = _lib.BaWindows()
    wp.nw = 4
    wp.pr_m = 4096
    assert lf(wp=ctypes.byref(wp)) == E and b"marginal prior" in L.xcb_last_error()
    assert lf(wp=ctypes.byref(w0)) == OK
