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
