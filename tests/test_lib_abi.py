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
