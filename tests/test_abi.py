"""The C-ABI library: it loads without a GPU, exports every function that
include/cgfdm_b200.h declares, and the ctypes binding covers them all.  No
compute entry point is called here."""
import ctypes
import os
import re

import pytest

cgfdm = pytest.importorskip("cgfdm")
from cgfdm import _lib  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cgfdm_b200.h")


def declared_functions():
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(cgfdm_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("cgfdm_create", "cgfdm_run", "cgfdm_propagate", "cgfdm_run_directory",
              "cgfdm_setup_from_directory", "cgfdm_destroy"):
        assert n in names


def test_library_exports_every_declared_function():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_function():
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_version_and_error_text_without_gpu():
    assert _lib.lib().cgfdm_version().decode().startswith("cgfdm")
    d = cgfdm.make_desc(0, 10, 10, 0, 100.0, 0.008, 10)
    h = ctypes.c_void_p()
    rc = _lib.lib().cgfdm_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == 1  # CGFDM_ERR_ARG: the grid must be non-empty (checked before any device)
    assert not h.value
    assert _lib.lib().cgfdm_last_error()
