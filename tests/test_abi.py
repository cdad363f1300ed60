"""The C ABI library loads and exports every function include/delta_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes

from delta_b200 import LIB_PATH, header_functions


def test_library_exports_every_header_function():
    assert LIB_PATH.exists(), "libdelta_b200.so not built"
    lib = ctypes.CDLL(str(LIB_PATH))
    names = header_functions()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    from delta_b200 import lib

    assert b"sm_100a" in lib().delta_version()


def test_python_signatures_cover_header():
    from delta_b200._lib import SIGNATURES

    assert set(header_functions()) <= set(SIGNATURES)
