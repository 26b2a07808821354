"""The C-ABI library loads and exports every entry point include/granb200.h declares
(no device calls: this runs without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "liggghts-public_b200", "libgranb200.so")
HDR = os.path.join(ROOT, "include", "granb200.h")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "liggghts-public_b200", "csrc")], check=True)
    return ctypes.CDLL(LIB)


def declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b(gb2_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_exported(lib):
    names = declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_python_front_end_matches_header():
    import granb200
    assert set(granb200.EXPORTS) <= set(declared())


def test_version_string(lib):
    lib.gb2_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.gb2_version()


def test_create_rejects_bad_params(lib):
    import granb200
    p = granb200.Params()
    p.ntypes = 0
    h = ctypes.c_void_p()
    assert lib.gb2_create(ctypes.byref(p), ctypes.byref(h)) == -1
