"""The C-ABI library loads without a GPU and exports every entry point the
header declares; the Python binding declares the same set."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mset_\w+)\s*\(", txt, flags=re.M))
    return names


def test_header_declares_entry_points():
    s = header_symbols()
    for must in ("mset_create", "mset_upload", "mset_run", "mset_error", "mset_batch_gradient"):
        assert must in s


def test_library_exports_every_declared_symbol():
    import mset_b200
    lib = mset_b200.load()
    out = subprocess.run(["nm", "-D", "--defined-only", mset_b200.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mset_\w+)", out))
    missing = header_symbols() - exported
    assert not missing, missing
    for name in header_symbols():
        assert hasattr(lib, name)


def test_binding_matches_header():
    from mset_b200._lib import SIGNATURES
    assert set(SIGNATURES) == header_symbols()


def test_create_without_gpu_fails_cleanly():
    import ctypes as C
    import mset_b200
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    lib = mset_b200.load()
    h = C.c_void_p()
    rc = lib.mset_create(0, C.byref(h))
    assert rc != 0 and not h.value
    assert b"CUDA" in lib.mset_last_error() or b"device" in lib.mset_last_error()


def test_implicit_session_is_null_before_upload():
    """mset_mex_session: the MEX-style global session does not exist until
    the first mset_mex_upload (no device work; runs without a GPU)"""
    import mset_b200
    lib = mset_b200.load()
    assert lib.mset_mex_session() is None
