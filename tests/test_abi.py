"""The C-ABI library loads on a machine without a GPU and exports every function include/ifea_gpu.h declares."""
import ctypes
import os
import re

from impressionfea_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "ifea_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ifea\w*)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert len(names) > 30
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"missing exports: {missing}"


def test_wrapper_signatures_cover_the_header():
    assert set(_declared()) <= set(_lib.SIGNATURES)


def test_version_string_without_a_gpu():
    assert b"sm_100a" in _lib.lib().ifea_version()
