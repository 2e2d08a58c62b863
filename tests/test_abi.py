"""The C-ABI library loads and exports every symbol declared in include/ (CPU, no compute)."""
import ctypes
import os
import re

from ccsd_gpu_b200 import _native
from tests.conftest import ROOT


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, f)).read(), flags=re.S)
            names |= set(re.findall(r"\b(ccsd_b200_\w+)\s*\(", txt))
    return names


def test_library_exports_declared_symbols():
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared_symbols()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(lib, n), n
    assert names <= set(_native.SIGNATURES), names - set(_native.SIGNATURES)


def test_last_error_callable_without_gpu():
    assert isinstance(_native.load().ccsd_b200_last_error(), bytes)
