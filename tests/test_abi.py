"""The C-ABI library loads and exports every symbol include/qxmd_b200.h
declares (no compute: no GPU here)."""
import ctypes
import os
import re

from qxmd_b200 import build, lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "qxmd_b200.h")


def header_symbols():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qx\w+)\s*\(", txt)) - {"qx_ctx"})


def test_library_exports_every_declared_symbol():
    so = build.build()
    L = ctypes.CDLL(so)
    syms = header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(lib.EXPORTS) == syms


def test_version_and_error_string():
    L = lib.lib()
    assert L.qx_version() == 1
    assert isinstance(lib.last_error(), str)


def test_create_rejects_bad_sizes():
    import numpy as np
    L = lib.lib()
    h = ctypes.c_void_p()
    ij = np.zeros(3, dtype=np.int32)
    dk = np.zeros(4)
    # FFT length with a prime factor 11 is refused before any device work
    rc = L.qx_create(ctypes.byref(h), 0, 11, 12, 12, 1, ij, dk, 2, None)
    assert rc == 1
    assert "2,3,5,7" in lib.last_error()
