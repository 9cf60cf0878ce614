"""The C-ABI library loads and exports every entry point include/dsb200.h
declares; the ctypes binding declares exactly those (no GPU needed)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dsb200.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char\*)\s+(dsb_\w+)\s*\(", src,
                                 re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "dsb_corr_tc" in names and "dsb_detect" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from dsb200 import _lib
    if not os.path.exists(_lib.SO_PATH):
        pytest.skip("native library not built")
    so = ctypes.CDLL(_lib.SO_PATH)
    missing = [n for n in _declared() if not hasattr(so, n)]
    assert not missing, missing
    assert so.dsb_version() == 1


def test_binding_covers_header():
    from dsb200 import _lib
    assert sorted(_lib.declared_symbols()) == _declared()


def test_binding_argument_counts_match_header():
    """Every ctypes signature has as many arguments as the header's
    prototype (ctypes itself does not check)."""
    from dsb200 import _lib
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    for name, args in _lib._SIGNATURES.items():
        m = re.search(r"\b" + name + r"\s*\(([^;]*?)\)\s*;", src, re.S)
        assert m, name
        params = [q for q in m.group(1).split(",") if q.strip() and q.strip() != "void"]
        assert len(params) == len(args), (name, len(params), len(args))


def test_strerror_without_gpu():
    from dsb200 import _lib
    if not os.path.exists(_lib.SO_PATH):
        pytest.skip("native library not built")
    L = _lib.lib()
    assert L.dsb_strerror(0) == b"ok"
    assert L.dsb_strerror(4).startswith(b"device-side")


def test_no_cpu_path():
    """Every op refuses CPU tensors instead of computing on the host."""
    import torch
    from dsb200.corr import FastCorrKernel
    with pytest.raises(ValueError, match="CUDA"):
        FastCorrKernel(torch.device("cpu"))
