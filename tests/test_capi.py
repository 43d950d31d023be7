"""The C ABI library loads and exports every symbol include/lpc_b200.h declares;
argument validation happens on the host (no GPU needed for these calls)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "lpc_b200.h"
LIB = ROOT / "torchlpc_b200" / "liblpc_b200.so"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(lpc_b200_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        from torchlpc_b200.build import build_lib
        build_lib()
    return C.CDLL(str(LIB))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ["lpc_b200_forward", "lpc_b200_backward", "lpc_b200_scan",
                     "lpc_b200_scan_backward", "lpc_b200_forward_workspace_size",
                     "lpc_b200_backward_workspace_size", "lpc_b200_status_string"]:
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    lib.lpc_b200_status_string.restype = C.c_char_p
    assert lib.lpc_b200_status_string(0) == b"ok"
    assert b"workspace" in lib.lpc_b200_status_string(3)
    assert lib.lpc_b200_version() >= 100


def test_invalid_arguments_rejected_on_host(lib):
    i64, vp, sz = C.c_int64, C.c_void_p, C.c_size_t
    lib.lpc_b200_forward.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, i64, i64, i64, i64, vp, sz, vp]
    dummy = C.c_void_p(16)
    # bad dtype
    assert lib.lpc_b200_forward(7, 0, dummy, dummy, None, dummy, 1, 1, 2, 2, 2, None, 0, None) == 1
    # order 0 and order above the limit
    assert lib.lpc_b200_forward(0, 0, dummy, dummy, None, dummy, 1, 1, 0, 0, 0, None, 0, None) == 1
    assert lib.lpc_b200_forward(0, 0, dummy, dummy, None, dummy, 1, 1, 5000, 5000, 5000, None, 0, None) == 1
    # NULL input pointers with work to do
    assert lib.lpc_b200_forward(0, 0, None, dummy, None, dummy, 1, 4, 2, 8, 2, None, 0, None) == 1
    # row stride smaller than the order
    assert lib.lpc_b200_forward(0, 0, dummy, dummy, None, dummy, 1, 4, 4, 16, 2, None, 0, None) == 1
    # empty problems are valid no-ops
    assert lib.lpc_b200_forward(0, 0, None, None, None, None, 0, 0, 2, 0, 2, None, 0, None) == 0
