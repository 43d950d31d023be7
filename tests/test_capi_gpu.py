"""Direct calls through the C ABI (ctypes, raw device pointers, the current
torch stream) compared with the FP64 oracle."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import lpc_oracle as O
from torchlpc_b200.synth import make_workload

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parents[1] / "torchlpc_b200" / "liblpc_b200.so"
i64, vp, sz = C.c_int64, C.c_void_p, C.c_size_t


@pytest.fixture(scope="module")
def lib():
    L = C.CDLL(str(LIB))
    L.lpc_b200_forward.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, i64, i64, i64, i64, vp, sz, vp]
    L.lpc_b200_backward.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, i64, i64, i64, i64, i64,
                                    vp, sz, vp]
    L.lpc_b200_forward_workspace_size.argtypes = [C.c_int, C.c_int, i64, i64, i64, i64]
    L.lpc_b200_forward_workspace_size.restype = sz
    L.lpc_b200_backward_workspace_size.argtypes = [C.c_int, C.c_int, i64, i64, i64, i64]
    L.lpc_b200_backward_workspace_size.restype = sz
    return L


def p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("algo", [1, 2])
def test_forward_backward_through_c_abi(lib, algo):
    w = make_workload("cfg2", seed=3, B=4, T=3000)
    x, A, zi, gy = (w[k].cuda() for k in ("x", "A", "zi", "gy"))
    B, T, N = A.shape
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    y = torch.empty_like(x)
    wsb = lib.lpc_b200_forward_workspace_size(0, algo, B, T, N, N)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    assert lib.lpc_b200_forward(0, algo, p(x), p(A), p(zi), p(y), B, T, N, T * N, N, p(ws), wsb, st) == 0
    gx, gA, gzi = torch.empty_like(x), torch.empty_like(A), torch.empty_like(zi)
    wsb = lib.lpc_b200_backward_workspace_size(0, algo, B, T, N, N)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    assert lib.lpc_b200_backward(0, algo, p(gy), p(A), p(zi), p(y), p(gx), p(gA), p(gzi),
                                 B, T, N, T * N, N, p(ws), wsb, st) == 0
    torch.cuda.synchronize()
    yo = O.lpc_forward(w["x"], w["A"], w["zi"])
    gxo, gAo, gzio = O.lpc_backward(w["gy"], w["A"], w["zi"], yo)
    assert O.normwise_err(y, yo) < 1e-4
    assert O.normwise_err(gx, gxo) < 1e-4
    assert O.normwise_err(gA, gAo) < 1e-4
    assert O.normwise_err(gzi, gzio) < 1e-4


def test_workspace_too_small_is_reported(lib):
    x = torch.zeros(2, 1 << 16, device="cuda")
    A = torch.zeros(2, 1 << 16, 16, device="cuda")
    y = torch.empty_like(x)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    need = lib.lpc_b200_forward_workspace_size(0, 2, 2, 1 << 16, 16, 16)
    if need == 0:
        pytest.skip("chunked path needs no workspace here")
    rc = lib.lpc_b200_forward(0, 2, p(x), p(A), None, p(y), 2, 1 << 16, 16, 16 << 16, 16, None, 0, st)
    assert rc == 3


def test_bounded_lookback_wait_reports_timeout_and_context_survives(lib):
    """A chunked forward whose ticket queue skips batch 0: batch 1 waits for a
    flag nothing sets.  The wait gives up after its spin limit, the status word
    carries code 1, the call returns LPC_ERR_TIMEOUT, and the context still runs
    ordinary work afterwards (no trap, no hang)."""
    lib.lpc_b200_selftest_workspace_size.restype = sz
    lib.lpc_b200_selftest_timeout.argtypes = [vp, sz, C.c_uint, C.POINTER(C.c_uint), vp]
    lib.lpc_b200_workspace_status.argtypes = [vp, C.POINTER(C.c_uint), vp]
    wsb = lib.lpc_b200_selftest_workspace_size()
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    status = C.c_uint(0)
    rc = lib.lpc_b200_selftest_timeout(p(ws), wsb, 2000, C.byref(status), st)
    assert rc == 5, rc
    assert status.value & 1
    again = C.c_uint(0)
    assert lib.lpc_b200_workspace_status(p(ws), C.byref(again), st) == 0 and again.value == status.value
    # the context is intact: an ordinary call through the same library works
    w = make_workload("cfg3", seed=1, B=2, T=40000)
    x, A, zi = (w[k].cuda() for k in ("x", "A", "zi"))
    B, T, N = A.shape
    y = torch.empty_like(x)
    wsb = lib.lpc_b200_forward_workspace_size(0, 2, B, T, N, N)
    ws2 = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    assert lib.lpc_b200_forward(0, 2, p(x), p(A), p(zi), p(y), B, T, N, T * N, N, p(ws2), wsb, st) == 0
    ok = C.c_uint(7)
    assert lib.lpc_b200_workspace_status(p(ws2), C.byref(ok), st) == 0 and ok.value == 0
    assert O.normwise_err(y, O.lpc_forward(w["x"], w["A"], w["zi"])) < 1e-4
    # the give-up also reached the process-wide error word (when the operator
    # layer installed one): consume it so later calls in this process start clean
    import torchlpc_b200 as tl
    try:
        tl.check_status()
    except RuntimeError:
        pass
