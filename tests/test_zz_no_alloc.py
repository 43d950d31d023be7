"""The forward entry point that allocates nothing (lpc_b200_forward_noalloc).

It exists for callers that cannot allocate device memory: code that must not
call an allocator (a real-time audio thread, a host callback) or an FFI
binding without a memory manager.  Its scratch is an array inside the library
instead of a caller-supplied workspace.  This test calls it through the C ABI
and checks it against lpc_b200_forward (chunked algorithm, workspace
allocated here) on two calls in a row with different inputs, so that contents
the shared array keeps from the previous call cannot leak into the next.
The file is named to be collected last.
"""
import ctypes as C
from pathlib import Path

import pytest
import torch

from oracle import lpc_oracle as O
from torchlpc_b200.synth import make_workload

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parents[1] / "torchlpc_b200" / "liblpc_b200.so"
i64, vp, sz = C.c_int64, C.c_void_p, C.c_size_t
TOL = 1e-4  # normwise, as the other float32 parity tests


@pytest.fixture(scope="module")
def lib():
    L = C.CDLL(str(LIB))
    L.lpc_b200_forward.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, i64, i64, i64, i64, vp, sz, vp]
    L.lpc_b200_forward_workspace_size.argtypes = [C.c_int, C.c_int, i64, i64, i64, i64]
    L.lpc_b200_forward_workspace_size.restype = sz
    L.lpc_b200_forward_noalloc.argtypes = [C.c_int, vp, vp, vp, vp, i64, i64, i64, i64, i64, vp]
    L.lpc_b200_noalloc_status.argtypes = [C.POINTER(C.c_uint), vp]
    return L


def ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def test_noalloc_matches_workspace_entry_point_twice(lib):
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for seed, (cfg, B, T) in enumerate([("cfg3", 4, 1 << 17), ("cfg2", 3, 20000)]):
        w = make_workload(cfg, seed=100 + seed, B=B, T=T)
        x, A, zi = (w[k].cuda() for k in ("x", "A", "zi"))
        B, T, N = A.shape
        y_ref = torch.empty_like(x)
        wsb = lib.lpc_b200_forward_workspace_size(0, 2, B, T, N, N)
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
        assert lib.lpc_b200_forward(0, 2, ptr(x), ptr(A), ptr(zi), ptr(y_ref), B, T, N, T * N, N,
                                    ptr(ws), wsb, st) == 0
        y = torch.full_like(x, float("nan"))
        assert lib.lpc_b200_forward_noalloc(0, ptr(x), ptr(A), ptr(zi), ptr(y), B, T, N, T * N, N, st) == 0
        torch.cuda.synchronize()
        assert O.normwise_err(y, y_ref) < TOL
        assert O.normwise_err(y, O.lpc_forward(w["x"], w["A"], w["zi"])) < TOL


@pytest.mark.parametrize("dtype,code,tol", [(torch.float32, 0, 1e-4), (torch.float64, 1, 1e-10)])
@pytest.mark.parametrize("with_zi", [True, False])
@pytest.mark.parametrize("time_invariant", [False, True])
def test_noalloc_dtypes_initial_conditions_and_strides(lib, dtype, code, tol, with_zi, time_invariant):
    """float32 and float64, zi given or NULL, dense (B,T,N) coefficients or a
    stride-0 (B,N) set broadcast over time; two calls in a row, each checked
    against lpc_b200_forward and the FP64 oracle, and the array's status
    word read back through lpc_b200_noalloc_status."""
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for seed in (0, 1):
        cfg = "cfg5" if time_invariant else "cfg3"
        w = make_workload(cfg, seed=200 + seed, B=3, T=30000 + 7 * seed, dtype=dtype)
        x, A = w["x"].cuda(), w["A"].cuda()
        zi = w["zi"].cuda() if with_zi else None
        B, T = x.shape
        N = A.shape[-1]
        sb, stt = (N, 0) if time_invariant else (T * N, N)
        y_ref = torch.empty_like(x)
        wsb = lib.lpc_b200_forward_workspace_size(code, 2, B, T, N, stt)
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
        assert lib.lpc_b200_forward(code, 2, ptr(x), ptr(A), ptr(zi), ptr(y_ref), B, T, N, sb, stt,
                                    ptr(ws), wsb, st) == 0
        y = torch.full_like(x, float("nan"))
        assert lib.lpc_b200_forward_noalloc(code, ptr(x), ptr(A), ptr(zi), ptr(y), B, T, N, sb, stt, st) == 0
        status = C.c_uint(7)
        assert lib.lpc_b200_noalloc_status(C.byref(status), st) == 0 and status.value == 0
        assert O.normwise_err(y, y_ref) < tol
        assert O.normwise_err(y, O.lpc_forward(w["x"], w["A"], w["zi"] if with_zi else None)) < tol


def test_noalloc_rejects_problems_beyond_its_scratch(lib):
    x = torch.zeros(4, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    B, T, N = 64, 1 << 20, 16  # needs tens of MiB of scratch
    rc = lib.lpc_b200_forward_noalloc(0, ptr(x), ptr(x), None, ptr(x), B, T, N, T * N, N, st)
    assert rc == 3  # LPC_ERR_WORKSPACE; nothing was launched
    rc = lib.lpc_b200_forward_noalloc(0, ptr(x), ptr(x), None, ptr(x), 1, 100, 40, 4000, 40, st)
    assert rc == 2  # LPC_ERR_UNSUPPORTED: no chunked kernel above order 32
