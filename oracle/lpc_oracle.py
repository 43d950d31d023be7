"""ctypes bindings of the FP64 C oracle (oracle/lpc_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  All functions take and return
numpy float64 arrays (inputs are converted with ``np.ascontiguousarray``) and
follow the reference algorithm cited in lpc_oracle.c.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import build_oracle

_lib = None
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int64)


def _load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build_oracle()))
        i64 = C.c_int64
        _lib.oracle_lpc_forward.argtypes = [i64, i64, i64, _D, _D, i64, i64, _D, _D]
        _lib.oracle_lpc_backward.argtypes = [i64, i64, i64, _D, _D, i64, i64, _D, _D, _D, _D, _D, _D]
        _lib.oracle_lpc_forward_ragged.argtypes = [i64, i64, _I, _D, _D, _D, _D]
        _lib.oracle_lpc_backward_ragged.argtypes = [i64, i64, _I, _D, _D, _D, _D, _D, _D, _D]
        _lib.oracle_scan_forward.argtypes = [i64, i64, _D, _D, _D, _D]
        _lib.oracle_scan_backward.argtypes = [i64, i64, _D, _D, _D, _D, _D, _D, _D]
    return _lib


def _f64(a):
    if a is None:
        return None
    if hasattr(a, "detach"):  # torch tensor
        a = a.detach().cpu().double().numpy()
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(_D)


def _coeff_view(A, B, T, N):
    """Return (contiguous fp64 buffer, as_b, as_t) for A of shape (B,T,N) or (B,N)."""
    A = _f64(A)
    if A.ndim == 2:  # time-invariant (B, N)
        assert A.shape == (B, N)
        return A, N, 0
    assert A.shape == (B, T, N), (A.shape, (B, T, N))
    return A, T * N, N


def lpc_forward(x, A, zi=None):
    """y = all-pole filter of x; A (B,T,N) or time-invariant (B,N)."""
    x = _f64(x)
    B, T = x.shape
    N = (A.shape[-1])
    Ab, as_b, as_t = _coeff_view(A, B, T, N)
    zi = _f64(zi)
    y = np.empty((B, T), np.float64)
    _load().oracle_lpc_forward(B, T, N, _p(x), _p(Ab), as_b, as_t, _p(zi), _p(y))
    return y


def lpc_backward(gy, A, zi, y, want_gA=True, want_gzi=True):
    """Returns (gx, gA, gzi).  gA is (B,T,N), or (B,N) summed over T when A is (B,N)."""
    gy = _f64(gy)
    y = _f64(y)
    B, T = gy.shape
    N = A.shape[-1]
    Ab, as_b, as_t = _coeff_view(A, B, T, N)
    zi = _f64(zi)
    gx = np.empty((B, T), np.float64)
    gA = ga = gzi = None
    if want_gA:
        if as_t == 0:
            ga = np.empty((B, N), np.float64)
        else:
            gA = np.empty((B, T, N), np.float64)
    if want_gzi:
        gzi = np.empty((B, N), np.float64)
    _load().oracle_lpc_backward(B, T, N, _p(gy), _p(Ab), as_b, as_t, _p(zi), _p(y),
                                _p(gx), _p(gA), _p(ga), _p(gzi))
    return gx, (ga if as_t == 0 else gA), gzi


def lpc_forward_ragged(x, A, zi, offsets):
    x, A, zi = _f64(x), _f64(A), _f64(zi)
    off = np.ascontiguousarray(np.asarray(offsets), dtype=np.int64)
    B = off.shape[0] - 1
    N = A.shape[-1]
    y = np.empty_like(x)
    _load().oracle_lpc_forward_ragged(B, N, off.ctypes.data_as(_I), _p(x), _p(A), _p(zi), _p(y))
    return y


def lpc_backward_ragged(gy, A, zi, y, offsets):
    gy, A, zi, y = _f64(gy), _f64(A), _f64(zi), _f64(y)
    off = np.ascontiguousarray(np.asarray(offsets), dtype=np.int64)
    B = off.shape[0] - 1
    N = A.shape[-1]
    gx = np.empty_like(gy)
    gA = np.empty_like(A)
    gzi = np.empty((B, N), np.float64)
    _load().oracle_lpc_backward_ragged(B, N, off.ctypes.data_as(_I), _p(gy), _p(A), _p(zi), _p(y),
                                       _p(gx), _p(gA), _p(gzi))
    return gx, gA, gzi


def scan_forward(impulse, decay, init=None):
    """out[t] = decay[t]*out[t-1] + impulse[t]."""
    impulse, decay, init = _f64(impulse), _f64(decay), _f64(init)
    B, T = impulse.shape
    out = np.empty_like(impulse)
    _load().oracle_scan_forward(B, T, _p(impulse), _p(decay), _p(init), _p(out))
    return out


def scan_backward(grad_out, decay, init, out):
    """Returns (grad_impulse, grad_decay, grad_init)."""
    grad_out, decay, init, out = _f64(grad_out), _f64(decay), _f64(init), _f64(out)
    B, T = grad_out.shape
    gi = np.empty_like(grad_out)
    gd = np.empty_like(grad_out)
    ginit = np.empty((B,), np.float64)
    _load().oracle_scan_backward(B, T, _p(grad_out), _p(decay), _p(init), _p(out), _p(gi), _p(gd), _p(ginit))
    return gi, gd, ginit


def normwise_err(a, ref) -> float:
    """max|a - ref| / max|ref| (0 when both are empty or ref is all zeros and a == ref)."""
    a = _f64(a)
    ref = _f64(ref)
    if ref.size == 0:
        return 0.0
    den = np.abs(ref).max()
    num = np.abs(a - ref).max()
    if den == 0.0:
        return float(num)
    return float(num / den)
