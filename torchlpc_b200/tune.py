"""Autotuner: kernel family and chunk length per problem shape.

For a shape (B, T, N, dtype, time-invariant or not) it times one forward and
one fused backward of a synthetic stable filter of that shape for each
candidate -- the plain kernel, the chunked scan at several chunk lengths and,
for time-invariant coefficients, the time-invariant scan -- and keeps the
fastest.  Choices are cached per shape bucket (T and B rounded up to powers
of two) in memory and, when ``LPC_B200_TUNE_CACHE`` names a file, in that
JSON file across processes.  ``set_algo("tuned")`` makes every call use them.
"""
from __future__ import annotations

import json
import os
import threading
from typing import Dict, List, Optional, Tuple

import torch

from . import _ops

CHUNK_LENGTHS = (128, 256, 512)
_TABLE: Dict[str, dict] = {}
_LOCK = threading.RLock()
_LOADED = False


def _bucket(n: int) -> int:
    return 1 << max(0, int(n - 1).bit_length())


def key(B: int, T: int, N: int, dtype: torch.dtype, time_invariant: bool) -> str:
    return f"N{N}:T{_bucket(T)}:B{_bucket(B)}:{str(dtype).split('.')[-1]}:{'ti' if time_invariant else 'tv'}"


def candidates(N: int, time_invariant: bool) -> List[Tuple[str, int]]:
    c = [("plain", 0)]
    if N <= 32:
        c += [("chunked", L) for L in CHUNK_LENGTHS]
        if time_invariant:
            c.append(("ti", 0))
    return c


def _cache_path() -> Optional[str]:
    return os.environ.get("LPC_B200_TUNE_CACHE") or None


def _load() -> None:
    global _LOADED
    if _LOADED:
        return
    _LOADED = True
    p = _cache_path()
    if p and os.path.exists(p):
        try:
            with open(p) as f:
                _TABLE.update(json.load(f))
        except (OSError, ValueError):
            pass


def _save() -> None:
    p = _cache_path()
    if not p:
        return
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(_TABLE, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def _problem(B, T, N, dtype, time_invariant, device):
    g = torch.Generator(device="cpu").manual_seed(1234)
    x = torch.randn(B, T, generator=g, dtype=torch.float64).to(device=device, dtype=dtype)
    gy = torch.randn(B, T, generator=g, dtype=torch.float64).to(device=device, dtype=dtype)
    # sum |a_i| < 1 keeps every filter stable
    shape = (B, N) if time_invariant else (B, T, N)
    A = (torch.rand(shape, generator=g, dtype=torch.float64) * (0.9 / N)).to(device=device, dtype=dtype)
    zi = torch.zeros(B, N, device=device, dtype=dtype)
    return x, A, zi, gy


def measure(B: int, T: int, N: int, dtype=torch.float32, time_invariant: bool = False, device="cuda",
            reps: int = 3) -> Dict[str, float]:
    """ms per fwd+bwd for every candidate on a synthetic problem of the shape."""
    x, A, zi, gy = _problem(B, T, N, dtype, time_invariant, device)
    old_algo, old_len = _ops.get_algo(), _ops.get_chunk_length()
    out: Dict[str, float] = {}
    try:
        for algo, L in candidates(N, time_invariant):
            _ops.set_algo(algo)
            _ops.set_chunk_length(L)

            def run():
                y = _ops.lpc(x, A, zi)
                _ops.lpc_backward(gy, A, zi, y, True, True)

            run()
            torch.cuda.synchronize(device)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(reps):
                run()
            e.record()
            torch.cuda.synchronize(device)
            out[f"{algo}:{L}"] = s.elapsed_time(e) / reps
    finally:
        _ops.set_algo(old_algo)
        _ops.set_chunk_length(old_len)
    return out


def autotune(B: int, T: int, N: int, dtype=torch.float32, time_invariant: bool = False, device="cuda",
             reps: int = 3) -> dict:
    """Time the candidates for this shape and record the fastest."""
    times = measure(B, T, N, dtype, time_invariant, device, reps)
    best = min(times, key=times.get)
    algo, L = best.split(":")
    cfg = {"algo": algo, "chunk": int(L), "ms": times[best], "times": times}
    with _LOCK:
        _load()
        _TABLE[key(B, T, N, dtype, time_invariant)] = cfg
        _save()
    return cfg


def lookup(B: int, T: int, N: int, dtype, time_invariant: bool) -> Optional[dict]:
    with _LOCK:
        _load()
        return _TABLE.get(key(B, T, N, dtype, time_invariant))


def choice(B: int, T: int, N: int, dtype, time_invariant: bool, device) -> dict:
    """The recorded choice for this shape; tunes it on first sight (on a
    bounded sample of the shape: at most 64 signals of at most 2^20 samples)."""
    cfg = lookup(B, T, N, dtype, time_invariant)
    if cfg is None:
        cfg = autotune(min(B, 64), min(T, 1 << 20), N, dtype, time_invariant, device)
        with _LOCK:
            _TABLE[key(B, T, N, dtype, time_invariant)] = cfg
            _save()
    return cfg


def table() -> Dict[str, dict]:
    with _LOCK:
        _load()
        return dict(_TABLE)
