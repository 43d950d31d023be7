"""Loader of the native operator library and the algorithm switch.

There is no fallback: when the extension cannot be loaded, ``EXTENSION_LOADED``
is False and every filter call raises.
"""
from __future__ import annotations

import os

import torch

ALGOS = {"auto": 0, "plain": 1, "chunked": 2, "ti": 3}

try:
    from . import _C  # noqa: F401  (registers torch.ops.torchlpc_b200.*)

    EXTENSION_LOADED = True
    _LOAD_ERROR = None
except ImportError as e:  # pragma: no cover - exercised only without a build
    EXTENSION_LOADED = False
    _LOAD_ERROR = e

TUNED = -1  # "tuned": per-shape choice from torchlpc_b200.tune
_algo = TUNED if os.environ.get("LPC_B200_ALGO") == "tuned" else ALGOS[os.environ.get("LPC_B200_ALGO", "auto")]
_LIB = None


def _lib():
    """The C ABI library the operators are linked against (same instance)."""
    import ctypes
    from pathlib import Path

    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(str(Path(__file__).resolve().parent / "liblpc_b200.so"))
        lib.lpc_b200_set_chunk_length.argtypes = [ctypes.c_int64]
        lib.lpc_b200_chunk_length.restype = ctypes.c_int64
        lib.lpc_b200_checkpoint_chunk.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
        lib.lpc_b200_checkpoint_chunk.restype = ctypes.c_int64
        _LIB = lib
    return _LIB


def set_chunk_length(samples: int) -> None:
    """Target chunk length of the chunked scan (0 restores the default)."""
    _require()
    _lib().lpc_b200_set_chunk_length(int(samples))


def get_chunk_length() -> int:
    """The chunk-length setting (0: chosen per call by signal length)."""
    _require()
    return int(_lib().lpc_b200_chunk_length())


def set_algo(name: str) -> None:
    """Select the kernel family: "auto" (default), "plain", "chunked", "ti"
    (time-invariant coefficients only; other calls fall back as "auto") or
    "tuned" (the autotuner's choice per shape, tuning unseen shapes on first
    use)."""
    global _algo
    _algo = TUNED if name == "tuned" else ALGOS[name]


def get_algo() -> str:
    return "tuned" if _algo == TUNED else {v: k for k, v in ALGOS.items()}[_algo]


def _resolve(x, A):
    """Algorithm code for one call (the tuner's choice in "tuned" mode)."""
    if _algo != TUNED:
        return _algo
    from . import tune

    B, T = x.shape
    cfg = tune.choice(B, T, A.shape[-1], x.dtype, A.dim() == 2 or A.stride(1) == 0, x.device)
    set_chunk_length(cfg["chunk"])
    return ALGOS[cfg["algo"]]


def available_algos():
    """Kernel families this build can run ("auto" picks among them)."""
    return ["plain", "chunked", "ti"] if _CHUNKED else ["plain"]


_CHUNKED = True


def _require():
    if not EXTENSION_LOADED:
        raise RuntimeError(
            "torchlpc_b200 native extension is not loaded (build it with "
            f"`python -m torchlpc_b200.build`): {_LOAD_ERROR}")


def lpc(x, A, zi):
    _require()
    return torch.ops.torchlpc_b200.lpc(x, A, zi, _resolve(x, A))


def lpc_backward(grad_y, A, zi, y, need_A, need_zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_backward(grad_y, A, zi, y, need_A, need_zi, _resolve(y, A))


def scan(impulse, decay, init):
    _require()
    return torch.ops.torchlpc_b200.scan(impulse, decay, init, max(_algo, 0))


def scan_backward(grad_out, decay, init, out, need_decay, need_init):
    _require()
    return torch.ops.torchlpc_b200.scan_backward(grad_out, decay, init, out, need_decay, need_init, max(_algo, 0))


def checkpoint_chunk(T: int, N: int, dtype) -> int:
    """Chunk length a checkpointed forward and its backward share (the
    current chunk-length setting applied to signals of T samples)."""
    _require()
    return int(_lib().lpc_b200_checkpoint_chunk(0 if dtype == torch.float32 else 1, int(T), int(N)))


def lpc_checkpointed(x, A, zi, chunk):
    _require()
    return torch.ops.torchlpc_b200.lpc_checkpointed(x, A, zi, chunk)


def lpc_backward_checkpointed(grad_y, A, zi, x, states, chunk, need_A, need_zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_backward_checkpointed(grad_y, A, zi, x, states, chunk, need_A, need_zi)


def check_status(synchronize: bool = True) -> None:
    """Raise RuntimeError if a chunked kernel's bounded device-side wait gave
    up since the last check (its call's outputs are invalid).  Synchronises the
    current stream first unless ``synchronize`` is False; clears the word.
    Every operator call also checks it on entry, without synchronising."""
    _require()
    w = int(torch.ops.torchlpc_b200.check_status(bool(synchronize)))
    if w:
        raise RuntimeError(
            f"torchlpc_b200: a bounded device-side wait of a chunked kernel gave up (status word {w:#x}; "
            "1: a predecessor's flag never appeared, 2: inconsistent flags, 8: a ragged signal with a "
            "negative length); the outputs of that call are invalid")


def lpc_ragged(x, A, offsets, zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_ragged(x, A, offsets, zi)


def lpc_backward_ragged(grad_y, A, offsets, zi, y, need_A, need_zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_backward_ragged(grad_y, A, offsets, zi, y, need_A, need_zi)
