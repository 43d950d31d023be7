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

_algo = ALGOS[os.environ.get("LPC_B200_ALGO", "auto")]


def set_algo(name: str) -> None:
    """Select the kernel family: "auto" (default), "plain", "chunked" or "ti"
    (time-invariant coefficients only; other calls fall back as "auto")."""
    global _algo
    _algo = ALGOS[name]


def get_algo() -> str:
    return {v: k for k, v in ALGOS.items()}[_algo]


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
    return torch.ops.torchlpc_b200.lpc(x, A, zi, _algo)


def lpc_backward(grad_y, A, zi, y, need_A, need_zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_backward(grad_y, A, zi, y, need_A, need_zi, _algo)


def scan(impulse, decay, init):
    _require()
    return torch.ops.torchlpc_b200.scan(impulse, decay, init, _algo)


def scan_backward(grad_out, decay, init, out, need_decay, need_init):
    _require()
    return torch.ops.torchlpc_b200.scan_backward(grad_out, decay, init, out, need_decay, need_init, _algo)


def lpc_ragged(x, A, offsets, zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_ragged(x, A, offsets, zi)


def lpc_backward_ragged(grad_y, A, offsets, zi, y, need_A, need_zi):
    _require()
    return torch.ops.torchlpc_b200.lpc_backward_ragged(grad_y, A, offsets, zi, y, need_A, need_zi)
