"""torchlpc_b200 — B200-native (sm_100a) differentiable time-varying all-pole filter.

Drop-in for the ``sample_wise_lpc`` / ``linear_recurrence`` path of
DiffAPF/torchlpc (torchlpc/__init__.py:28-104): same functions, argument
meaning, shapes and error behaviour, computed by hand-written CUDA kernels
behind the C ABI of ``liblpc_b200`` (include/lpc_b200.h).  CUDA tensors only;
there is no CPU fallback.
"""
from __future__ import annotations

from typing import Optional, Tuple, Union

import torch

from . import _ops
from ._ops import EXTENSION_LOADED, available_algos, check_status, get_algo, set_algo
from .core import LPC, LPCBoundary, LPCCheckpointed, LPCRagged
from .recurrence import Recurrence

__all__ = ["sample_wise_lpc", "linear_recurrence", "LPC", "Recurrence", "EXTENSION_LOADED",
           "set_algo", "get_algo", "available_algos", "sample_wise_lpc_ragged", "LPCRagged",
           "set_checkpoint_segment", "LPCCheckpointed", "set_checkpointing", "get_checkpointing", "LPCBoundary",
           "check_status"]


def linear_recurrence(a: torch.Tensor, x: torch.Tensor, zi: Optional[torch.Tensor] = None) -> torch.Tensor:
    """y[n] = x[n] + a[n] * y[n-1], y[-1] = zi (torchlpc/__init__.py:31-60).

    Shapes: a (B,T), x (B,T), zi (B,) (defaults to zeros).
    """
    assert a.shape == x.shape
    assert a.ndim == 2
    assert x.ndim == 2
    B, _ = a.shape
    if zi is None:
        zi = a.new_zeros(B)
    else:
        assert zi.shape == (B,)
    return Recurrence.apply(a, x, zi)  # type: ignore


def _time_invariant_source(a: torch.Tensor) -> Optional[torch.Tensor]:
    """For coefficients broadcast over time (stride 0 along T, e.g.
    ``a0[:, None, :].expand(-1, T, -1)``) return the (B, N) tensor they view, so
    that the fused time-invariant kernels run and the coefficient gradient
    reaches ``a0`` as a (B, N) reduction instead of a materialised (B, T, N)
    tensor.  Returns None when the pattern is not recognised."""
    try:
        if a.dim() != 3 or a.shape[1] <= 1 or a.stride(1) != 0:
            return None
        if torch._C._functorch.is_functorch_wrapped_tensor(a):
            return None
        B, _, N = a.shape
        if not a.requires_grad:
            return a[:, 0, :]
        base = a._base
        if base is None or base.data_ptr() != a.data_ptr():
            return None
        if base.shape == (B, N) and (B == 1 or base.stride(0) == a.stride(0)) and \
                (N == 1 or base.stride(1) == a.stride(2)):
            return base
        if base.shape == (B, 1, N) and (B == 1 or base.stride(0) == a.stride(0)) and \
                (N == 1 or base.stride(2) == a.stride(2)):
            return base.squeeze(1)
    except (RuntimeError, AttributeError):
        return None
    return None


_CHECKPOINT_SEGMENT = 0
_CHECKPOINTING = "auto"
# Signals of at least this many samples keep chunk-boundary states instead of y
# under the "auto" checkpointing mode.
CHECKPOINT_MIN_SAMPLES = 1 << 20


def set_checkpointing(mode: str) -> None:
    """Boundary-state checkpointing inside the chunked kernels
    (``LPCBoundary``): "auto" (default) for signals of at least 2^20 samples,
    "on" for every signal the chunked scan can take, "off" never.  It applies
    to time-varying (B,T,N) coefficients of order 2 to 32 under the "auto",
    "chunked" and "tuned" algorithms, when a gradient is wanted and no
    forward-mode AD or functorch transform is active; other calls keep y as
    torchlpc does."""
    global _CHECKPOINTING
    assert mode in ("auto", "on", "off"), mode
    _CHECKPOINTING = mode


def get_checkpointing() -> str:
    return _CHECKPOINTING


def _boundary_checkpoint(x: torch.Tensor, A: torch.Tensor, zi: torch.Tensor, T: int, order: int) -> bool:
    if _CHECKPOINTING == "off" or (_CHECKPOINTING == "auto" and T < CHECKPOINT_MIN_SAMPLES):
        return False
    if not (2 <= order <= 32) or A.dim() != 3 or A.stride(1) == 0 or not x.is_cuda:
        return False
    if get_algo() == "plain" or x.dtype not in (torch.float32, torch.float64):
        return False
    if not torch.is_grad_enabled() or not any(t.requires_grad for t in (x, A, zi)):
        return False
    try:
        from torch._C._functorch import is_functorch_wrapped_tensor
        from torch.autograd.forward_ad import unpack_dual

        for t in (x, A, zi):
            if is_functorch_wrapped_tensor(t) or unpack_dual(t).tangent is not None:
                return False
    except (ImportError, RuntimeError):
        return False
    return True


def set_checkpoint_segment(samples: int) -> None:
    """Boundary-state checkpointing for long signals: when ``samples`` > 0,
    ``sample_wise_lpc`` on signals longer than that keeps the N-sample state
    entering every segment of ``samples`` samples instead of the output y, and
    its backward recomputes y segment by segment (``LPCCheckpointed``).  0
    (the default) turns it off; segments shorter than the filter order are not
    checkpointed.  For plain reverse-mode autograd (no forward AD, vmap or
    double backward through the checkpointed filter).
    """
    global _CHECKPOINT_SEGMENT
    assert samples >= 0
    _CHECKPOINT_SEGMENT = int(samples)


def sample_wise_lpc(
    x: torch.Tensor,
    a: torch.Tensor,
    zi: Optional[torch.Tensor] = None,
    return_zf: bool = False,
) -> Union[torch.Tensor, Tuple[torch.Tensor, torch.Tensor]]:
    """Sample-wise all-pole (LPC) filtering (torchlpc/__init__.py:63-104).

    y[b,t] = x[b,t] - sum_{i=1..N} a[b,t,i-1] * y[b,t-i], with zi[b,k] = y[b,-1-k].

    Shapes: x (B,T), a (B,T,N), zi (B,N) (defaults to zeros).  Returns y (B,T),
    and with ``return_zf`` also the final delay values ``y[:, -N:].flip(1)``.
    """
    assert x.shape[0] == a.shape[0]
    assert x.shape[1] == a.shape[1]
    assert x.ndim == 2
    assert a.ndim == 3

    B, T, order = a.shape
    if zi is None:
        zi = a.new_zeros(B, order)
    else:
        assert zi.shape == (B, order)

    if order == 1:
        y = linear_recurrence(-a.squeeze(2), x, zi.squeeze(1))
    else:
        src = _time_invariant_source(a)
        A = src if src is not None else a
        if _CHECKPOINT_SEGMENT and T > _CHECKPOINT_SEGMENT >= order:
            y = LPCCheckpointed.apply(x, A, zi, _CHECKPOINT_SEGMENT)
        elif _boundary_checkpoint(x, A, zi, T, order):
            y = LPCBoundary.apply(x, A, zi, _ops.checkpoint_chunk(T, order, x.dtype))
        else:
            y = LPC.apply(x, A, zi)

    if return_zf:
        return y, y[:, -order:].flip(1)
    return y


def sample_wise_lpc_ragged(
    x: torch.Tensor,
    a: torch.Tensor,
    offsets: torch.Tensor,
    zi: Optional[torch.Tensor] = None,
) -> torch.Tensor:
    """All-pole filtering of a ragged batch in one launch (no padding).

    Signal s occupies samples ``offsets[s]:offsets[s+1]`` of x (S,) and rows of
    a (S, N); zi (nsig, N) defaults to zeros.  Equivalent to running
    ``sample_wise_lpc`` on each signal separately; orders up to 32.
    """
    assert x.ndim == 1 and a.ndim == 2 and a.shape[0] == x.shape[0]
    assert offsets.ndim == 1 and offsets.dtype == torch.int64
    nsig, order = offsets.shape[0] - 1, a.shape[1]
    if zi is None:
        zi = a.new_zeros(nsig, order)
    else:
        assert zi.shape == (nsig, order)
    return LPCRagged.apply(x, a, offsets, zi)
