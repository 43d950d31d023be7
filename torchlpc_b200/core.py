"""``LPC``: the all-pole filter as a torch.autograd.Function.

Interface and semantics follow torchlpc.core.LPC (torchlpc/core.py:159-265):
``LPC.apply(x, A, zi)`` with x (B,T), A (B,T,N), zi (B,N); it saves (A, zi, y)
for backward and forward-mode AD, defines ``jvp`` and ``vmap``.  As an
extension, A may also be a time-invariant (B,N) tensor.

Backward: one fused CUDA kernel produces grad_x, grad_A and grad_zi
(``torch.ops.torchlpc_b200.lpc_backward``).  When a graph of the backward is
requested (``create_graph=True``, e.g. gradgradcheck) the backward is instead
composed from differentiable pieces around ``LPC.apply`` itself: the reversed
filter over the coefficient diagonal A[t+1+i, i], gathered from a
time-padded A.
"""
from __future__ import annotations

from typing import Any, List, Optional, Tuple

import torch
import torch.nn.functional as F
from torch.autograd import Function

from . import _ops


def _lagged_outputs(y: torch.Tensor, zi: torch.Tensor, order: int) -> torch.Tensor:
    """(B,T,N) with [b,t,i] = y[b,t-1-i] (zi[b,k] standing for y[b,-1-k])."""
    return torch.cat([zi.flip(1), y[:, :-1]], dim=1).unfold(1, order, 1).flip(2)


def _composed_backward(grad_y, A, zi, y, needs):
    """Differentiable backward (used only when create_graph=True)."""
    B, T = grad_y.shape
    order = A.shape[-1]
    A3 = A[:, None, :].expand(B, T, order) if A.dim() == 2 else A
    # D[t', i] = A[t'-N+1+i, i] for t' = 0..T+N-1 (t = t'-N), zero outside [0, T)
    A_pad = F.pad(A3, (0, 0, order, order + 1))
    tp = torch.arange(T + order, device=A.device)
    idx = (tp[:, None] + 1 + torch.arange(order, device=A.device)[None, :])
    D = A_pad.gather(1, idx[None].expand(B, -1, -1))
    gy_ext = F.pad(grad_y, (order, 0))
    u = LPC.apply(gy_ext.flip(1), D.flip(1).conj_physical(), torch.zeros_like(zi))
    gx_ext = u.flip(1)
    grad_x = gx_ext[:, order:] if needs[0] else None
    grad_zi = gx_ext[:, :order].flip(1) if needs[2] else None
    grad_A = None
    if needs[1]:
        gA = -_lagged_outputs(y, zi, order).conj_physical() * gx_ext[:, order:].unsqueeze(2)
        grad_A = gA.sum(1) if A.dim() == 2 else gA
    return grad_x, grad_A, grad_zi


class LPC(Function):
    @staticmethod
    def forward(x: torch.Tensor, A: torch.Tensor, zi: torch.Tensor) -> torch.Tensor:
        return _ops.lpc(x, A, zi)

    @staticmethod
    def setup_context(ctx: Any, inputs: List[Any], output: Any) -> Any:
        _, A, zi = inputs
        y = output
        ctx.save_for_backward(A, zi, y)
        ctx.save_for_forward(A, zi, y)

    @staticmethod
    def backward(ctx: Any, grad_y: torch.Tensor
                 ) -> Tuple[Optional[torch.Tensor], Optional[torch.Tensor], Optional[torch.Tensor]]:
        A, zi, y = ctx.saved_tensors
        needs = ctx.needs_input_grad
        if torch.is_grad_enabled():
            return _composed_backward(grad_y, A, zi, y, needs)
        gx, gA, gzi = _ops.lpc_backward(grad_y, A, zi, y, bool(needs[1]), bool(needs[2]))
        return (gx if needs[0] else None, gA if needs[1] else None, gzi if needs[2] else None)

    @staticmethod
    def jvp(ctx: Any, grad_x: torch.Tensor, grad_A: torch.Tensor, grad_zi: torch.Tensor) -> torch.Tensor:
        A, zi, y = ctx.saved_tensors
        order = A.shape[-1]
        fwd_zi = grad_zi if grad_zi is not None else torch.zeros_like(zi)
        fwd_x = grad_x if grad_x is not None else torch.zeros_like(y)
        if grad_A is not None:
            lagged = _lagged_outputs(y, zi, order)
            dA = grad_A[:, None, :] if grad_A.dim() == 2 else grad_A
            fwd_x = fwd_x - torch.sum(lagged * dA, dim=2)
        return LPC.apply(fwd_x, A, fwd_zi)

    @staticmethod
    def vmap(info, in_dims, *args):
        def front(t, bdim):
            if bdim is None:
                return t.expand(info.batch_size, *t.shape)
            return t.movedim(bdim, 0)

        x, A, zi = (t.reshape(-1, *t.shape[2:]) for t in map(front, args, in_dims))
        y = LPC.apply(x, A, zi)
        return y.reshape(info.batch_size, -1, *y.shape[1:]), 0


class LPCRagged(Function):
    """The all-pole filter over a ragged batch: signals concatenated along time.

    ``LPCRagged.apply(x, A, offsets, zi)`` with x (S,), A (S,N), offsets
    (nsig+1,) int64 on x's device (signal s is samples offsets[s] to
    offsets[s+1]) and zi (nsig,N).  No counterpart in the reference, which
    filters a dense (B,T) batch (torchlpc/core.py:159-229).  The backward is
    the fused CUDA kernel; it is not itself differentiable.
    """

    @staticmethod
    def forward(x: torch.Tensor, A: torch.Tensor, offsets: torch.Tensor, zi: torch.Tensor) -> torch.Tensor:
        return _ops.lpc_ragged(x, A, offsets, zi)

    @staticmethod
    def setup_context(ctx: Any, inputs: List[Any], output: Any) -> Any:
        _, A, offsets, zi = inputs
        ctx.save_for_backward(A, offsets, zi, output)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx: Any, grad_y: torch.Tensor):
        A, offsets, zi, y = ctx.saved_tensors
        needs = ctx.needs_input_grad
        gx, gA, gzi = _ops.lpc_backward_ragged(grad_y, A, offsets, zi, y, bool(needs[1]), bool(needs[3]))
        return (gx if needs[0] else None, gA if needs[1] else None, None, gzi if needs[3] else None)


class LPCBoundary(Function):
    """The filter with boundary-state checkpointing in the kernels.

    ``LPCBoundary.apply(x, A, zi, chunk)``: same result as ``LPC.apply(x, A,
    zi)``.  torchlpc's LPC saves (A, zi, y) for the backward
    (torchlpc/core.py:179-184); this one saves (x, A, zi) and the N-sample
    state entering every half of every ``chunk``-sample chunk of the scan,
    which the checkpointed forward kernel writes beside y (2N values per
    chunk).  The backward recomputes y from those states with one exact pass
    over independent half-chunks, then runs the fused backward kernel, so y is
    not kept alive between forward and backward.  Time-varying (B,T,N)
    coefficients of order up to 32; not itself differentiable (no
    forward-mode AD or double backward).
    """

    @staticmethod
    def forward(ctx: Any, x: torch.Tensor, A: torch.Tensor, zi: torch.Tensor, chunk: int) -> torch.Tensor:
        y, states = _ops.lpc_checkpointed(x, A, zi, chunk)
        ctx.save_for_backward(x, A, zi, states)
        ctx.chunk = chunk
        return y

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx: Any, grad_y: torch.Tensor):
        x, A, zi, states = ctx.saved_tensors
        needs = ctx.needs_input_grad
        gx, gA, gzi = _ops.lpc_backward_checkpointed(grad_y, A, zi, x, states, ctx.chunk, bool(needs[1]),
                                                     bool(needs[2]))
        return (gx if needs[0] else None, gA if needs[1] else None, gzi if needs[2] else None, None)


class LPCCheckpointed(Function):
    """The filter with boundary-state checkpointing for long signals, by segments.

    ``LPCCheckpointed.apply(x, A, zi, segment)``: same result as
    ``LPC.apply(x, A, zi)``, but instead of the output y (B,T) it keeps the
    N-sample state entering every segment of ``segment`` samples (torchlpc's
    LPC saves y, core.py:179-184).  The backward walks the segments from last
    to first: it recomputes a segment's outputs from its saved entry state (one
    forward call), runs the fused backward on it, and carries the adjoint of the
    segment's entry state (its grad_zi) into the last N output gradients of the
    segment before it.  Costs one extra forward pass; keeps x instead of y, so
    it saves memory when the caller holds x anyway; y then exists only for one
    segment at a time during the backward.  Not itself differentiable.
    """

    @staticmethod
    def forward(x: torch.Tensor, A: torch.Tensor, zi: torch.Tensor, segment: int) -> torch.Tensor:
        return _ops.lpc(x, A, zi)

    @staticmethod
    def setup_context(ctx: Any, inputs: List[Any], output: Any) -> Any:
        x, A, zi, segment = inputs
        y = output
        N = A.shape[-1]
        T = y.shape[1]
        # entry state of segment k >= 1: zi convention, state[j] = y[s-1-j]
        states = [zi] + [y[:, s - N:s].flip(1) for s in range(segment, T, segment)]
        ctx.save_for_backward(x, A, zi, torch.stack(states))
        ctx.segment = segment

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx: Any, grad_y: torch.Tensor):
        x, A, zi, states = ctx.saved_tensors
        needs = ctx.needs_input_grad
        seg = ctx.segment
        B, T = x.shape
        N = A.shape[-1]
        ti = A.dim() == 2
        gx = torch.empty_like(x) if needs[0] else None
        gA = (torch.zeros_like(A) if ti else torch.empty_like(A)) if needs[1] else None
        carry = None  # grad_zi of the segment after the current one
        starts = list(range(0, T, seg))
        for k in reversed(range(len(starts))):
            s = starts[k]
            e = min(s + seg, T)
            Ak = A if ti else A[:, s:e]
            zk = states[k]
            yk = _ops.lpc(x[:, s:e].contiguous(), Ak, zk)
            gyk = grad_y[:, s:e].contiguous()
            if carry is not None:  # the next segment starts from this one's last N outputs
                gyk = gyk.clone()
                gyk[:, -N:] += carry.flip(1)
            gxk, gAk, carry = _ops.lpc_backward(gyk, Ak, zk, yk, gA is not None, True)
            if gx is not None:
                gx[:, s:e] = gxk
            if gA is not None:
                if ti:
                    gA += gAk
                else:
                    gA[:, s:e] = gAk
        return gx, gA, carry if needs[2] else None, None
