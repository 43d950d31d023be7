"""``Recurrence``: the order-1 recurrence out[t] = decay[t]*out[t-1] + impulse[t].

Interface follows torchlpc.recurrence.Recurrence (torchlpc/recurrence.py:73-168):
``Recurrence.apply(decay, impulse, initial_state)`` with (B,T), (B,T), (B,).
Both directions run on the CUDA kernels of ``torch.ops.torchlpc_b200``
(order-1 instances of the all-pole kernels).  With ``create_graph=True`` the
backward is composed from ``Recurrence.apply`` on reversed time so that it is
itself differentiable.
"""
from __future__ import annotations

from typing import Any, List, Optional, Tuple

import torch
import torch.nn.functional as F
from torch.autograd import Function

from . import _ops


class Recurrence(Function):
    @staticmethod
    def forward(decay: torch.Tensor, impulse: torch.Tensor, initial_state: torch.Tensor) -> torch.Tensor:
        return _ops.scan(impulse, decay, initial_state)

    @staticmethod
    def setup_context(ctx: Any, inputs: List[Any], output: Any) -> Any:
        decay, _, initial_state = inputs
        ctx.save_for_backward(decay, initial_state, output)
        ctx.save_for_forward(decay, initial_state, output)

    @staticmethod
    def backward(ctx: Any, grad_out: torch.Tensor
                 ) -> Tuple[Optional[torch.Tensor], Optional[torch.Tensor], Optional[torch.Tensor]]:
        decay, initial_state, out = ctx.saved_tensors
        need_d, need_i, need_0 = ctx.needs_input_grad
        if torch.is_grad_enabled():
            # grad_impulse[t] = grad_out[t] + decay[t+1] * grad_impulse[t+1]
            shifted = F.pad(decay[:, 1:], (0, 1))
            gi = Recurrence.apply(shifted.flip(1).conj_physical(), grad_out.flip(1),
                                  grad_out.new_zeros(grad_out.shape[0])).flip(1)
            g0 = decay[:, 0].conj_physical() * gi[:, 0] if need_0 else None
            gd = None
            if need_d:
                prev = torch.cat([initial_state.unsqueeze(1), out[:, :-1]], dim=1)
                gd = prev.conj_physical() * gi
            return gd, (gi if need_i else None), g0
        gi, gd, g0 = _ops.scan_backward(grad_out, decay, initial_state, out, bool(need_d), bool(need_0))
        return (gd if need_d else None, gi if need_i else None, g0 if need_0 else None)

    @staticmethod
    def jvp(ctx: Any, grad_decay: torch.Tensor, grad_impulse: torch.Tensor,
            grad_initial_state: torch.Tensor) -> torch.Tensor:
        decay, initial_state, out = ctx.saved_tensors
        fwd_init = grad_initial_state if grad_initial_state is not None else torch.zeros_like(initial_state)
        fwd_impulse = grad_impulse if grad_impulse is not None else torch.zeros_like(out)
        if grad_decay is not None:
            prev = torch.cat([initial_state.unsqueeze(1), out[:, :-1]], dim=1)
            fwd_impulse = fwd_impulse + prev * grad_decay
        return Recurrence.apply(decay, fwd_impulse, fwd_init)

    @staticmethod
    def vmap(info, in_dims, *args):
        def front(t, bdim):
            if bdim is None:
                return t.expand(info.batch_size, *t.shape)
            return t.movedim(bdim, 0)

        decay, impulse, init = (t.reshape(-1, *t.shape[2:]) for t in map(front, args, in_dims))
        out = Recurrence.apply(decay, impulse, init)
        return out.reshape(info.batch_size, -1, *out.shape[1:]), 0
