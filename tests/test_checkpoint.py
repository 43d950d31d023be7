"""Boundary-state checkpointing: the backward recomputes y segment by segment
from saved N-sample entry states and must give the same gradients as the
fused backward on the saved y (LPC), including a last segment shorter than
the order and time-invariant coefficients."""
import pytest
import torch

import torchlpc_b200 as tl
from torchlpc_b200.synth import make_workload

pytestmark = pytest.mark.gpu


def _grads(x, A, zi, gy, segment, time_invariant=False):
    tl.set_checkpoint_segment(segment)
    try:
        xx, AA, zz = (t.detach().clone().requires_grad_(True) for t in (x, A, zi))
        T = xx.shape[1]
        Ae = AA[:, None, :].expand(-1, T, -1) if time_invariant else AA
        y = tl.sample_wise_lpc(xx, Ae, zz)
        (y * gy).sum().backward()
        return y.detach(), xx.grad, AA.grad, zz.grad
    finally:
        tl.set_checkpoint_segment(0)


@pytest.mark.parametrize("algo", ["chunked", "plain"])
@pytest.mark.parametrize("T,segment", [(12000, 3000), (9005, 3000), (6003, 2000)])
def test_checkpointed_backward_matches_saved_output(algo, T, segment):
    old = tl.get_algo()
    tl.set_algo(algo)
    try:
        w = make_workload("cfg3", seed=4, device="cuda", B=2, T=T)
        ref = _grads(w["x"], w["A"], w["zi"], w["gy"], 0)
        ck = _grads(w["x"], w["A"], w["zi"], w["gy"], segment)
    finally:
        tl.set_algo(old)
    for a, b in zip(ck, ref):
        den = b.abs().max().item()
        assert (a - b).abs().max().item() <= 1e-4 * max(den, 1.0)


def test_checkpointed_time_invariant():
    w = make_workload("cfg5", seed=2, device="cuda", B=3, T=10000)
    ref = _grads(w["x"], w["A"], w["zi"], w["gy"], 0, time_invariant=True)
    ck = _grads(w["x"], w["A"], w["zi"], w["gy"], 4096, time_invariant=True)
    for a, b in zip(ck, ref):
        den = b.abs().max().item()
        assert (a - b).abs().max().item() <= 1e-4 * max(den, 1.0)
