"""Gradient checks in the form of the reference's tests/test_grad.py, on CUDA.

gradcheck (with forward-mode AD) and gradgradcheck of LPC.apply at B=4, T=32,
N=2 over the {A, zi} requires_grad grid; float32 vs float64 forward; the same
checks on the order-1 Recurrence at T=123.  Complex inputs are not supported
by torchlpc_b200 (the reference's cmplx=True cases are out of scope).
"""
import math

import pytest
import torch
from torch.autograd.gradcheck import gradcheck, gradgradcheck

import torchlpc_b200 as tl
from torchlpc_b200.core import LPC
from torchlpc_b200.recurrence import Recurrence

pytestmark = pytest.mark.gpu


def get_random_biquads(g):
    mag = torch.rand(1, dtype=torch.double, generator=g)
    phase = torch.rand(1, dtype=torch.double, generator=g) * math.pi
    return torch.tensor([-mag * torch.cos(phase) * 2, mag ** 2], dtype=torch.double)


def create_test_inputs(batch_size, samples, seed=0):
    g = torch.Generator().manual_seed(seed)
    s, e = get_random_biquads(g), get_random_biquads(g)
    A = torch.stack([torch.linspace(float(s[i]), float(e[i]), samples, dtype=torch.double)
                     for i in range(2)]).T.unsqueeze(0).repeat(batch_size, 1, 1)
    x = torch.randn(batch_size, samples, dtype=torch.double, generator=g)
    zi = torch.randn(batch_size, 2, dtype=torch.double, generator=g)
    return x, A, zi


@pytest.fixture(params=["plain", "chunked"])
def algo(request):
    old = tl.get_algo()
    tl.set_algo(request.param)
    yield request.param
    tl.set_algo(old)


@pytest.mark.parametrize("a_requires_grad", [True, False])
@pytest.mark.parametrize("zi_requires_grad", [True, False])
def test_low_order(a_requires_grad, zi_requires_grad, algo):
    x, A, zi = (t.cuda() for t in create_test_inputs(4, 32))
    A.requires_grad = a_requires_grad
    x.requires_grad = True
    zi.requires_grad = zi_requires_grad
    assert gradcheck(LPC.apply, (x, A, zi), check_forward_ad=True)
    assert gradgradcheck(LPC.apply, (x, A, zi))


@pytest.mark.parametrize("order", [3, 16, 40])
def test_higher_order_gradcheck(order, algo):
    g = torch.Generator().manual_seed(order)
    B, T = 2, 48
    x = torch.randn(B, T, dtype=torch.double, generator=g).cuda().requires_grad_()
    A = ((torch.rand(B, T, order, dtype=torch.double, generator=g) * 2 - 1) * 0.5 / order).cuda()
    A.requires_grad_()
    zi = torch.randn(B, order, dtype=torch.double, generator=g).cuda().requires_grad_()
    assert gradcheck(LPC.apply, (x, A, zi), check_forward_ad=True)


def test_float64_vs_32_cuda(algo):
    x, A, zi = (t.cuda() for t in create_test_inputs(4, 32))
    y64 = LPC.apply(x, A, zi)
    y32 = LPC.apply(x.float(), A.float(), zi.float())
    assert torch.allclose(y64, y32.double(), atol=1e-6), torch.max(torch.abs(y64 - y32.double()))


@pytest.mark.parametrize("a_requires_grad", [True, False])
@pytest.mark.parametrize("zi_requires_grad", [True, False])
def test_parallel_scan(a_requires_grad, zi_requires_grad, algo):
    g = torch.Generator().manual_seed(1)
    B, T = 2, 123
    x = torch.randn(B, T, dtype=torch.double, generator=g).cuda()
    A = (torch.rand(B, T, dtype=torch.double, generator=g) * 2 - 1).cuda()
    zi = torch.randn(B, dtype=torch.double, generator=g).cuda()
    A.requires_grad = a_requires_grad
    x.requires_grad = True
    zi.requires_grad = zi_requires_grad
    assert gradcheck(Recurrence.apply, (A, x, zi), check_forward_ad=True)
    assert gradgradcheck(Recurrence.apply, (A, x, zi))
