"""jacfwd (forward-mode AD + vmap) vs .backward(), as the reference's
tests/test_vmap.py, on CUDA; the LPC case uses a time-invariant A broadcast
with expand (the reference idiom, tests/test_vmap.py:41)."""
import pytest
import torch
import torch.nn.functional as F
from torch.func import jacfwd

import torchlpc_b200 as tl
from torchlpc_b200.core import LPC
from torchlpc_b200.recurrence import Recurrence
from tests.test_grad import create_test_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo", ["plain", "chunked"])
def test_vmap(algo):
    tl.set_algo(algo)
    try:
        samples = 40
        x, A, zi = (t.cuda() for t in create_test_inputs(4, samples))
        y = torch.randn_like(x)
        A = A[:, 0, :].clone()
        A.requires_grad = True
        zi.requires_grad = True
        x.requires_grad = True
        args = (x, A, zi)

        def func(x, A, zi):
            return F.mse_loss(LPC.apply(x, A[:, None, :].expand(-1, samples, -1), zi), y)

        jacs = jacfwd(func, argnums=tuple(range(len(args))))(*args)
        loss = func(*args)
        loss.backward()
        for jac, arg in zip(jacs, args):
            assert torch.allclose(jac, arg.grad)
    finally:
        tl.set_algo("auto")


@pytest.mark.parametrize("algo", ["plain", "chunked"])
def test_parallel_scan_vmap(algo):
    tl.set_algo(algo)
    try:
        g = torch.Generator().manual_seed(3)
        x = torch.randn(3, 255, dtype=torch.double, generator=g).cuda()
        A = (torch.rand(3, 255, dtype=torch.double, generator=g) * 2 - 1).cuda()
        zi = torch.randn(3, dtype=torch.double, generator=g).cuda()
        y = torch.randn(3, 255, dtype=torch.double, generator=g).cuda()
        for t in (A, x, zi):
            t.requires_grad = True
        args = (x, A, zi)

        def func(x, A, zi):
            return F.mse_loss(Recurrence.apply(A, x, zi), y)

        jacs = jacfwd(func, argnums=tuple(range(len(args))))(*args)
        loss = func(*args)
        loss.backward()
        for jac, arg in zip(jacs, args):
            assert torch.allclose(jac, arg.grad)
    finally:
        tl.set_algo("auto")
