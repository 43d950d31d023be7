"""Operator-level equivalence, in the form of the reference's
tests/test_extension.py: the order-1 scan and the LPC operator against the
FP64 oracle (the reference compared against its Numba kernels)."""
import numpy as np
import pytest
import torch

from oracle import lpc_oracle as O
from tests.test_grad import create_test_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo", [1, 2])
@pytest.mark.parametrize("samples", [64, 4097])
def test_scan_equiv(samples, algo):
    g = torch.Generator().manual_seed(samples)
    x = torch.randn(4, samples, generator=g)
    A = torch.rand(4, samples, generator=g) * 1.8 - 0.9
    zi = torch.randn(4, generator=g)
    ref = O.scan_forward(x, A, zi)
    out = torch.ops.torchlpc_b200.scan(x.cuda(), A.cuda(), zi.cuda(), algo)
    assert np.allclose(out.cpu().double().numpy(), ref, atol=5e-6)


@pytest.mark.parametrize("algo", [1, 2])
@pytest.mark.parametrize("samples", [1021, 4097])
def test_lpc_equiv(samples, algo):
    x, A, zi = create_test_inputs(4, samples, seed=samples)
    ref = O.lpc_forward(x, A, zi)
    out = torch.ops.torchlpc_b200.lpc(x.cuda(), A.cuda(), zi.cuda(), algo)
    assert np.allclose(out.cpu().numpy(), ref)
    out32 = torch.ops.torchlpc_b200.lpc(x.float().cuda(), A.float().cuda(), zi.float().cuda(), algo)
    assert O.normwise_err(out32, O.lpc_forward(x.float(), A.float(), zi.float())) < 1e-5
