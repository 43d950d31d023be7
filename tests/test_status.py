"""Device-side failure reaches Python as an exception.

The chunked kernels' waits on other CTAs are bounded; a wait that gives up
records a code in the call's status word and, through the library's
process-wide error word (pinned host memory installed by the operator layer),
reaches every later operator call and ``torchlpc_b200.check_status()`` as a
RuntimeError.  The give-up is produced by the library's self-test (a chunked
forward whose look-back waits for a flag nothing sets, with a short spin
limit): a bounded wait that ends, not a fault.  The reference's operators
report errors the same way, as RuntimeError (torchlpc/csrc/cuda/lpc.cu:117-127).
"""
import pytest
import torch

import torchlpc_b200 as tl

pytestmark = pytest.mark.gpu


def _drain():
    try:
        tl.check_status()
    except RuntimeError:
        pass


def test_timeout_raises_in_check_status_and_next_call():
    like = torch.zeros(1, device="cuda")
    _drain()
    tl.check_status()  # nothing pending
    assert torch.ops.torchlpc_b200.selftest_timeout(like, 2000) == 5  # LPC_ERR_TIMEOUT
    with pytest.raises(RuntimeError, match="bounded device-side wait"):
        tl.check_status()
    tl.check_status()  # the check cleared the word

    assert torch.ops.torchlpc_b200.selftest_timeout(like, 2000) == 5
    x = torch.randn(2, 5000, device="cuda")
    A = 0.01 * torch.randn(2, 5000, 4, device="cuda")
    with pytest.raises(RuntimeError, match="earlier call"):
        tl.sample_wise_lpc(x, A)
    # raised once, then cleared: the context keeps working
    y = tl.sample_wise_lpc(x, A)
    torch.cuda.synchronize()
    assert torch.isfinite(y).all()
    tl.check_status()
