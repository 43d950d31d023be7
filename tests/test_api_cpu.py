"""Host-side behaviour of the Python surface (no GPU): same names and argument
checks as torchlpc (torchlpc/__init__.py:28-104), and no silent CPU fallback."""
import inspect

import pytest
import torch

import torchlpc_b200 as tl


def test_public_surface():
    for name in ["sample_wise_lpc", "linear_recurrence", "LPC", "Recurrence", "EXTENSION_LOADED"]:
        assert hasattr(tl, name)
    assert list(inspect.signature(tl.sample_wise_lpc).parameters) == ["x", "a", "zi", "return_zf"]
    assert list(inspect.signature(tl.linear_recurrence).parameters) == ["a", "x", "zi"]
    assert tl.EXTENSION_LOADED


def test_shape_assertions_like_reference():
    x = torch.zeros(2, 10)
    with pytest.raises(AssertionError):
        tl.sample_wise_lpc(x, torch.zeros(3, 10, 2))
    with pytest.raises(AssertionError):
        tl.sample_wise_lpc(x, torch.zeros(2, 10))
    with pytest.raises(AssertionError):
        tl.sample_wise_lpc(x, torch.zeros(2, 10, 2), torch.zeros(2, 3))
    with pytest.raises(AssertionError):
        tl.linear_recurrence(torch.zeros(2, 10), torch.zeros(2, 9))


def test_cpu_tensors_fail_loudly():
    x = torch.zeros(2, 10)
    A = torch.zeros(2, 10, 2)
    with pytest.raises(RuntimeError, match="CUDA"):
        tl.sample_wise_lpc(x, A)
    with pytest.raises(RuntimeError, match="CUDA"):
        tl.linear_recurrence(torch.zeros(2, 10), x)


def test_algo_switch():
    old = tl.get_algo()
    tl.set_algo("plain")
    assert tl.get_algo() == "plain"
    tl.set_algo(old)
    with pytest.raises(KeyError):
        tl.set_algo("bogus")
