"""Ragged batches: signals concatenated along time, one persistent launch.

The oracle filters each signal of the concatenation on its own
(oracle/lpc_oracle.c, the per-signal restatement of torchlpc/csrc/
scan_cpu.cpp:80-122 and core.py:186-229); the GPU path must agree with it
and with the dense per-signal operator.  Lengths cover the edge cases of the
tiling: empty signals, signals shorter than the order, shorter than a chunk,
exactly one batch, many batches, and offsets that are not 16-byte aligned.
"""
import numpy as np
import pytest
import torch

import torchlpc_b200 as tl
from oracle import lpc_oracle as O
from tests.conftest import load_golden

LENGTHS = [0, 1, 7, 300, 3584, 4000, 9001, 33000, 2, 0, 70001]


def _ragged_case(lengths, N, seed, dtype):
    g = np.random.default_rng(seed)
    off = np.zeros(len(lengths) + 1, np.int64)
    off[1:] = np.cumsum(lengths)
    S = int(off[-1])
    x = g.standard_normal(S)
    # stable per-sample filters: poles of radius <= 0.9 with slowly drifting angles
    A = np.zeros((S, N))
    for s in range(len(lengths)):
        a, b = off[s], off[s + 1]
        if b == a:
            continue
        t = np.arange(b - a)[:, None]
        P = N // 2
        r = 0.5 + 0.4 * g.random(P)
        th = (np.arange(P) + g.random(P)) * np.pi / max(P, 1)
        th = th[None, :] + 0.2 * np.sin(2 * np.pi * t / 997.0)
        coef = np.zeros((b - a, N + 1))
        coef[:, 0] = 1.0
        quads = [(-2 * r[k] * np.cos(th[:, k]), np.full(b - a, r[k] ** 2)) for k in range(P)]
        if N % 2:
            quads.append((np.full(b - a, -0.5), np.zeros(b - a)))
        for q1, q2 in quads:  # multiply by (1 + q1 z^-1 + q2 z^-2), row-wise
            new = coef.copy()
            new[:, 1:] += q1[:, None] * coef[:, :-1]
            new[:, 2:] += q2[:, None] * coef[:, :-2]
            coef = new
        A[a:b] = coef[:, 1:N + 1]
    zi = 0.1 * g.standard_normal((len(lengths), N))
    gy = g.standard_normal(S)
    cast = (lambda v: v.astype(np.float32)) if dtype == torch.float32 else (lambda v: v)
    return off, cast(x), cast(A), cast(zi), cast(gy)


def _dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t.to(dtype) if dtype is not None else t).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("N,dtype,tol", [(24, torch.float32, 1e-4), (16, torch.float32, 1e-4),
                                         (5, torch.float32, 1e-4), (16, torch.float64, 1e-10)])
def test_ragged_matches_oracle(N, dtype, tol):
    off, x, A, zi, gy = _ragged_case(LENGTHS, N, seed=N, dtype=dtype)
    xt = _dev(x).requires_grad_(True)
    At = _dev(A).requires_grad_(True)
    zt = _dev(zi).requires_grad_(True)
    offt = _dev(off)
    y = tl.sample_wise_lpc_ragged(xt, At, offt, zt)
    (y * _dev(gy)).sum().backward()
    torch.cuda.synchronize()
    ry = O.lpc_forward_ragged(x, A, zi, off)
    rgx, rgA, rgzi = O.lpc_backward_ragged(gy, A, zi, ry, off)
    assert O.normwise_err(y.detach().cpu().numpy(), ry) < tol
    assert O.normwise_err(xt.grad.cpu().numpy(), rgx) < tol
    assert O.normwise_err(At.grad.cpu().numpy(), rgA) < tol
    assert O.normwise_err(zt.grad.cpu().numpy(), rgzi) < tol


@pytest.mark.gpu
def test_ragged_equals_dense_per_signal():
    N = 16
    off, x, A, zi, gy = _ragged_case([5000, 12345, 800], N, seed=3, dtype=torch.float32)
    y = tl.sample_wise_lpc_ragged(_dev(x), _dev(A), _dev(off), _dev(zi))
    for s in range(3):
        a, b = off[s], off[s + 1]
        yd = tl.sample_wise_lpc(_dev(x[a:b])[None], _dev(A[a:b])[None], _dev(zi[s:s + 1]))
        assert O.normwise_err(y[a:b].cpu().numpy(), yd[0].cpu().numpy()) < 1e-5


@pytest.mark.gpu
def test_ragged_golden_fixture():
    d = load_golden("cfg4_small_ragged")
    off = d["offsets"].astype(np.int64)
    x = _dev(d["x"], torch.float32).requires_grad_(True)
    A = _dev(d["A"], torch.float32).requires_grad_(True)
    zi = _dev(d["zi"], torch.float32).requires_grad_(True)
    y = tl.sample_wise_lpc_ragged(x, A, _dev(off), zi)
    (y * _dev(d["gy"], torch.float32)).sum().backward()
    assert O.normwise_err(y.detach().cpu().numpy(), d["ref64_y"]) < 1e-4
    assert O.normwise_err(x.grad.cpu().numpy(), d["ref64_gx"]) < 1e-4
    assert O.normwise_err(A.grad.cpu().numpy(), d["ref64_gA"]) < 1e-4
    assert O.normwise_err(zi.grad.cpu().numpy(), d["ref64_gzi"]) < 1e-4


def test_ragged_refuses_cpu_tensors():
    x = torch.zeros(10)
    A = torch.zeros(10, 4)
    off = torch.tensor([0, 4, 10])
    with pytest.raises((RuntimeError, NotImplementedError)):
        tl.sample_wise_lpc_ragged(x, A, off)


def test_ragged_shape_checks():
    with pytest.raises(AssertionError):
        tl.sample_wise_lpc_ragged(torch.zeros(10), torch.zeros(9, 4), torch.tensor([0, 10]))
    with pytest.raises(AssertionError):
        tl.sample_wise_lpc_ragged(torch.zeros(10), torch.zeros(10, 4), torch.tensor([0, 10]),
                                  torch.zeros(2, 4))
