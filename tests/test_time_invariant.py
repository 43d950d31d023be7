"""Time-invariant coefficients (one (N,) set per signal) through the dedicated
time-invariant scan: chunk transitions C^L by squaring, an FP64 chain of
chunk entry states, each chunk re-filtered from its exact entry state.

The reference feeds such filters as A[:, None, :].expand(-1, T, -1)
(tests/test_vmap.py:41, README.md:108-130); the oracle is the FP64 sequential
restatement with a stride-0 coefficient row.  Cases cover one partial chunk,
several chunks with a partial last one, orders that pad (N < padded order)
and both dtypes.
"""
import numpy as np
import pytest
import torch

from oracle import lpc_oracle as O
from tests.gpu_helpers import TOL32, TOL64, err, run_fwd_bwd, to_dev

pytestmark = pytest.mark.gpu


def _stable_ti(B, N, rng, rmax=0.95):
    A = np.zeros((B, N))
    P = N // 2
    for b in range(B):
        r = 0.5 + (rmax - 0.5) * rng.random(P)
        th = (np.arange(P) + rng.random(P)) * np.pi / max(P, 1)
        c = np.array([1.0])
        for k in range(P):
            c = np.convolve(c, [1.0, -2 * r[k] * np.cos(th[k]), r[k] ** 2])
        if N % 2:
            c = np.convolve(c, [1.0, -0.6])
        A[b] = c[1:N + 1]
    return A


@pytest.mark.parametrize("N", [32, 16, 7, 2])
@pytest.mark.parametrize("T", [1000, 5000, 70001])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_time_invariant_scan_matches_oracle(N, T, dtype):
    rng = np.random.default_rng(1000 * N + T)
    B = 3
    A = _stable_ti(B, N, rng)
    x = rng.standard_normal((B, T))
    zi = 0.3 * rng.standard_normal((B, N))
    gy = rng.standard_normal((B, T))
    if dtype == torch.float32:
        A, x, zi, gy = (v.astype(np.float32) for v in (A, x, zi, gy))
    tol = TOL32 if dtype == torch.float32 else TOL64
    out = run_fwd_bwd(to_dev(x), to_dev(A), to_dev(zi), to_dev(gy), time_invariant=True, algo="ti")
    y = O.lpc_forward(x, A, zi)
    gx, ga, gzi = O.lpc_backward(gy, A, zi, y)
    assert err(out["y"], y) < tol
    assert err(out["zf"], y[:, -N:][:, ::-1]) < tol
    assert err(out["gx"], gx) < tol
    assert err(out["gA"], ga) < tol
    assert err(out["gzi"], gzi) < tol


def test_time_invariant_auto_picks_the_scan_for_long_signals():
    """AUTO with a stride-0 coefficient row and T >= 2048 takes the
    time-invariant scan; the result must equal the plain kernel's."""
    import torchlpc_b200 as tl

    rng = np.random.default_rng(7)
    B, T, N = 2, 9000, 12
    A = _stable_ti(B, N, rng).astype(np.float32)
    x = rng.standard_normal((B, T)).astype(np.float32)
    zi = np.zeros((B, N), np.float32)
    outs = []
    for algo in ("auto", "plain"):
        old = tl.get_algo()
        tl.set_algo(algo)
        try:
            At = to_dev(A)
            y = tl.sample_wise_lpc(to_dev(x), At[:, None, :].expand(-1, T, -1), to_dev(zi))
        finally:
            tl.set_algo(old)
        outs.append(y.cpu().numpy())
    assert err(outs[0], outs[1].astype(np.float64)) < 1e-5
