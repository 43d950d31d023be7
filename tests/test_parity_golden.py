"""GPU parity against vectors produced by the reference itself (tests/golden/).

Each fixture holds inputs and DiffAPF/torchlpc's float64 outputs (y, zf,
grad_x, grad_A / grad_a, grad_zi) for the reference tests' input pattern, for
scaled-down instances of the five benchmark workloads and for edge cases
(T < N, T = 1, N = 1, N = 64, no zi gradient).  Tolerance (normwise
max|out-ref|/max|ref|): 1e-4 for float32 kernels, 1e-10 for float64 kernels.
"""
import numpy as np
import pytest
import torch

from tests.conftest import golden_names, load_golden
from tests.gpu_helpers import TOL32, TOL64, err, oracle_fwd_bwd, run_fwd_bwd, to_dev

pytestmark = pytest.mark.gpu

ALGOS = ["plain", "chunked", "ti"]  # "ti" serves time-invariant cases, the rest as "auto"
CASES = [n for n in golden_names() if not n.startswith("scan") and "ragged" not in n]


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("name", CASES)
def test_golden_lpc(name, algo):
    d = load_golden(name)
    f32 = d["x"].dtype == np.float32
    tol = TOL32 if f32 else TOL64
    ti = bool(d["time_invariant"])
    zi_grad = "ref64_gzi" in d
    x, A, zi, gy = (to_dev(d[k]) for k in ("x", "A", "zi", "gy"))
    out = run_fwd_bwd(x, A, zi, gy, time_invariant=ti, zi_grad=zi_grad, algo=algo)
    assert err(out["y"], d["ref64_y"]) < tol
    assert err(out["zf"], d["ref64_zf"]) < tol
    assert err(out["gx"], d["ref64_gx"]) < tol
    assert err(out["gA"], d["ref64_ga" if ti else "ref64_gA"]) < tol
    if zi_grad:
        assert err(out["gzi"], d["ref64_gzi"]) < tol
    # and the same against the FP64 oracle on identical inputs
    o = oracle_fwd_bwd(d["x"], d["A"], d["zi"], d["gy"])
    if not ti:
        assert err(out["gA"], o["gA"]) < tol
    assert err(out["y"], o["y"]) < tol


@pytest.mark.parametrize("algo", ALGOS)
def test_golden_scan(algo):
    import torchlpc_b200 as tl
    from torchlpc_b200.recurrence import Recurrence

    d = load_golden("scan_T123")
    old = tl.get_algo()
    tl.set_algo(algo)
    try:
        dd, ii, i0 = (to_dev(d[k]).requires_grad_(True) for k in ("decay", "impulse", "init"))
        out = Recurrence.apply(dd, ii, i0)
        (out * to_dev(d["go"])).sum().backward()
    finally:
        tl.set_algo(old)
    assert err(out.detach(), d["ref64_out"]) < TOL64
    assert err(ii.grad, d["ref64_gimpulse"]) < TOL64
    assert err(dd.grad, d["ref64_gdecay"]) < TOL64
    assert err(i0.grad, d["ref64_ginit"]) < TOL64
