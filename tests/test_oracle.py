"""Pin the FP64 C oracle against vectors produced by the reference itself.

The fixtures in tests/golden/ were generated by tests/golden/make_golden.py,
which runs DiffAPF/torchlpc's own CPU operator and autograd Functions.  The
oracle restates the same algorithm in plain C (oracle/lpc_oracle.c); on the
reference's float64 outputs it must agree to rounding level.
"""
import numpy as np
import pytest

from oracle import lpc_oracle as O
from tests.conftest import golden_names, load_golden

TOL64 = 1e-11  # normwise, FP64 restatement vs FP64 reference (different summation order only)

LPC_CASES = [n for n in golden_names() if not n.startswith("scan") and "ragged" not in n]


@pytest.mark.parametrize("name", LPC_CASES)
def test_oracle_matches_reference(name):
    d = load_golden(name)
    ti = bool(d["time_invariant"])
    y = O.lpc_forward(d["x"], d["A"], d["zi"])
    assert O.normwise_err(y, d["ref64_y"]) < TOL64
    N = d["A"].shape[-1]
    zf = y[:, -N:][:, ::-1]
    assert O.normwise_err(zf, d["ref64_zf"]) < TOL64
    gx, gA, gzi = O.lpc_backward(d["gy"], d["A"], d["zi"], y)
    assert O.normwise_err(gx, d["ref64_gx"]) < TOL64
    assert O.normwise_err(gA, d["ref64_ga" if ti else "ref64_gA"]) < TOL64
    if "ref64_gzi" in d:
        assert O.normwise_err(gzi, d["ref64_gzi"]) < TOL64


def test_oracle_ragged_matches_reference():
    d = load_golden("cfg4_small_ragged")
    y = O.lpc_forward_ragged(d["x"], d["A"], d["zi"], d["offsets"])
    assert O.normwise_err(y, d["ref64_y"]) < TOL64
    gx, gA, gzi = O.lpc_backward_ragged(d["gy"], d["A"], d["zi"], y, d["offsets"])
    assert O.normwise_err(gx, d["ref64_gx"]) < TOL64
    assert O.normwise_err(gA, d["ref64_gA"]) < TOL64
    assert O.normwise_err(gzi, d["ref64_gzi"]) < TOL64


def test_oracle_scan_matches_reference():
    d = load_golden("scan_T123")
    out = O.scan_forward(d["impulse"], d["decay"], d["init"])
    assert O.normwise_err(out, d["ref64_out"]) < TOL64
    gi, gd, g0 = O.scan_backward(d["go"], d["decay"], d["init"], out)
    assert O.normwise_err(gi, d["ref64_gimpulse"]) < TOL64
    assert O.normwise_err(gd, d["ref64_gdecay"]) < TOL64
    assert O.normwise_err(g0, d["ref64_ginit"]) < TOL64


def test_reference_fp32_within_tolerance_of_oracle():
    """The reference's own float32 CPU outputs sit well inside the 1e-4 bar."""
    for name in [n for n in LPC_CASES if "ref32_y" in load_golden(n)]:
        d = load_golden(name)
        y = O.lpc_forward(d["x"], d["A"], d["zi"])
        assert O.normwise_err(d["ref32_y"], y) < 1e-4, name


def test_oracle_gradient_finite_difference():
    """Independent check of the backward formulas: directional finite differences."""
    rng = np.random.default_rng(0)
    B, T, N = 2, 40, 3
    x = rng.standard_normal((B, T))
    A = rng.uniform(-0.3, 0.3, (B, T, N)) / N
    zi = rng.standard_normal((B, N))
    gy = rng.standard_normal((B, T))
    y = O.lpc_forward(x, A, zi)
    gx, gA, gzi = O.lpc_backward(gy, A, zi, y)
    dx, dA, dz = rng.standard_normal(x.shape), rng.standard_normal(A.shape), rng.standard_normal(zi.shape)
    eps = 1e-6
    lp = (O.lpc_forward(x + eps * dx, A + eps * dA, zi + eps * dz) * gy).sum()
    lm = (O.lpc_forward(x - eps * dx, A - eps * dA, zi - eps * dz) * gy).sum()
    fd = (lp - lm) / (2 * eps)
    an = (gx * dx).sum() + (gA * dA).sum() + (gzi * dz).sum()
    assert abs(fd - an) < 1e-6 * max(1.0, abs(an))
