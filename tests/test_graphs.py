"""fwd+bwd captured in one CUDA graph and replayed.

Every launch takes the current stream and its workspace from the caching
allocator, nothing synchronises or allocates outside the allocator, so the
filter, its fused backward and the ragged and time-invariant paths can be
captured once and replayed with new data in the static input tensors.  Each
replay must equal the eager result on the same inputs.
"""
import pytest
import torch

import torchlpc_b200 as tl
from oracle import lpc_oracle as O
from torchlpc_b200.synth import make_workload

pytestmark = pytest.mark.gpu


def _capture(step):
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            step()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = step()
    return g, out


def _dense_case(seed):
    w = make_workload("cfg3", seed=seed, device="cuda", B=2, T=40000)
    return w["x"], w["A"], w["zi"], w["gy"]


@pytest.mark.parametrize("algo", ["chunked", "plain"])
def test_graph_replay_matches_eager(algo):
    old = tl.get_algo()
    tl.set_algo(algo)
    try:
        x0, A0, zi0, gy0 = _dense_case(11)
        x = x0.clone().requires_grad_(True)
        A = A0.clone().requires_grad_(True)
        zi = zi0.clone().requires_grad_(True)
        gy = gy0.clone()

        def step():
            x.grad = A.grad = zi.grad = None
            y = tl.sample_wise_lpc(x, A, zi)
            y.backward(gy)
            return y

        g, y_static = _capture(step)
        gx_static, gA_static, gzi_static = x.grad, A.grad, zi.grad
        for seed in (12, 13):
            x1, A1, zi1, gy1 = _dense_case(seed)
            with torch.no_grad():
                x.copy_(x1)
                A.copy_(A1)
                zi.copy_(zi1)
                gy.copy_(gy1)
            g.replay()
            torch.cuda.synchronize()
            xe, Ae, ze = (t.clone().requires_grad_(True) for t in (x1, A1, zi1))
            ye = tl.sample_wise_lpc(xe, Ae, ze)
            ye.backward(gy1)
            assert torch.equal(y_static, ye.detach())
            assert torch.equal(gx_static, xe.grad)
            assert torch.equal(gA_static, Ae.grad)
            assert torch.equal(gzi_static, ze.grad)
    finally:
        tl.set_algo(old)


def test_graph_replay_ragged_and_time_invariant():
    w = make_workload("cfg4", seed=5, device="cuda", B=12, lengths_hi=20000)
    x = w["x"].clone().requires_grad_(True)
    A = w["A"].clone().requires_grad_(True)
    zi = w["zi"].clone().requires_grad_(True)
    off = w["offsets"]

    def step_r():
        x.grad = A.grad = zi.grad = None
        y = tl.sample_wise_lpc_ragged(x, A, off, zi)
        y.backward(w["gy"])
        return y

    g, y_static = _capture(step_r)
    g.replay()
    torch.cuda.synchronize()
    ref = O.lpc_forward_ragged(w["x"].cpu().numpy(), w["A"].cpu().numpy(), w["zi"].cpu().numpy(),
                               w["offsets"].cpu().numpy())
    assert O.normwise_err(y_static.detach().cpu().numpy(), ref) < 1e-4

    wt = make_workload("cfg5", seed=6, device="cuda", B=3, T=20000)
    xt = wt["x"].clone().requires_grad_(True)
    at = wt["A"].clone().requires_grad_(True)
    T = xt.shape[1]

    def step_t():
        xt.grad = at.grad = None
        y = tl.sample_wise_lpc(xt, at[:, None, :].expand(-1, T, -1))
        y.backward(wt["gy"])
        return y

    g2, yt_static = _capture(step_t)
    g2.replay()
    torch.cuda.synchronize()
    reft = O.lpc_forward(wt["x"].cpu().numpy(), wt["A"].cpu().numpy(), None)
    assert O.normwise_err(yt_static.detach().cpu().numpy(), reft) < 1e-4
