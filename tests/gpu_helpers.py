"""Shared helpers of the GPU parity tests (oracle = FP64 C restatement)."""
import numpy as np
import torch

import torchlpc_b200 as tl
from oracle import lpc_oracle as O

DEV = "cuda"
TOL32 = 1e-4   # normwise max|out-ref|/max|ref|, fp32 kernels vs FP64 reference
TOL64 = 1e-10  # fp64 kernels vs FP64 reference


def err(a, ref):
    return O.normwise_err(a, ref)


def run_fwd_bwd(x, A, zi, gy, time_invariant=False, zi_grad=True, algo="plain"):
    """sample_wise_lpc forward + backward of sum(y*gy) on the GPU.
    time_invariant: A is (B,N) and is passed as A[:,None,:].expand(-1,T,-1)."""
    old = tl.get_algo()
    tl.set_algo(algo)
    try:
        x = x.detach().clone().requires_grad_(True)
        A = A.detach().clone().requires_grad_(True)
        zi = zi.detach().clone().requires_grad_(zi_grad)
        T = x.shape[1]
        Ae = A[:, None, :].expand(-1, T, -1) if time_invariant else A
        y, zf = tl.sample_wise_lpc(x, Ae, zi, return_zf=True)
        (y * gy).sum().backward()
        torch.cuda.synchronize()
    finally:
        tl.set_algo(old)
    out = {"y": y.detach(), "zf": zf.detach(), "gx": x.grad, "gA": A.grad}
    if zi_grad:
        out["gzi"] = zi.grad
    return out


def oracle_fwd_bwd(x, A, zi, gy):
    y = O.lpc_forward(x, A, zi)
    gx, gA, gzi = O.lpc_backward(gy, A, zi, y)
    N = A.shape[-1]
    return {"y": y, "zf": y[:, -N:][:, ::-1], "gx": gx, "gA": gA, "gzi": gzi}


def to_dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(DEV)
