"""Seeded synthetic workloads for the all-pole filter.

The five workloads are the ones the filter is benchmarked on: frame-rate
conjugate pole pairs, linearly interpolated per sample and expanded to
direct-form coefficients ``A[b,t,:]`` (coefficients 1..N of
``prod_k (1 - 2 r_k cos(th_k) z^-1 + r_k^2 z^-2)``).

Generation rules (kept identical on every device so that fp32 problem
instances are reproducible):

* all random draws come from a CPU ``torch.Generator`` seeded with ``seed``;
  draws and the expansion are fp64, the problem instance is the fp32 cast;
* pole angles are *stratified*: pair k draws ``th ~ U[k*pi/P, (k+1)*pi/P]``
  (marginally still U[0, pi]).  Independent U[0, pi] angles cluster, and the
  fp32-rounded direct-form coefficients of 8-16 clustered pairs are unstable
  (outputs overflow even in fp64), so the error of a kernel against an FP64
  oracle would be meaningless;
* every fp32-rounded coefficient row is audited with the Schur-Cohn step-down
  test in fp64; a signal with any unstable row is redrawn from a generator
  seeded by (seed, signal, attempt).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import torch

__all__ = ["WORKLOADS", "Workload", "make_workload", "pole_pair_coeffs",
           "schur_cohn_stable", "ragged_lengths"]


@dataclass(frozen=True)
class Workload:
    name: str
    B: int                   # signals (ragged: number of signals)
    T: int                   # samples per signal (ragged: 0)
    npairs: int              # conjugate pole pairs; order N = 2*npairs
    hop: int                 # samples per frame (0: time-invariant)
    rlo: float
    rhi: float
    zi_std: float            # 0 -> zero initial conditions
    ragged: bool = False
    time_invariant: bool = False
    note: str = ""

    @property
    def N(self) -> int:
        return 2 * self.npairs


WORKLOADS = {
    "cfg1": Workload("cfg1", 4, 2048, 1, 128, 0.5, 0.9, 0.0,
                     note="plain sequential fwd+bwd, B=4 T=2048 N=2"),
    "cfg2": Workload("cfg2", 64, 16000, 11, 80, 0.7, 0.98, 0.1,
                     note="analysis-by-synthesis frame rate, B=64 T=16000 N=22"),
    "cfg3": Workload("cfg3", 8, 1 << 20, 8, 512, 0.9, 0.999, 1.0,
                     note="long-sequence chunked scan, B=8 T=2^20 N=16, fwd+bwd with boundary-state "
                          "checkpointing"),
    "cfg4": Workload("cfg4", 1024, 0, 12, 160, 0.6, 0.99, 0.1, ragged=True,
                     note="ragged batch, 1024 signals, lengths log-uniform in [1024, 262144], N=24"),
    "cfg5": Workload("cfg5", 2048, 65536, 16, 0, 0.5, 0.95, 0.0, time_invariant=True,
                     note="time-invariant filter, B=2048 T=65536 N=32"),
}


def schur_cohn_stable(a: torch.Tensor) -> torch.Tensor:
    """Step-down (Schur-Cohn) stability test of ``1 + sum_i a[..., i] z^-(i+1)``.

    ``a``: (..., N) coefficients, evaluated in fp64.  Returns a bool tensor
    (...) that is True where every reflection coefficient has |k| < 1, i.e. all
    poles lie strictly inside the unit circle.
    """
    c = a.double().clone()
    N = c.shape[-1]
    ok = torch.ones(c.shape[:-1], dtype=torch.bool, device=c.device)
    for m in range(N, 0, -1):
        k = c[..., m - 1]
        ok &= k.abs() < 1.0
        if m == 1:
            break
        denom = (1.0 - k * k).clamp_min(1e-300).unsqueeze(-1)
        head = c[..., : m - 1]
        rev = c[..., : m - 1].flip(-1)
        c = (head - k.unsqueeze(-1) * rev) / denom
    return ok


def _expand_pairs(r: torch.Tensor, th: torch.Tensor) -> torch.Tensor:
    """(…, P) radii/angles -> (…, 2P) direct-form coefficients 1..2P (fp64)."""
    P = r.shape[-1]
    poly = torch.zeros(*r.shape[:-1], 2 * P + 1, dtype=torch.float64, device=r.device)
    poly[..., 0] = 1.0
    c1 = -2.0 * r * torch.cos(th)
    c2 = r * r
    for k in range(P):
        d = 2 * k  # degree of the product so far
        new = poly.clone()
        new[..., 1 : d + 2] += poly[..., 0 : d + 1] * c1[..., k : k + 1]
        new[..., 2 : d + 3] += poly[..., 0 : d + 1] * c2[..., k : k + 1]
        poly = new
    return poly[..., 1:]


def _draw_knots(nsig: int, nknots: int, wl: Workload, g: torch.Generator):
    P = wl.npairs
    r = torch.rand(nsig, nknots, P, generator=g, dtype=torch.float64) * (wl.rhi - wl.rlo) + wl.rlo
    u = torch.rand(nsig, nknots, P, generator=g, dtype=torch.float64)
    th = (torch.arange(P, dtype=torch.float64) + u) * (math.pi / P)
    return r, th


def pole_pair_coeffs(r: torch.Tensor, th: torch.Tensor, T: int, hop: int,
                     device="cpu", block: int = 1 << 20) -> torch.Tensor:
    """Interpolate per-frame poles to T samples and expand.  Returns (S, T, N) fp64.

    r, th: (S, K, P) knot values; knot k sits at sample k*hop (align_corners).
    Processed in blocks of samples to bound the fp64 intermediates.
    """
    S, K, P = r.shape
    out = torch.empty(S, T, 2 * P, dtype=torch.float64, device=device)
    r = r.to(device)
    th = th.to(device)
    for t0 in range(0, T, block):
        t1 = min(T, t0 + block)
        t = torch.arange(t0, t1, dtype=torch.float64, device=device)
        pos = t / hop
        k0 = pos.floor().long().clamp(max=K - 2)
        w = (pos - k0.double()).view(1, -1, 1)
        rr = r[:, k0] * (1 - w) + r[:, k0 + 1] * w
        tt = th[:, k0] * (1 - w) + th[:, k0 + 1] * w
        out[:, t0:t1] = _expand_pairs(rr, tt)
    return out


def ragged_lengths(nsig: int, lo: int, hi: int, g: torch.Generator) -> torch.Tensor:
    u = torch.rand(nsig, generator=g, dtype=torch.float64)
    return torch.exp(math.log(lo) + u * (math.log(hi) - math.log(lo))).round().long()


def _signal_coeffs(wl: Workload, T: int, g: torch.Generator, device) -> torch.Tensor:
    """One signal's coefficients, (1, T, N) fp64 (time-invariant: (1, 1, N))."""
    if wl.time_invariant:
        r, th = _draw_knots(1, 1, wl, g)
        return _expand_pairs(r, th).to(device)
    K = math.ceil(T / wl.hop) + 1
    r, th = _draw_knots(1, K, wl, g)
    return pole_pair_coeffs(r, th, T, wl.hop, device=device)


def _audit_and_redraw(A64: torch.Tensor, wl: Workload, T_of, seed: int, device) -> torch.Tensor:
    """Redraw signals whose fp32-rounded rows fail the stability test."""
    ok_all = schur_cohn_stable(A64.float()).reshape(A64.shape[0], -1).all(1).tolist()
    for b in range(A64.shape[0]):
        attempt = 0
        ok = ok_all[b]
        while not ok:
            attempt += 1
            if attempt > 64:
                raise RuntimeError(f"could not draw a stable filter for signal {b}")
            gb = torch.Generator().manual_seed(hash((seed, b, attempt)) & 0x7FFFFFFF)
            A64[b] = _signal_coeffs(wl, T_of(b), gb, device)[0]
            ok = bool(schur_cohn_stable(A64[b].float()).all())
    return A64


def make_workload(name: str, seed: int = 0, device="cpu", dtype=torch.float32,
                  B: Optional[int] = None, T: Optional[int] = None,
                  with_grad_output: bool = True, lengths_hi: Optional[int] = None):
    """Build one seeded problem instance.

    Returns a dict with x, A, zi, gy (gy: the upstream gradient g of the loss
    sum(y*g)) as ``dtype`` tensors on ``device`` and, for the ragged workload,
    ``offsets`` (int64, B+1) and ``lengths``.  ``B``/``T`` override the sizes
    (scaled-down instances for tests); ``lengths_hi`` caps ragged lengths.

    Layouts: dense x (B,T), A (B,T,N) [time-invariant: (B,N)], zi (B,N);
    ragged x (S,), A (S,N), y (S,) with S = sum of lengths.
    """
    wl = WORKLOADS[name]
    B = wl.B if B is None else B
    N = wl.N
    g = torch.Generator().manual_seed(seed)
    out = {"workload": wl, "B": B, "N": N}
    if wl.ragged:
        hi = lengths_hi or 262144
        lo = min(1024, hi)
        lengths = ragged_lengths(B, lo, hi, g)
        offsets = torch.zeros(B + 1, dtype=torch.int64)
        offsets[1:] = torch.cumsum(lengths, 0)
        S = int(offsets[-1])
        parts = []
        for b in range(B):
            Tb = int(lengths[b])
            parts.append(_signal_coeffs(wl, Tb, g, device)[0])
        # audit per signal, redraw on failure
        for b in range(B):
            attempt = 0
            while not bool(schur_cohn_stable(parts[b].float()).all()):
                attempt += 1
                if attempt > 64:
                    raise RuntimeError("could not draw a stable filter")
                gb = torch.Generator().manual_seed(hash((seed, b, attempt)) & 0x7FFFFFFF)
                parts[b] = _signal_coeffs(wl, int(lengths[b]), gb, device)[0]
        A = torch.cat(parts, 0).to(dtype)
        x = torch.randn(S, generator=g, dtype=torch.float64).to(device=device, dtype=dtype)
        zi = (torch.randn(B, N, generator=g, dtype=torch.float64) * wl.zi_std).to(device=device, dtype=dtype)
        out.update(x=x, A=A, zi=zi, offsets=offsets.to(device), lengths=lengths, S=S, T=0)
        if with_grad_output:
            out["gy"] = torch.randn(S, generator=g, dtype=torch.float64).to(device=device, dtype=dtype)
        return out

    T = wl.T if T is None else T
    if wl.time_invariant:
        r, th = _draw_knots(B, 1, wl, g)
        A64 = _expand_pairs(r, th).to(device)  # (B,1,N)
    else:
        K = math.ceil(T / wl.hop) + 1
        r, th = _draw_knots(B, K, wl, g)
        A64 = pole_pair_coeffs(r, th, T, wl.hop, device=device)
    A64 = _audit_and_redraw(A64, wl, lambda b: T, seed, device)
    if wl.time_invariant:
        A = A64[:, 0, :].to(dtype).contiguous()
    else:
        A = A64.to(dtype)
    del A64
    x = torch.randn(B, T, generator=g, dtype=torch.float32).to(device=device, dtype=dtype)
    if wl.zi_std > 0:
        zi = (torch.randn(B, N, generator=g, dtype=torch.float64) * wl.zi_std).to(device=device, dtype=dtype)
    else:
        zi = torch.zeros(B, N, dtype=dtype, device=device)
    out.update(x=x, A=A, zi=zi, T=T)
    if with_grad_output:
        out["gy"] = torch.randn(B, T, generator=g, dtype=torch.float32).to(device=device, dtype=dtype)
    return out
