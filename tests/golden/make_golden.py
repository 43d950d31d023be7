"""Generate golden input/output vectors by running the reference itself.

Runs DiffAPF/torchlpc's own CPU path (its compiled ``torchlpc::lpc`` /
``torchlpc::scan`` operators plus its Python autograd Functions), built by
``oracle/build.py`` from the reference sources into ``oracle/_ref``.  Needs the
reference tree (only available where the sources are mounted); the resulting
``*.npz`` fixtures are committed and are what the tests read everywhere else.

Each fixture holds the inputs (``x``, ``A``, ``zi``, ``gy`` ...), the outputs of
the reference in float64 (``ref64_*``: the reference run on the float64 cast of
the inputs) and, for float32 cases, the reference's own float32 outputs
(``ref32_*``).  Outputs: ``y``, ``zf``, ``gx``, ``gA`` (or ``ga`` for a
time-invariant A), ``gzi``.  Gradients are of the loss ``sum(y * gy)``.

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.build import build_reference  # noqa: E402
from torchlpc_b200.synth import make_workload  # noqa: E402

OUT = Path(__file__).resolve().parent


def _ref():
    path = build_reference()
    if path is None:
        raise SystemExit("reference sources not present; fixtures cannot be regenerated here")
    sys.path.insert(0, str(path))
    import torchlpc  # noqa: F401  (the reference package)

    assert torchlpc.EXTENSION_LOADED, "reference C++ extension did not load"
    return torchlpc


def biquad_inputs(batch, samples, g, dtype=torch.float64):
    """The reference tests' input pattern (tests/test_grad.py:8-38): two random
    biquads, coefficients linearly interpolated over time, repeated over batch."""
    def rnd():
        mag = torch.rand(1, generator=g, dtype=torch.float64)
        phase = torch.rand(1, generator=g, dtype=torch.float64) * math.pi
        return torch.cat([-mag * torch.cos(phase) * 2, mag ** 2])

    s, e = rnd(), rnd()
    A = torch.stack([torch.linspace(float(s[i]), float(e[i]), samples, dtype=torch.float64)
                     for i in range(2)]).T.unsqueeze(0).repeat(batch, 1, 1)
    x = torch.randn(batch, samples, generator=g, dtype=torch.float64)
    zi = torch.randn(batch, 2, generator=g, dtype=torch.float64)
    return x.to(dtype), A.to(dtype), zi.to(dtype)


def run_lpc(tl, x, A, zi, gy, time_invariant=False, zi_grad=True):
    """Reference forward + backward through its public API."""
    x = x.clone().requires_grad_(True)
    A = A.clone().requires_grad_(True)
    zi_l = zi.clone().requires_grad_(zi_grad)
    T = x.shape[1]
    Ae = A[:, None, :].expand(-1, T, -1) if time_invariant else A
    y, zf = tl.sample_wise_lpc(x, Ae, zi_l, return_zf=True)
    (y * gy).sum().backward()
    out = {"y": y, "zf": zf, "gx": x.grad, ("ga" if time_invariant else "gA"): A.grad}
    if zi_grad:
        out["gzi"] = zi_l.grad
    return {k: v.detach().numpy() for k, v in out.items()}


def save(name, inputs, tl, time_invariant=False, zi_grad=True):
    x, A, zi, gy = (inputs[k] for k in ("x", "A", "zi", "gy"))
    d = {k: v.numpy() for k, v in inputs.items()}
    r64 = run_lpc(tl, x.double(), A.double(), zi.double(), gy.double(), time_invariant, zi_grad)
    d.update({f"ref64_{k}": v for k, v in r64.items()})
    if x.dtype == torch.float32:
        r32 = run_lpc(tl, x, A, zi, gy, time_invariant, zi_grad)
        d.update({f"ref32_{k}": v for k, v in r32.items()})
    d["time_invariant"] = np.array(time_invariant)
    np.savez_compressed(OUT / f"{name}.npz", **d)
    print(name, {k: v.shape for k, v in d.items()})


def main():
    tl = _ref()
    g = torch.Generator().manual_seed(1234)

    # 1. the reference tests' own input pattern (test_grad.py / test_extension.py sizes)
    for T in (32, 1021):
        x, A, zi = biquad_inputs(4, T, g)
        gy = torch.randn(4, T, generator=g, dtype=torch.float64)
        save(f"biquad_T{T}_f64", dict(x=x, A=A, zi=zi, gy=gy), tl)
    x, A, zi = biquad_inputs(4, 4097, g, torch.float32)
    gy = torch.randn(4, 4097, generator=g, dtype=torch.float32)
    save("biquad_T4097_f32", dict(x=x, A=A, zi=zi, gy=gy), tl)

    # 2. scaled-down instances of the five benchmark workloads (float32 problem instances)
    for name, kw in [("cfg1", {}), ("cfg2", dict(B=2, T=800)), ("cfg3", dict(B=2, T=1024)),
                     ("cfg5", dict(B=3, T=1500))]:
        w = make_workload(name, seed=7, **kw)
        ti = w["workload"].time_invariant
        save(f"{name}_small", {k: w[k] for k in ("x", "A", "zi", "gy")}, tl, time_invariant=ti)

    # ragged: the reference has no ragged API; each signal runs on its own
    w = make_workload("cfg4", seed=7, B=4, lengths_hi=1400)
    off = w["offsets"].numpy()
    d = {"x": w["x"].numpy(), "A": w["A"].numpy(), "zi": w["zi"].numpy(), "gy": w["gy"].numpy(),
         "offsets": off}
    parts = {"y": [], "gx": [], "gA": [], "gzi": []}
    for b in range(len(off) - 1):
        s, e = off[b], off[b + 1]
        r = run_lpc(tl, w["x"][None, s:e].double(), w["A"][None, s:e].double(),
                    w["zi"][b:b + 1].double(), w["gy"][None, s:e].double())
        for k in parts:
            parts[k].append(r[k][0])
    d.update({"ref64_y": np.concatenate(parts["y"]), "ref64_gx": np.concatenate(parts["gx"]),
              "ref64_gA": np.concatenate(parts["gA"]), "ref64_gzi": np.stack(parts["gzi"])})
    np.savez_compressed(OUT / "cfg4_small_ragged.npz", **d)
    print("cfg4_small_ragged", {k: v.shape for k, v in d.items()})

    # 3. edge cases
    def rand_stable(B, T, N, dtype=torch.float64, scale=0.5):
        A = (torch.rand(B, T, N, generator=g, dtype=torch.float64) * 2 - 1) * (scale / N)
        x = torch.randn(B, T, generator=g, dtype=torch.float64)
        zi = torch.randn(B, N, generator=g, dtype=torch.float64)
        gy = torch.randn(B, T, generator=g, dtype=torch.float64)
        return dict(x=x.to(dtype), A=A.to(dtype), zi=zi.to(dtype), gy=gy.to(dtype))

    save("edge_T_lt_N", rand_stable(3, 3, 8), tl)       # T < N: zf has T columns
    save("edge_T1", rand_stable(2, 1, 4), tl)
    save("edge_N1", rand_stable(3, 300, 1), tl)         # order 1 -> reference routes to linear_recurrence
    save("edge_N64", rand_stable(2, 200, 64), tl)       # order above one warp
    save("edge_N3_f32", rand_stable(5, 257, 3, torch.float32), tl)
    save("edge_no_zi_grad", rand_stable(2, 100, 5), tl, zi_grad=False)

    # 4. order-1 recurrence through the reference Recurrence Function (test_grad.py:114-171)
    from torchlpc.recurrence import Recurrence

    B, T = 2, 123
    decay = (torch.rand(B, T, generator=g, dtype=torch.float64) * 2 - 1)
    impulse = torch.randn(B, T, generator=g, dtype=torch.float64)
    init = torch.randn(B, generator=g, dtype=torch.float64)
    go = torch.randn(B, T, generator=g, dtype=torch.float64)
    dd, ii, i0 = (t.clone().requires_grad_(True) for t in (decay, impulse, init))
    out = Recurrence.apply(dd, ii, i0)
    (out * go).sum().backward()
    np.savez_compressed(OUT / "scan_T123.npz", decay=decay.numpy(), impulse=impulse.numpy(),
                        init=init.numpy(), go=go.numpy(), ref64_out=out.detach().numpy(),
                        ref64_gdecay=dd.grad.numpy(), ref64_gimpulse=ii.grad.numpy(),
                        ref64_ginit=i0.grad.numpy())
    print("scan_T123")


if __name__ == "__main__":
    main()
