#!/usr/bin/env python
"""Benchmark of the all-pole (LPC) filter on B200: fwd+bwd samples/s.

One step = forward + backward of the filter over one batch of the workload,
through the public API (``sample_wise_lpc`` then ``y.backward(grad_y)``, i.e.
the gradients of sum(y * g) for x, A and zi).  Inputs are seeded synthetic
signals with the workload's shapes and pole statistics (torchlpc_b200.synth).

Default workload: B=8 signals, T=2^20 samples, order N=16 (8 pole pairs per
512-sample frame, radius U[0.9, 0.999], zi ~ N(0,1)) — the long-sequence
configuration the chunked scan targets.  ``--config`` selects another one.

Prints ONE JSON line (rank 0).  ``--impl reference`` times the reference's own
CPU implementation (DiffAPF/torchlpc's compiled operator and autograd, built
into oracle/_ref) on the host cores instead.

Multi-GPU (torchrun): every rank filters its own copy of the workload (signals
are independent; there is no collective on the data path) -> weak scaling.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from datetime import timedelta
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

METRIC = "fwd+bwd samples/s & % HBM peak, scan vs plain, at ≤1e-4 rel err vs FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-cuda-probe"])
    ap.add_argument("--config", default="cfg3", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"])
    ap.add_argument("--algo", default="auto", choices=["auto", "plain", "chunked"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the per-config summary")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--B", type=int, default=None, help="override signals (scaled-down instance for profiling)")
    ap.add_argument("--T", type=int, default=None, help="override samples per signal (scaled-down instance)")
    return ap.parse_args()


# --------------------------------------------------------------------------- utilities
def rank_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rk = int(os.environ.get("RANK", "0"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rk, lr


def max_over_ranks(v: float, device) -> float:
    if not dist.is_initialized():
        return v
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def bytes_per_sample(N: int, time_invariant: bool):
    """Algorithmic HBM bytes per sample (fp32): fwd reads x, A and writes y;
    bwd reads grad_y, A, y and writes grad_x, grad_A."""
    if time_invariant:
        return 8.0, 12.0
    return 8.0 + 4.0 * N, 12.0 + 8.0 * N


# --------------------------------------------------------------------------- workloads
def _synth():
    """The workload generator, loaded from its file so that importing it does
    not import the torchlpc_b200 package (and its native libraries): the
    reference arm uses it too."""
    name = "_lpc_b200_synth"
    if name in sys.modules:
        return sys.modules[name]
    import importlib.util

    spec = importlib.util.spec_from_file_location(name, ROOT / "torchlpc_b200" / "synth.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workload(cfg: str, device, seed: int = 0, B=None, T=None):
    return _synth().make_workload(cfg, seed=seed, device=device, B=B, T=T)


def config_of(args, w, ws: int) -> dict:
    """The workload description both arms print (same keys, same values)."""
    A = w["A"]
    return {"workload": f"{args.config}: {w['workload'].note}", "B": w["B"], "T": w["T"], "N": w["N"],
            "samples_per_step": samples_of(w),
            "l2": "inputs larger than L2 (coefficients alone %.0f MiB)" % (A.numel() * A.element_size() / 2 ** 20),
            "parallelism": f"replicas x{ws} (independent signals, no collective)"}


def samples_of(w) -> int:
    return int(w["S"]) if w["workload"].ragged else int(w["B"]) * int(w["T"])


def coeff_arg(w, A):
    """Coefficients as the public API takes them (time-invariant: expanded view)."""
    if w["workload"].time_invariant:
        return A[:, None, :].expand(-1, w["T"], -1)
    return A


# --------------------------------------------------------------------------- our arm
def make_step(tl, w, x, A, zi, gy):
    ragged = w["workload"].ragged

    def step():
        x.grad = A.grad = zi.grad = None
        if ragged:
            y = tl.sample_wise_lpc_ragged(x, A, w["offsets_dev"], zi)
        else:
            y = tl.sample_wise_lpc(x, coeff_arg(w, A), zi)
        y.backward(gy)
        return y

    return step


def count_kernels(fn) -> int:
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    n = 0
    for e in prof.events():
        if e.device_type.name == "CUDA" and "lpcb::" in e.name:
            n += 1
    return n


def time_loop(fn, steps, warmup, device):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(device)
    if dist.is_initialized():
        dist.barrier()
    torch.cuda.synchronize(device)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        fn()
    e.record()
    torch.cuda.synchronize(device)
    if dist.is_initialized():
        dist.barrier()
    return s.elapsed_time(e) / steps  # ms per step


def kernel_times(tl, w, x, A, zi, gy, steps, device, ckpt=False):
    """Average device time of the forward and the fused backward operator
    (CUDA events on the launching stream); ``ckpt``: the boundary-state
    checkpointed pair the public API runs for long signals."""
    from torchlpc_b200 import _ops

    Aa = coeff_arg(w, A).detach()
    if w["workload"].time_invariant:
        Aa = A.detach()
    with torch.no_grad():
        if w["workload"].ragged:
            fwd = lambda: _ops.lpc_ragged(x.detach(), A.detach(), w["offsets_dev"], zi.detach())
            y = fwd()
            bwd = lambda: _ops.lpc_backward_ragged(gy, A.detach(), w["offsets_dev"], zi.detach(), y, True, True)
        elif ckpt:
            L = _ops.checkpoint_chunk(w["T"], w["N"], x.dtype)
            fwd = lambda: _ops.lpc_checkpointed(x.detach(), Aa, zi.detach(), L)
            _, states = fwd()
            bwd = lambda: _ops.lpc_backward_checkpointed(gy, Aa, zi.detach(), x.detach(), states, L, True, True)
        else:
            fwd = lambda: _ops.lpc(x.detach(), Aa, zi.detach())
            y = fwd()
            bwd = lambda: _ops.lpc_backward(gy, Aa, zi.detach(), y, True, True)
        tf = time_loop(fwd, steps, 3, device)
        tb = time_loop(bwd, steps, 3, device)
    return tf, tb


def oracle_errors(tl, w, x, A, zi, gy, max_signals=None):
    """Normwise max|out - oracle| / max|oracle| of y, zf and the three
    gradients of the timed float32 path (one untimed fwd+bwd through the public
    API) against the FP64 sequential oracle (oracle/lpc_oracle.c, the checker)
    on the same float32 inputs.  Dense workloads compare every signal, or the
    first ``max_signals``; the ragged workload compares its 32 shortest and 32
    longest signals out of the full launch."""
    import numpy as np

    from oracle import lpc_oracle as O

    xx = x.detach().clone().requires_grad_(True)
    AA = A.detach().clone().requires_grad_(True)
    zz = zi.detach().clone().requires_grad_(True)
    got = {}
    if w["workload"].ragged:
        y = tl.sample_wise_lpc_ragged(xx, AA, w["offsets_dev"], zz)
        y.backward(gy)
        torch.cuda.synchronize()
        off = w["offsets"].cpu()
        lens = (off[1:] - off[:-1]).numpy()
        order = np.argsort(lens, kind="stable")
        pick = np.concatenate([order[:32], order[-32:]])
        rows = torch.from_numpy(np.concatenate([np.arange(int(off[b]), int(off[b + 1])) for b in pick])).to(x.device)
        sub = np.zeros(len(pick) + 1, np.int64)
        sub[1:] = np.cumsum(lens[pick])
        sig = torch.from_numpy(pick).to(x.device)
        xs, As, gs, zs = x.detach()[rows], A.detach()[rows], gy[rows], zi.detach()[sig]
        yo = O.lpc_forward_ragged(xs, As, zs, sub)
        gxo, gAo, gzio = O.lpc_backward_ragged(gs, As, zs, yo, sub)
        ref = {"y": yo, "gx": gxo, "gA": gAo, "gzi": gzio}
        got = {"y": y.detach()[rows], "gx": xx.grad[rows], "gA": AA.grad[rows], "gzi": zz.grad[sig]}
        what = f"{len(pick)} of {w['B']} ragged signals (32 shortest, 32 longest) from the full launch"
    else:
        y, zf = tl.sample_wise_lpc(xx, coeff_arg(w, AA), zz, return_zf=True)
        y.backward(gy)
        torch.cuda.synchronize()
        nb = w["B"] if max_signals is None else min(w["B"], max_signals)
        s = slice(0, nb)
        yo = O.lpc_forward(x.detach()[s], A.detach()[s], zi.detach()[s])
        gxo, gAo, gzio = O.lpc_backward(gy[s], A.detach()[s], zi.detach()[s], yo)
        N = w["N"]
        ref = {"y": yo, "zf": yo[:, -N:][:, ::-1], "gx": gxo, "gA": gAo, "gzi": gzio}
        got = {"y": y.detach()[s], "zf": zf.detach()[s], "gx": xx.grad[s], "gA": AA.grad[s], "gzi": zz.grad[s]}
        what = f"{nb} of {w['B']} signals, full length"
    errs = {k: O.normwise_err(got[k], ref[k]) for k in ref}
    tol = 1e-4
    return {**errs, "max": max(errs.values()), "tolerance": tol, "within": max(errs.values()) <= tol,
            "oracle": "FP64 sequential C restatement (oracle/lpc_oracle.c)", "compared": what}


def e2e_time(tl, w, x_dev, A_dev, zi_dev, gy_dev, steps, warmup, device, slices=8):
    """The same step through the public API with HOST inputs: every step copies
    x, A, zi and grad_y from pinned host memory and reads y and the three
    gradients back into pinned host memory.  The batch is cut into ``slices``
    groups of whole signals, filtered independently and pipelined over two
    CUDA streams (host-to-device copy, fwd+bwd, device-to-host copy), so that
    the copies of one group overlap the compute and the opposite copy
    direction of its neighbours; every copy is one cudaMemcpyAsync of a
    contiguous range.  Dense workloads only (ragged: one group)."""
    hx, hA, hz, hg = (t.detach().cpu().pin_memory() for t in (x_dev, A_dev, zi_dev, gy_dev))
    outs = {k: torch.empty(s, dtype=x_dev.dtype).pin_memory()
            for k, s in (("y", x_dev.shape), ("gx", x_dev.shape), ("gA", A_dev.shape), ("gzi", zi_dev.shape))}
    ragged = w["workload"].ragged
    B = hx.shape[0]
    k = 1 if ragged else max(1, min(slices, B))
    bounds = [(i * B // k, (i + 1) * B // k) for i in range(k)]
    streams = [torch.cuda.Stream(device) for _ in range(2)]
    main = torch.cuda.current_stream(device)

    def one(lo, hi, st):
        with torch.cuda.stream(st):
            sl = slice(lo, hi)
            if ragged:
                x, A, zi, gy = (t.to(device, non_blocking=True) for t in (hx, hA, hz, hg))
            else:
                x, A, zi, gy = (t[sl].to(device, non_blocking=True) for t in (hx, hA, hz, hg))
            x.requires_grad_(True)
            A.requires_grad_(True)
            zi.requires_grad_(True)
            if ragged:
                y = tl.sample_wise_lpc_ragged(x, A, w["offsets_dev"], zi)
            else:
                y = tl.sample_wise_lpc(x, coeff_arg(w, A), zi)
            y.backward(gy)
            dst = (lambda t: outs[t]) if ragged else (lambda t: outs[t][sl])
            dst("y").copy_(y.detach(), non_blocking=True)
            dst("gx").copy_(x.grad, non_blocking=True)
            dst("gA").copy_(A.grad, non_blocking=True)
            dst("gzi").copy_(zi.grad, non_blocking=True)

    def step():
        for st in streams:
            st.wait_stream(main)
        for i, (lo, hi) in enumerate(bounds):
            one(lo, hi, streams[i % 2])
        for st in streams:
            main.wait_stream(st)

    ms = time_loop(step, steps, warmup, device)
    h2d = sum(t.numel() * t.element_size() for t in (hx, hA, hz, hg))
    d2h = sum(t.numel() * t.element_size() for t in outs.values())
    return ms, h2d, d2h, k


def traffic_from_profiles(cfg: str, kernel: str):
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        e = d.get(cfg, {}).get(kernel)
        return None if e is None else float(e["bytes_per_launch"])
    except (ValueError, KeyError, TypeError):
        return None


# --------------------------------------------------------------------------- reference (CPU)
def reference_module():
    from oracle.build import build_reference

    path = build_reference()
    if path is None:
        return None, "reference CPU operator not built (oracle/_ref missing)"
    sys.path.insert(0, str(path))
    import warnings

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        import torchlpc  # the reference package, CPU operator compiled from its sources

    if not torchlpc.EXTENSION_LOADED:
        return None, "reference C++ extension failed to load"
    return torchlpc, None


def reference_sample(w, budget_signals=None):
    """A bounded sample of the workload on the host: whole signals (dense: all
    of B unless budget_signals; ragged: the first signals up to ~1/8 of the
    samples, padded per the reference API, one signal per call)."""
    wl = w["workload"]
    if wl.ragged:
        off = w["offsets"].cpu()
        lens = (off[1:] - off[:-1]).tolist()
        tot, picks = 0, []
        for b, L in enumerate(lens):
            picks.append(b)
            tot += L
            if tot >= samples_of(w) // 8:
                break
        return ("ragged", picks)
    B = w["B"] if budget_signals is None else min(w["B"], budget_signals)
    return ("dense", B)


def reference_calls(ref, w):
    """The reference CPU fwd+bwd (sample_wise_lpc + backward of sum(y*g)) over a
    bounded sample of the workload.  Returns (run_once, samples, description)."""
    wl = w["workload"]
    x, A, zi, gy = (w[k].detach().cpu() for k in ("x", "A", "zi", "gy"))
    kind, sel = reference_sample(w)
    calls = []
    if kind == "dense":
        B = sel
        T = w["T"]
        if wl.time_invariant:
            B = max(1, min(B, 64))  # the reference materialises (B,T,N) A; bound the host memory
        calls.append((x[:B], A[:B], zi[:B], gy[:B]))
        desc = f"{B} of {w['B']} signals x T={T}"
        nsamp = B * T
    else:
        off = w["offsets"].cpu()
        nsamp = 0
        for b in sel:
            s, e = int(off[b]), int(off[b + 1])
            calls.append((x[None, s:e], A[None, s:e], zi[b:b + 1], gy[None, s:e]))
            nsamp += e - s
        desc = f"{len(sel)} of {w['B']} ragged signals ({nsamp} samples), one call per signal"

    def once():
        for xs, As, zs, gs in calls:
            xx = xs.clone().requires_grad_(True)
            AA = As.clone().requires_grad_(True)
            zz = zs.clone().requires_grad_(True)
            Ae = AA[:, None, :].expand(-1, xx.shape[1], -1) if wl.time_invariant else AA
            y = ref.sample_wise_lpc(xx, Ae, zz)
            y.backward(gs)

    return once, nsamp, desc


def time_reference(ref, w, seconds: float):
    """Reference CPU fwd+bwd looped until `seconds` have elapsed (after one
    warm-up pass); returns (samples/s, description, seconds per pass)."""
    once, nsamp, desc = reference_calls(ref, w)
    once()
    t0 = time.perf_counter()
    reps = 0
    while True:
        once()
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds or reps >= 50:
            break
    return nsamp * reps / el, desc, el / reps


def run_reference(args):
    ws, rk, lr = rank_info()
    if rk != 0:
        return 0
    ref, why = reference_module()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    # inputs are generated on the host: this arm runs no GPU work and loads
    # none of this repository's native libraries
    w = load_workload(args.config, "cpu", B=args.B, T=args.T)
    once, nsamp, desc = reference_calls(ref, w)
    for _ in range(max(1, args.warmup)):
        once()
    secs = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        once()
        secs.append(time.perf_counter() - t0)
    per_step = sum(secs) / len(secs)
    value = nsamp / per_step
    threads = torch.get_num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_of(args, w, ws),
        "cpu_baseline": {"value": value, "unit": "samples/s", "cores": threads, "kind": "reference",
                         "sample": f"{desc}; reference torchlpc CPU operator (scan_cpu.cpp, OpenMP) + "
                                   f"its autograd backward, fp32"},
        "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------- reference CUDA kernels
REF_CUDA_T = 1 << 15  # samples per signal of the bounded sample the reference CUDA kernels are timed on


def run_reference_cuda_probe(args):
    """The reference's own CUDA path (torchlpc/csrc/cuda/lpc.cu and its
    autograd backward, built unmodified for sm_100a into oracle/_ref_cuda) on
    a bounded sample of the workload: all B signals, the first REF_CUDA_T
    samples.  Runs in its own process (it registers the torchlpc op
    namespace); prints one JSON line."""
    from oracle.build import build_reference_cuda

    path = build_reference_cuda()
    if path is None:
        print(json.dumps({"unavailable": "reference CUDA build (oracle/_ref_cuda) missing"}))
        return 0
    sys.path.insert(0, str(path))
    import warnings

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        import torchlpc
    if not torchlpc.EXTENSION_LOADED:
        print(json.dumps({"unavailable": "reference CUDA extension failed to load"}))
        return 0
    T = min(REF_CUDA_T, args.T) if args.T else REF_CUDA_T
    w = load_workload(args.config, "cpu", T=T)
    if w["workload"].ragged:
        print(json.dumps({"unavailable": "no ragged API in the reference"}))
        return 0
    dev = "cuda"
    x, A, zi, gy = (w[k].to(dev) for k in ("x", "A", "zi", "gy"))

    def step():
        xx, AA, zz = (t.clone().requires_grad_(True) for t in (x, A, zi))
        Ae = AA[:, None, :].expand(-1, w["T"], -1) if w["workload"].time_invariant else AA
        y = torchlpc.sample_wise_lpc(xx, Ae, zz)
        y.backward(gy)

    ms = time_loop(step, max(1, args.steps), max(1, args.warmup), torch.device(dev))
    S = samples_of(w)
    print(json.dumps({"value": S / (ms * 1e-3), "unit": "samples/s", "ms_per_step": ms,
                      "sample": f"{w['B']} signals x T={w['T']} (first samples of the workload's shapes)",
                      "path": "reference torchlpc CUDA kernel lpc.cu (one block per signal) + its autograd "
                              "backward, built unmodified for sm_100a"}))
    return 0


def reference_cuda_line(args):
    """Run the probe above in a child process; returns its JSON or an
    'unavailable' record."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference-cuda-probe", "--config", args.config,
           "--steps", "3", "--warmup", "1"]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        for line in reversed(r.stdout.strip().splitlines()):
            if line.startswith("{"):
                return json.loads(line)
        return {"unavailable": f"probe exited {r.returncode}: {r.stderr.strip().splitlines()[-1:]}"}
    except (subprocess.TimeoutExpired, OSError, ValueError) as e:
        return {"unavailable": f"probe failed: {e}"}


def other_configs(tl, headline: str, device) -> dict:
    """fwd+bwd samples/s of the other workloads at their full sizes (operator
    level, CUDA events; the default algorithm, and the plain kernel where it
    finishes in seconds), outside the timed region of the headline."""
    out = {}
    for cfg in ("cfg2", "cfg4", "cfg5"):
        if cfg == headline:
            continue
        w = load_workload(cfg, device)
        if w["workload"].ragged:
            w["offsets_dev"] = w["offsets"].to(device)
        S = samples_of(w)
        x, A, zi, gy = w["x"], w["A"], w["zi"], w["gy"]
        entry = {"samples_per_step": S, "note": w["workload"].note}
        for algo in ("auto", "plain"):
            if algo == "plain" and w["workload"].ragged:
                continue
            tl.set_algo(algo)
            tf, tb = kernel_times(tl, w, x, A, zi, gy, 3 if algo == "plain" else 10, device)
            entry[algo] = {"GS_per_s": S / ((tf + tb) * 1e-3) / 1e9, "fwd_ms": tf, "bwd_ms": tb}
        tl.set_algo("auto")
        entry["max_rel_err_vs_fp64"] = oracle_errors(tl, w, x, A, zi, gy,
                                                     max_signals=256 if w["workload"].time_invariant else None)
        out[cfg] = entry
        del w, x, A, zi, gy
        torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------------- main
def run_ours(args):
    ws, rk, lr = rank_info()
    if ws > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    device = torch.device("cuda", lr)
    torch.cuda.set_device(device)
    import torchlpc_b200 as tl
    from torchlpc_b200 import _ops

    assert tl.EXTENSION_LOADED
    tl.set_algo(args.algo)
    w = load_workload(args.config, device, seed=rk, B=args.B, T=args.T)
    if w["workload"].ragged:
        w["offsets_dev"] = w["offsets"].to(device)
    wl = w["workload"]
    S = samples_of(w)
    x = w["x"].requires_grad_(True)
    A = w["A"].requires_grad_(True)
    zi = w["zi"].requires_grad_(True)
    gy = w["gy"]
    step = make_step(tl, w, x, A, zi, gy)

    y0 = step()
    ckpt = y0.grad_fn is not None and "LPCBoundary" in type(y0.grad_fn).__name__
    del y0
    launches_per_step = count_kernels(step)
    sampler = ClockSampler(torch.cuda.current_device()) if rk == 0 else None
    if sampler:
        sampler.start()
    ms = time_loop(step, args.steps, max(3, args.warmup), device)
    clocks = sampler.stop() if sampler else None
    ms = max_over_ranks(ms, device)
    value = ws * S / (ms * 1e-3)

    line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; x, g ~ N(0,1); per-frame pole pairs interpolated per sample)",
            "config": config_of(args, w, ws), "algo": args.algo,
            "gpu_launches": launches_per_step * args.steps,
            "checkpointing": ("boundary states: the forward kernel keeps every half-chunk's entry state instead "
                              "of y; the backward recomputes y from them and x (one exact pass over independent "
                              "half-chunks) before the fused backward kernel" if ckpt else "off (y saved)")}
    if clocks:
        line["clocks"] = clocks

    if rk == 0:
        # roofline of the dominant kernel: the forward and the fused backward
        # kernels timed alone (the saved-y operators, one launch each; the
        # checkpointed backward operator adds the exact-pass recompute of y)
        tf, tb = kernel_times(tl, w, x, A, zi, gy, max(5, args.steps // 2), device, ckpt=ckpt)
        if ckpt:
            tkf, tkb = kernel_times(tl, w, x, A, zi, gy, max(5, args.steps // 2), device, ckpt=False)
        else:
            tkf, tkb = tf, tb
        peak, peak_kind = measured_peaks()
        bf, bb = bytes_per_sample(w["N"], wl.time_invariant)
        kern, t_k, b_k = ("backward", tkb, bb) if tkb >= tkf else ("forward", tkf, bf)
        achieved = S * b_k / (t_k * 1e-3) / 1e9
        tr = traffic_from_profiles(args.config, kern)
        line["roofline"] = {"bound": "hbm", "kernel": f"fused {kern} kernel (chunked scan)", "achieved": achieved,
                            "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                            "peak_source": peak_kind, "traffic": tr,
                            "algorithmic_bytes_per_launch": S * b_k, "launch_ms": t_k,
                            "bytes_per_sample": {"forward": bf, "backward": bb},
                            "kernel_frac": {"forward": S * bf / (tkf * 1e-3) / 1e9 / peak,
                                            "backward": S * bb / (tkb * 1e-3) / 1e9 / peak}}
        step_bytes = S * (bf + bb)
        line["hbm_frac_fwd_bwd"] = step_bytes / (ms * 1e-3) / 1e9 / peak
        line["kernel_ms"] = {"forward": tf, "backward": tb}
        if ckpt:
            line["kernel_ms"]["backward_kernel"] = tkb
            line["kernel_ms"]["recompute_pass"] = tb - tkb
        if ckpt:
            # the same step keeping y for the backward instead of the states
            old = tl.get_checkpointing()
            tl.set_checkpointing("off")
            mss = time_loop(step, args.steps, 3, device)
            tl.set_checkpointing(old)
            line["saved_y"] = {"value": S / (mss * 1e-3), "ms_per_step": mss,
                               "kernel_ms": {"forward": tkf, "backward": tkb}}
        # scan vs plain on the same GPU
        if args.algo != "plain" and "chunked" in tl.available_algos():
            tl.set_algo("plain")
            msp = time_loop(step, max(2, args.steps // 4), 1, device)
            tl.set_algo(args.algo)
            # the reference's own CUDA kernels on the same GPU (bounded sample)
            line["reference_cuda"] = reference_cuda_line(args)
            if "value" in line["reference_cuda"]:
                line["reference_cuda"]["ours_over_reference_cuda"] = value / line["reference_cuda"]["value"]
            line["plain"] = {"value": S / (msp * 1e-3), "ms_per_step": msp,
                             "speedup": msp / ms}
        line["max_rel_err_vs_fp64"] = oracle_errors(tl, w, x, A, zi, gy)
        if not args.no_extras and ws == 1:
            line["other_configs"] = other_configs(tl, args.config, device)
            tl.set_algo(args.algo)
        if not args.no_e2e:
            ems, h2d, d2h, nsl = e2e_time(tl, w, x, A, zi, gy, max(3, args.steps // 4), 3, device)
            line["e2e"] = {"value": S / (ems * 1e-3), "unit": "samples/s", "ms_per_step": ems,
                           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                           "pipeline": f"{nsl} groups of signals over 2 CUDA streams (copies overlap compute)"}
        if ws == 1 and not args.no_cpu_baseline:
            ref, why = reference_module()
            if ref is not None:
                v, desc, _ = time_reference(ref, w, args.cpu_seconds)
                line["cpu_baseline"] = {"value": v, "unit": "samples/s", "cores": torch.get_num_threads(),
                                        "kind": "reference",
                                        "sample": f"{desc}; reference torchlpc CPU operator + autograd, fp32, "
                                                  f"looped for ~{args.cpu_seconds:.0f} s"}
            else:
                line["cpu_baseline"] = {"value": None, "unavailable": why}
        print(json.dumps(line), flush=True)
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.impl == "reference-cuda-probe":
        return run_reference_cuda_probe(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
