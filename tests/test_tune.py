"""Autotuner: shape buckets, candidate sets, and the tuned mode end to end."""
import numpy as np
import pytest
import torch

import torchlpc_b200 as tl
from torchlpc_b200 import _ops, tune


def test_key_buckets_and_candidates():
    assert tune.key(3, 1000, 16, torch.float32, False) == tune.key(4, 1024, 16, torch.float32, False)
    assert tune.key(4, 1025, 16, torch.float32, False) != tune.key(4, 1024, 16, torch.float32, False)
    assert tune.key(4, 1024, 16, torch.float32, True) != tune.key(4, 1024, 16, torch.float32, False)
    c = tune.candidates(16, False)
    assert ("plain", 0) in c and ("chunked", 256) in c and all(a != "ti" for a, _ in c)
    assert ("ti", 0) in tune.candidates(32, True)
    assert tune.candidates(40, True) == [("plain", 0)]  # no scan above order 32


@pytest.mark.gpu
def test_tuned_mode_matches_auto(tmp_path, monkeypatch):
    monkeypatch.setenv("LPC_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(tune, "_LOADED", False)
    monkeypatch.setattr(tune, "_TABLE", {})
    cfg = tune.autotune(4, 20000, 16, torch.float32, False, reps=1)
    assert (cfg["algo"], cfg["chunk"]) in tune.candidates(16, False)
    assert tune.lookup(4, 20000, 16, torch.float32, False)["algo"] == cfg["algo"]
    assert (tmp_path / "tune.json").exists()
    g = torch.Generator().manual_seed(0)
    x = torch.randn(4, 20000, generator=g).cuda()
    A = (torch.rand(4, 20000, 16, generator=g) * 0.05).cuda()
    outs = []
    for algo in ("tuned", "auto"):
        old = tl.get_algo()
        tl.set_algo(algo)
        try:
            outs.append(tl.sample_wise_lpc(x, A).cpu().numpy())
        finally:
            tl.set_algo(old)
            _ops.set_chunk_length(0)
    assert np.abs(outs[0] - outs[1]).max() <= 1e-5 * max(1.0, np.abs(outs[1]).max())
