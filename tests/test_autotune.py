"""The grid path's autotuner (bf_autotune_grid, bf_tune_*).

CPU: the selection rule with made-up timings (a fake timer: the rule sees
only the times and the parity flags), the tuning table and its cache file.
GPU: tuning a class records a choice that later untuned calls use, and every
candidate choice, run explicitly, is within the path's bar of the FP64
oracle (the tuner's own gate compares candidates with the default only).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from beamform_project_b200 import api, native
from conftest import grid_weights, random_voltage

F = 336


def _pick(ms, ok, min_gain=0.02):
    n = len(ms)
    best = C.c_uint32(99)
    native.check(native.lib().bf_tune_pick(n, (C.c_double * n)(*ms), (C.c_uint8 * n)(*ok), min_gain,
                                           C.byref(best)))
    return best.value


def test_pick_fastest_passing_candidate():
    assert _pick([2.0, 1.5, 1.2, 1.9], [1, 1, 1, 1]) == 2


def test_pick_skips_candidates_that_failed_parity():
    assert _pick([2.0, 1.5, 1.2, 1.9], [1, 1, 0, 1]) == 1


def test_pick_keeps_the_default_within_the_noise_margin():
    assert _pick([2.0, 1.99, 1.97], [1, 1, 1]) == 0          # 1.5 % faster: noise
    assert _pick([2.0, 1.99, 1.95], [1, 1, 1]) == 2          # 2.5 % faster
    assert _pick([2.0, 1.99, 1.97], [1, 1, 1], min_gain=0.0) == 2


def test_pick_when_the_default_failed():
    assert _pick([1.0, 3.0, 2.0], [0, 1, 1]) == 2
    assert _pick([1.0, 3.0], [0, 0]) == 0


def test_pick_rejects_empty_input():
    best = C.c_uint32(0)
    st = native.lib().bf_tune_pick(0, None, None, 0.0, C.byref(best))
    assert st == 1


def test_table_set_get_save_load(tmp_path, clean_table):
    path = str(tmp_path / "cache.txt")
    assert api.tune_get(64, 128, 320, device="NVIDIA B200") is None
    api.tune_set(64, 128, 320, form=1, group_mult=2, paired=False, ms=1.5, device="NVIDIA B200")
    api.tune_set(32, 16, 10, form=0, group_mult=4, paired=True, ms=0.1, device="NVIDIA B200")
    assert api.tune_get(64, 128, 320, device="NVIDIA B200") == {"form": "checked covariance", "group_mult": 2,
                                                                "paired": False}
    assert api.tune_get(64, 128, 320, device="Other GPU") is None
    api.tune_save(path)
    text = open(path).read()
    assert "NVIDIA_B200 64 128 320 1 2 0" in text
    api.tune_clear()
    assert api.tune_get(32, 16, 10, device="NVIDIA B200") is None
    api.tune_load(path)
    assert api.tune_get(32, 16, 10, device="NVIDIA B200") == {"form": "split", "group_mult": 4, "paired": True}


def test_table_ignores_malformed_lines(tmp_path, clean_table):
    path = tmp_path / "cache.txt"
    path.write_text("# header\nNVIDIA_B200 64 128 320 7 1 1 0.5\nNVIDIA_B200 64 64 320 0 0 1 0.5\n"
                    "garbage line\nNVIDIA_B200 64 32 64 0 2 1 0.25\n")
    api.tune_clear()
    api.tune_load(str(path))
    assert api.tune_get(64, 128, 320, device="NVIDIA B200") is None   # form 7
    assert api.tune_get(64, 64, 320, device="NVIDIA B200") is None    # group 0
    assert api.tune_get(64, 32, 64, device="NVIDIA B200") == {"form": "split", "group_mult": 2, "paired": True}


def test_set_rejects_invalid_choices():
    with pytest.raises(api.InvalidArgument):
        api.tune_set(64, 128, 320, form=2, group_mult=1, paired=True, device="x")
    with pytest.raises(api.InvalidArgument):
        api.tune_set(64, 128, 320, form=0, group_mult=0, paired=True, device="x")


def test_cache_path_is_beside_the_library_or_from_the_environment():
    import os
    p = api.tune_cache_path()
    if "BF_TUNE_CACHE" in os.environ:
        assert p == os.environ["BF_TUNE_CACHE"]
    else:
        assert p == str(native.library_path().parent / "bf_tune_cache.txt")


@pytest.fixture
def clean_table():
    api.tune_clear()
    yield
    api.tune_clear()


@pytest.mark.gpu
@pytest.mark.parametrize("A,B,T,S", [(64, 128, 1280, 320), (64, 16, 1280, 320), (32, 40, 700, 10), (128, 40, 640, 64)])
def test_autotune_records_a_choice_and_every_candidate_meets_the_bar(cuda, orc, clean_table, A, B, T, S):
    torch = cuda
    d = api.Dimensions(T, F, A, B)
    res = api.autotune_grid(None, d, S, 1)
    print(res)
    cands = res["candidates"]
    assert len(cands) >= 6 and all(c["ms"] > 0 for c in cands)
    assert all(c["ok"] for c in cands)
    nbp = -(-B // 16) * 16
    chosen = api.tune_get(A, nbp, S)
    assert chosen is not None and chosen["form"] == res["chosen"]["form"]
    # every candidate, run explicitly on new data, against the FP64 oracle
    v = random_voltage(T, F, A, seed=A + B + S)
    w = grid_weights(A, F, B, seed=T)
    wd = torch.from_numpy(w).cuda()
    aw = torch.empty(api.auto_weight_bytes(d), dtype=torch.uint8, device="cuda")
    api.prepare_auto_weights(None, wd, aw, d)
    ws = torch.zeros(max(256, api.grid_auto_workspace_bytes(d, S)), dtype=torch.uint8, device="cuda")
    W = -(-T // S)
    ref64 = orc.beamform_integrated(v, w, T, F, A, B, S, f64=True)
    vd = torch.from_numpy(v).cuda()
    outs = []
    for c in cands:
        out = torch.empty(W * F * B, dtype=torch.float32, device="cuda")
        form = 1 if c["form"] == "checked covariance" else 0
        api.grid_auto_integrated_with(None, vd, aw, out, None, None, ws, d, S, 1, form, c["group_mult"], c["paired"])
        torch.cuda.synchronize()
        assert native.take_device_error() == 0
        got = out.cpu().numpy().reshape(W, F, B).astype(np.float64)
        assert np.all(np.abs(got - ref64) <= 1e-3 + 1e-5 * np.abs(ref64)), c
        outs.append((form, got))
    split = [g for f, g in outs if f == 0]
    assert all(np.array_equal(split[0], g) for g in split[1:])  # scheduling only
    # an untuned call now runs the recorded choice: the same products as running it explicitly
    form = 1 if chosen["form"] == "checked covariance" else 0
    exp = torch.empty(W * F * B, dtype=torch.float32, device="cuda")
    api.grid_auto_integrated_with(None, vd, aw, exp, None, None, ws, d, S, 1, form, chosen["group_mult"],
                                  chosen["paired"])
    out = torch.empty(W * F * B, dtype=torch.float32, device="cuda")
    api.grid_auto_integrated(None, vd, aw, out, None, None, ws, d, S)
    torch.cuda.synchronize()
    assert torch.equal(exp, out)
