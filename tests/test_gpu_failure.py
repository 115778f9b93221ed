"""Failure detection without a GPU fault: a bounded device wait that runs out
returns an error status the host reads, and the context stays usable."""
from __future__ import annotations

import time

import numpy as np
import pytest

from beamform_project_b200 import native


def test_probe_rejects_unbounded_limits():
    lib = native.lib()
    assert lib.bf_probe_bounded_wait(None, 0) == native.InvalidArgument(1, "").status
    assert lib.bf_probe_bounded_wait(None, 3 * 10**9) == 1
    assert "limit_ns" in native.last_error()


@pytest.mark.gpu
def test_wait_that_runs_out_is_reported_and_context_survives(cuda, orc):
    from beamform_project_b200 import api
    from conftest import grid_weights, random_voltage
    torch = cuda
    assert native.take_device_error() == 0
    t0 = time.perf_counter()
    native.check(native.lib().bf_probe_bounded_wait(None, 200_000_000))
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    code = native.take_device_error()
    assert code & (1 << 30), hex(code)
    assert 0.15 < elapsed < 5.0
    assert native.take_device_error() == 0          # read and cleared
    # the context still runs the tensor kernel correctly
    T, F, A, B, S = 256, 336, 64, 16, 128
    v = random_voltage(T, F, A, seed=7)
    w = grid_weights(A, F, B, seed=7)
    d = api.Dimensions(T, F, A, B)
    split = torch.empty(api.split_weight_bytes(d), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, torch.from_numpy(w).cuda(), split, d)
    out = torch.empty(2 * F * B, dtype=torch.float32, device="cuda")
    api.grid_tensor_integrated(None, torch.from_numpy(v).cuda(), split, out, None, None, d, S)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    ref = orc.beamform_integrated(v, w, T, F, A, B, S, f64=True)
    got = out.cpu().numpy().reshape(2, F, B).astype(np.float64)
    assert np.all(np.abs(got - ref) <= 1e-3 + 1e-5 * np.abs(ref))
