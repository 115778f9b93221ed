"""bf_grid_tensor_quantized_static: the allocation-free entry point.

Callers that cannot allocate device memory (memory fixed at start-up, or an
FFI caller holding only a stream and its data buffers) use this variant of
bf_grid_tensor_quantized; its scratch is a fixed array inside the library.
This file is collected last so a run that stops at the first failure has run
every other test first; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from beamform_project_b200 import native
from beamform_project_b200.native import Dims

F = 336
_P = C.c_void_p


def _static_fn():
    fn = native.lib().bf_grid_tensor_quantized_static
    fn.restype = C.c_int
    fn.argtypes = [_P, _P, _P, _P, _P, _P, C.POINTER(Dims), C.c_uint64, C.c_uint64]
    return fn


def test_static_entry_rejects_requests_beyond_its_scratch():
    """2 shards x 8192 windows x 21 channel groups needs 344064 counters > 16384;
    the check runs before any CUDA call."""
    d = Dims(8192 * 32, F, 64, 128)
    fake = C.c_void_p(4096)
    st = _static_fn()(None, fake, fake, fake, fake, fake, C.byref(d), 32, 2)
    assert st == native.BF_OK + 1
    assert "at most 16384" in native.last_error()


def test_static_entry_short_windows_are_not_held_to_the_array_size():
    """Windows below 32 spectra quantize in a second kernel and use no counters:
    16 spectra x 2048 windows x 21 groups x 2 shards (86016) passes the size
    check.  Null buffers then stop the call before any CUDA call, with the
    buffer message instead of the size message."""
    d = Dims(2048 * 16, F, 64, 128)
    st = _static_fn()(None, None, None, None, None, None, C.byref(d), 16, 2)
    assert st == native.BF_OK + 1
    msg = native.last_error()
    assert "every buffer must be given" in msg and "at most" not in msg


@pytest.mark.gpu
def test_static_entry_matches_allocating_entry_twice(cuda):
    from beamform_project_b200 import api
    torch = cuda
    T, A, B, S, shards = 1000, 64, 100, 320, 2
    d = api.Dimensions(T, F, A, B)
    W = -(-T // S)
    qd = api.Dimensions(W, F, A, B)
    rng = np.random.default_rng(2024)
    v = torch.from_numpy(rng.integers(0, 256, size=(shards, T, F, A), dtype=np.uint8)).cuda()
    ph = rng.uniform(-np.pi, np.pi, size=(shards, B, F, A))
    w = torch.from_numpy(np.stack([np.cos(ph), np.sin(ph)], -1).astype(np.float32)).cuda()
    split = torch.empty(api.split_weight_bytes(d, shards), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, w, split, d, shards)
    n_out = shards * W * F * B
    n_par = shards * 2 * api.quantization_parameter_count(qd)

    # the existing entry point, with a caller-allocated workspace
    ref_i = torch.empty(n_out, dtype=torch.float32, device="cuda")
    ref_c = torch.empty(n_out, dtype=torch.int8, device="cuda")
    ref_p = torch.empty(n_par, dtype=torch.float32, device="cuda")
    ws = torch.zeros(api.grid_tensor_workspace_bytes(d, S, shards), dtype=torch.uint8, device="cuda")
    api.grid_tensor_quantized(None, v, split, ref_i, ref_c, ref_p, ws, d, S, shards)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0

    fn = _static_fn()
    cd = d.c()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # the second call finds the previous call's counts in the array
        out_i = torch.full((n_out,), -1.0, dtype=torch.float32, device="cuda")
        out_c = torch.full((n_out,), 55, dtype=torch.int8, device="cuda")
        out_p = torch.full((n_par,), -1.0, dtype=torch.float32, device="cuda")
        native.check(fn(stream, v.data_ptr(), split.data_ptr(), out_i.data_ptr(), out_c.data_ptr(),
                        out_p.data_ptr(), C.byref(cd), S, shards))
        torch.cuda.synchronize()
        assert native.take_device_error() == 0, f"call {call}"
        got, exp = out_i.cpu().numpy(), ref_i.cpu().numpy()
        assert np.all(np.abs(got.astype(np.float64) - exp) <= 1e-3 + 1e-5 * np.abs(exp)), f"call {call}"
        assert torch.equal(out_c, ref_c), f"call {call}"
        assert torch.allclose(out_p, ref_p, rtol=1e-6, atol=0.0), f"call {call}"
