"""GPU parity: the host-buffer grid pipeline (bf_grid_pipeline_*) against one
launch of the tensor-core grid over the whole block.  Chunks start on
multiples of lcm(128, S) spectra, so every product is bit-identical to the
single launch, including the partial last window and the last, shorter chunk;
the single launch itself is held to the FP64 bar by test_gpu_grid_tensor.py.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import grid_weights, random_voltage

pytestmark = pytest.mark.gpu
F = 336


def _whole(torch, api, v, w, T, A, B, S, shards):
    from beamform_project_b200 import native
    d = api.Dimensions(T, F, A, B)
    W = -(-T // S)
    qd = api.Dimensions(W, F, A, B)
    split = torch.empty(api.split_weight_bytes(d, shards), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, torch.from_numpy(w).cuda(), split, d, shards)
    integ = torch.empty(shards * W * F * B, dtype=torch.float32, device="cuda")
    codes = torch.empty(shards * W * F * B, dtype=torch.int8, device="cuda")
    params = torch.empty(shards * 2 * api.quantization_parameter_count(qd), dtype=torch.float32, device="cuda")
    api.grid_tensor_integrated(None, torch.from_numpy(v).cuda(), split, integ, codes, params, d, S, shards)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    return integ.cpu().numpy(), codes.cpu().numpy(), params.cpu().numpy()


@pytest.mark.parametrize("A,B,T,S,shards,chunk", [(64, 128, 3000, 320, 2, 640), (32, 37, 2565, 10, 1, 640),
                                                  (64, 16, 1900, 64, 2, 1280), (32, 128, 700, 320, 1, 0),
                                                  (64, 8, 5120, 32, 1, 1024), (128, 70, 1500, 64, 2, 256),
                                                  (256, 20, 700, 10, 1, 0)])
def test_pipeline_equals_single_launch(cuda, A, B, T, S, shards, chunk):
    from beamform_project_b200 import api
    torch = cuda
    v = np.stack([random_voltage(T, F, A, seed=60 + s) for s in range(shards)])
    w = np.stack([grid_weights(A, F, B, seed=70 + s) for s in range(shards)])
    exp_i, exp_c, exp_p = _whole(torch, api, v, w, T, A, B, S, shards)
    d = api.Dimensions(T, F, A, B)
    with api.GridHostPipeline(d, S, shards, chunk) as pipe:
        if chunk:
            assert pipe.chunk_spectra == min(chunk, -(-T // pipe.chunk_spectra) * pipe.chunk_spectra)
        pipe.upload_weights(w)
        got_i = np.full(exp_i.shape, -1.0, np.float32)
        got_c = np.full(exp_c.shape, 99, np.int8)
        got_p = np.full(exp_p.shape, -1.0, np.float32)
        ms = pipe.run(v.reshape(-1), got_i, got_c, got_p)
        assert ms > 0
        assert np.array_equal(got_i, exp_i)
        assert np.array_equal(got_c, exp_c)
        assert np.array_equal(got_p, exp_p)
        # pinned host tensors, codes only, a second block through the same pipeline
        hv = torch.from_numpy(v.reshape(-1)).pin_memory()
        hc = torch.zeros(exp_c.size, dtype=torch.int8).pin_memory()
        hp = torch.zeros(exp_p.size, dtype=torch.float32).pin_memory()
        pipe.run(hv, None, hc, hp)
        assert np.array_equal(hc.numpy(), exp_c)
        assert np.array_equal(hp.numpy(), exp_p)


def test_pipeline_errors(cuda):
    from beamform_project_b200 import api
    d = api.Dimensions(1280, F, 64, 16)
    v = random_voltage(1280, F, 64, seed=1)
    out = np.zeros(4 * F * 16, np.float32)
    with api.GridHostPipeline(d, 320) as pipe:
        with pytest.raises(api.LogicError, match="weights have not been uploaded"):
            pipe.run(v.reshape(-1), out)
        pipe.upload_weights(grid_weights(64, F, 16))
        with pytest.raises(api.InvalidArgument, match="both be given"):
            pipe.run(v.reshape(-1), out, np.zeros(out.size, np.int8))
        with pytest.raises(api.InvalidArgument, match="smaller than dimensions"):
            pipe.run(v.reshape(-1)[:100], out)
        pipe.run(v.reshape(-1), out)
    with pytest.raises(api.LogicError, match="closed"):
        pipe.run(v.reshape(-1), out)


@pytest.mark.parametrize("A,B,T,S,shards,chunk", [(64, 128, 3000, 320, 2, 640), (64, 24, 2000, 64, 1, 256),
                                                  (32, 40, 1300, 320, 1, 640)])
def test_checked_pipeline_equals_single_checked_launch(cuda, ref, A, B, T, S, shards, chunk):
    """The checked form through the host pipeline: chunks hold whole windows,
    so every window's covariance, estimate and recomputation are those of
    one launch over the block: bit-identical products.  The strong-source
    data (every beam a sidelobe) makes units fall back to the split kernel."""
    from beamform_project_b200 import api
    torch = cuda
    pos, freq = ref.ref_default_positions(A), ref.ref_channelized_frequencies(F)
    v = np.stack([ref.ref_make_moving_point_source(T, F, A, pos, freq, 0.0, -0.05 + 0.01 * s, 0.0, 0.0, 3.0)
                  for s in range(shards)])
    w = np.stack([grid_weights(A, F, B, seed=80 + s) for s in range(shards)])
    d = api.Dimensions(T, F, A, B)
    W = -(-T // S)
    qd = api.Dimensions(W, F, A, B)
    aw = torch.empty(api.auto_weight_bytes(d, shards), dtype=torch.uint8, device="cuda")
    api.prepare_auto_weights(None, torch.from_numpy(w).cuda(), aw, d, shards)
    ws = torch.zeros(max(256, api.grid_auto_workspace_bytes(d, S, shards)), dtype=torch.uint8, device="cuda")
    integ = torch.empty(shards * W * F * B, dtype=torch.float32, device="cuda")
    codes = torch.empty(shards * W * F * B, dtype=torch.int8, device="cuda")
    params = torch.empty(shards * 2 * api.quantization_parameter_count(qd), dtype=torch.float32, device="cuda")
    api.grid_auto_integrated(None, torch.from_numpy(v).cuda(), aw, integ, codes, params, ws, d, S, shards)
    torch.cuda.synchronize()
    with api.GridHostPipeline(d, S, shards, chunk, checked=True) as pipe:
        pipe.upload_weights(w)
        got_i = np.full(integ.numel(), -1.0, np.float32)
        got_c = np.full(codes.numel(), 99, np.int8)
        got_p = np.full(params.numel(), -1.0, np.float32)
        pipe.run(v.reshape(-1), got_i, got_c, got_p)
    assert np.array_equal(got_i, integ.cpu().numpy())
    assert np.array_equal(got_c, codes.cpu().numpy())
    assert np.array_equal(got_p, params.cpu().numpy())
