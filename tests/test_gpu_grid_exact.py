"""GPU parity: reference-order grid kernels, quantizer and generator.

The Direct/Tiled kernels reproduce the reference's float32 operation order,
so they must equal the oracle bit for bit (the oracle itself equals the
reference CPU core bit for bit, tests/test_oracle_pins.py).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import grid_weights, random_voltage, tile_weights

pytestmark = pytest.mark.gpu
F = 336


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("A,B,T", [(32, 16, 40), (64, 128, 19), (128, 33, 9), (256, 5, 6), (64, 1, 3)])
@pytest.mark.parametrize("kernel", [0, 1])
def test_per_spectrum_bit_exact(cuda, orc, A, B, T, kernel):
    from beamform_project_b200 import api
    torch = cuda
    v = random_voltage(T, F, A, seed=A + B)
    w = grid_weights(A, F, B, seed=T)
    wk = w if kernel == 0 else tile_weights(w)
    out = torch.full((T * F * B,), -1.0, dtype=torch.float32, device="cuda")
    api.launch_packed_beamformer(kernel, None, _dev(torch, v), _dev(torch, wk), out,
                                 api.Dimensions(T, F, A, B))
    got = out.cpu().numpy().reshape(T, F, B)
    assert np.array_equal(got, orc.beamform(v, w, T, F, A, B))


@pytest.mark.parametrize("A,B,T,S", [(32, 16, 1024, 10), (64, 128, 650, 320), (64, 7, 33, 7),
                                     (128, 40, 70, 32), (256, 3, 20, 320), (32, 1, 321, 320)])
@pytest.mark.parametrize("kernel", [0, 1])
def test_integrated_bit_exact(cuda, orc, A, B, T, S, kernel):
    from beamform_project_b200 import api
    torch = cuda
    v = random_voltage(T, F, A, seed=S)
    w = grid_weights(A, F, B, seed=A)
    wk = w if kernel == 0 else tile_weights(w)
    W = -(-T // S)
    out = torch.full((W * F * B + 1,), -7.0, dtype=torch.float32, device="cuda")
    api.launch_packed_integrated_beamformer(kernel, None, _dev(torch, v), _dev(torch, wk), out,
                                            api.Dimensions(T, F, A, B), S)
    got = out.cpu().numpy()
    assert got[-1] == -7.0  # writes only the prefix (reference _into contract)
    assert np.array_equal(got[:-1].reshape(W, F, B), orc.beamform_integrated(v, w, T, F, A, B, S))


def test_known_answers_on_gpu(cuda, orc):
    # one-hot {3,-2} -> 13 (tests/cpu/test_cpu_beamformer.cpp:112-124),
    # constant {7,-8} at broadside -> A^2 * 113 (tests/cuda/test_cuda_packed.cu:178-189)
    from beamform_project_b200 import api
    torch = cuda
    A = 32
    pos, freq = api.default_positions(A), api.channelized_frequencies(F)
    dirs = np.stack([api.direction_from_lm(np.float32(b - 2) * np.float32(0.02), 0.0) for b in range(5)])
    w = orc.generate_weights(pos, freq, dirs)
    v = np.zeros((1, F, A), np.uint8)
    v[0, 17, 7] = orc.oracle().orc_pack(3, -2)
    out = api.cuda_beamform_packed_intensity(v, w, api.Dimensions(1, F, A, 5))
    exp = np.zeros((1, F, 5), np.float32)
    exp[0, 17] = 13.0
    assert np.allclose(out.reshape(1, F, 5), exp, rtol=1e-5, atol=1e-5)
    wb = orc.generate_weights(pos, freq, np.array([[0, 0, 1]], np.float32))
    vc = np.full((4, F, A), orc.oracle().orc_pack(7, -8), np.uint8)
    o = api.cuda_beamform_packed_integrated_intensity(vc, wb, api.Dimensions(4, F, A, 1), 320,
                                                      kernel=api.CudaBeamformerKernel.Direct)
    assert np.all(o == np.float32(4 * A * A * 113))


@pytest.mark.parametrize("W,B", [(2, 17), (103, 128), (5, 1), (3, 40)])
def test_quantizer_bit_exact(cuda, orc, W, B):
    from beamform_project_b200 import api
    torch = cuda
    I = np.random.default_rng(W * B).gamma(2.0, 400.0, size=(W, F, B)).astype(np.float32)
    if W > 2:
        I[1, 20, 0] = np.nan
        I[2, 300, B - 1] = np.inf
        I[0, 16:32, :16] = 5.0  # degenerate chunk
    qd = api.Dimensions(W, F, 32, B)
    codes = torch.zeros(W * F * B, dtype=torch.int8, device="cuda")
    params = torch.zeros(2 * api.quantization_parameter_count(qd), dtype=torch.float32, device="cuda")
    api.launch_quantize_integrated_intensity(None, _dev(torch, I), codes, params, qd)
    rc, rp = orc.quantize(I, W, F, B)
    assert np.array_equal(codes.cpu().numpy().reshape(W, F, B), rc)
    assert np.array_equal(params.cpu().numpy().reshape(rp.shape), rp)


@pytest.mark.parametrize("W,B", [(4, 16), (3, 12), (2, 8), (2, 20)])
def test_quantizer_ties_bit_exact(cuda, orc, W, B):
    """Integer values whose chunks span exactly 0 .. 255: scale 1, offset
    127.5, so every quotient is a half-integer and rounds by ties to even;
    beam counts on the vector path (multiples of four, also a partial beam
    tile) and off it."""
    from beamform_project_b200 import api
    torch = cuda
    I = np.random.default_rng(W + B).integers(0, 256, size=(W, F, B)).astype(np.float32)
    for ft in range(0, F, 16):
        for bt in range(0, B, 16):
            I[:, ft, bt] = 0.0
            I[:, ft + 1, bt] = 255.0
    qd = api.Dimensions(W, F, 32, B)
    codes = torch.zeros(W * F * B, dtype=torch.int8, device="cuda")
    params = torch.zeros(2 * api.quantization_parameter_count(qd), dtype=torch.float32, device="cuda")
    api.launch_quantize_integrated_intensity(None, _dev(torch, I), codes, params, qd)
    rc, rp = orc.quantize(I, W, F, B)
    assert np.array_equal(params.cpu().numpy().reshape(rp.shape), rp)
    assert np.array_equal(codes.cpu().numpy().reshape(W, F, B), rc)


def test_quantized_pipeline_matches_oracle_chain(cuda, orc):
    from beamform_project_b200 import api
    T, A, B, S = 700, 64, 20, 320
    v = random_voltage(T, F, A, 3)
    w = grid_weights(A, F, B, 3)
    codes, params = api.cuda_beamform_packed_quantized_integrated_intensity(
        v, tile_weights(w), api.Dimensions(T, F, A, B), S)
    ref_int = orc.beamform_integrated(v, w, T, F, A, B, S)
    rc, rp = orc.quantize(ref_int, 3, F, B)
    assert np.array_equal(codes.reshape(rc.shape), rc)
    assert np.array_equal(params.reshape(rp.shape), rp)


def test_generator_bit_exact(cuda, orc):
    from beamform_project_b200 import api
    torch = cuda
    T, A = 37, 64
    scale = api.generator_scale(2.5)
    out = torch.zeros(T * F * A, dtype=torch.uint8, device="cuda")
    api.generate_voltage(None, 12345, 0, 2.5, None, 1, out, api.Dimensions(T, F, A, 1))
    assert np.array_equal(out.cpu().numpy().reshape(T, F, A),
                          orc.generate_voltage(12345, 0, T, F, A, scale))
    mu = np.random.default_rng(0).normal(0, 3, size=(4, F, A, 2)).astype(np.float32)
    api.generate_voltage(None, 7, 999, 2.5, _dev(torch, mu), 10, out, api.Dimensions(T, F, A, 1))
    assert np.array_equal(out.cpu().numpy().reshape(T, F, A),
                          orc.generate_voltage(7, 999, T, F, A, scale, mu, 10))
