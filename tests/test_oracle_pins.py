"""Pin the oracle (C restatement) to the reference.

Two kinds of pins:
  * the reference's own known-answer tests, restated (tests/cpu/*.cpp in the
    reference, cited per test);
  * bit-exact agreement with the reference CPU core itself, compiled from its
    sources into oracle/_ref/libbfref.so, on identical inputs.
CPU only.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import grid_weights, random_voltage, tile_weights

F = 336


def default_grid_dirs(B: int, l_step: float = 0.02) -> np.ndarray:
    """default_beam_grid (geometry.cpp:108-125)."""
    from beamform_project_b200.api import direction_from_lm
    c = B // 2
    return np.stack([direction_from_lm(np.float32(b - c) * np.float32(l_step), 0.0) for b in range(B)])


def test_nibble_decode_all_256(orc):
    # tests/cpu/test_contract.cpp:34-47 and tests/cpu/test_cpu_beamformer.cpp:64-72
    raw = np.arange(256, dtype=np.uint8)
    re, im = orc.unpack(raw)
    lo, hi = raw & 0xF, raw >> 4
    assert np.array_equal(re, np.where(lo < 8, lo, lo.astype(int) - 16))
    assert np.array_equal(im, np.where(hi < 8, hi, hi.astype(int) - 16))
    for r in range(-8, 8):
        for i in range(-8, 8):
            b = orc.oracle().orc_pack(r, i)
            rr, ii = orc.unpack(np.array([b], np.uint8))
            assert (rr[0], ii[0]) == (r, i)
    assert orc.oracle().orc_pack(8, 0) == -1 and orc.oracle().orc_pack(0, -9) == -1
    re, im = orc.unpack(np.array([0x07, 0x08, 0x70, 0x80], np.uint8))
    assert re[0] == 7 and re[1] == -8 and im[2] == 7 and im[3] == -8


def test_geometry_matches_reference(ref):
    from beamform_project_b200 import api
    for A in (32, 64, 128, 256):
        assert np.array_equal(api.default_positions(A), ref.ref_default_positions(A))
    assert np.array_equal(api.channelized_frequencies(F), ref.ref_channelized_frequencies(F))


def test_weights_bit_exact_vs_reference(orc, ref):
    from beamform_project_b200 import api
    pos = api.default_positions(32)
    freq = api.channelized_frequencies(F)
    dirs = default_grid_dirs(5)
    w = orc.generate_weights(pos, freq, dirs)
    assert np.array_equal(w, ref.ref_generate_weights(pos, freq, dirs))
    # unit modulus (tests/cpu/test_cpu_beamformer.cpp:78-80)
    assert np.allclose(w[..., 0] ** 2 + w[..., 1] ** 2, 1.0, atol=1e-6)
    # tiled layout equals canonical, padding zero (test_cpu_beamformer.cpp:81-110)
    assert np.array_equal(tile_weights(w), ref.ref_generate_weights(pos, freq, dirs, tiled=True))


def test_one_hot_power_13(orc, ref):
    # tests/cpu/test_cpu_beamformer.cpp:112-124
    from beamform_project_b200 import api
    A, B = 32, 5
    w = orc.generate_weights(api.default_positions(A), api.channelized_frequencies(F), default_grid_dirs(B))
    v = ref.ref_make_one_hot(1, F, A, 0, 17, 7, 3, -2)
    I = orc.beamform(v, w, 1, F, A, B)
    expected = np.zeros((1, F, B), np.float32)
    expected[0, 17, :] = 13.0
    assert np.allclose(I, expected, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("value,power", [((1, 0), 1), ((7, -8), 113)])
def test_constant_broadside(orc, value, power):
    # tests/cpu/test_cpu_beamformer.cpp:144-160, tests/cuda/test_cuda_packed.cu:178-189
    from beamform_project_b200 import api
    for A in (32, 64):
        w = orc.generate_weights(api.default_positions(A), api.channelized_frequencies(F),
                                 np.array([[0.0, 0.0, 1.0]], np.float32))
        v = np.full((2, F, A), orc.oracle().orc_pack(*value), np.uint8)
        I = orc.beamform(v, w, 2, F, A, 1)
        assert np.all(I == np.float32(A * A * power))


def test_point_source_peak(orc, ref):
    # tests/cpu/test_cpu_beamformer.cpp:162-186 (peak at beam 4 of 5)
    from beamform_project_b200 import api
    A, B = 32, 5
    pos, freq = api.default_positions(A), api.channelized_frequencies(F)
    w = orc.generate_weights(pos, freq, default_grid_dirs(B))
    v = ref.ref_make_point_source(1, F, A, pos, freq, api.direction_from_lm(0.04, 0.0), 4.0)
    I = orc.beamform(v, w, 1, F, A, B)
    assert int(np.argmax(I.astype(np.float64).sum(axis=(0, 1)))) == 4


def test_beamformer_bit_exact_vs_reference(orc, ref):
    # noise from the reference generator (synthetic_data.cpp:107-119) and random bytes
    for T, A, B, seed in [(2, 32, 2, 4242), (3, 64, 17, 7)]:
        v = ref.ref_make_noise(T, F, A, seed)
        w = grid_weights(A, F, B, seed)
        assert np.array_equal(orc.beamform(v, w, T, F, A, B), ref.ref_beamform(v, w, T, F, A, B))
    v = random_voltage(3, F, 32, 5)
    w = grid_weights(32, F, 33, 5)
    assert np.array_equal(orc.beamform(v, w, 3, F, 32, 33), ref.ref_beamform(v, w, 3, F, 32, 33))


def test_integration_bit_exact_and_kats(orc, ref):
    # tests/cpu/test_temporal_integration.cpp:57-120
    T, B = 7, 3
    I = (100 * np.arange(T)[:, None, None] + 10 * np.arange(F)[None, :, None]
         + np.arange(B)[None, None, :]).astype(np.float32)
    for S in (1, 3, 320):
        assert np.array_equal(orc.integrate(I, T, F, B, S), ref.ref_integrate(I, T, F, 32, B, S))
    ones = np.ones((321, F, 1), np.float32)
    part = orc.integrate(ones, 321, F, 1, 320)
    assert part.shape == (2, F, 1) and np.all(part[0] == 320.0) and np.all(part[1] == 1.0)
    up = orc.integrate(np.ones((480, F, 3), np.float32), 480, F, 3, 10)
    assert up.shape == (48, F, 3) and np.all(up == 10.0)
    assert orc.oracle().orc_window_count(15360, 320) == 48


def test_fused_oracle_equals_chain(orc):
    T, A, B, S = 23, 32, 4, 10
    v = random_voltage(T, F, A, 11)
    w = grid_weights(A, F, B, 11)
    chain = orc.integrate(orc.beamform(v, w, T, F, A, B), T, F, B, S)
    assert np.array_equal(orc.beamform_integrated(v, w, T, F, A, B, S), chain)
    sub = orc.beamform_integrated(v, w, T, F, A, B, S, windows=[0, 2])
    assert np.array_equal(sub[[0, 2]], chain[[0, 2]])


def test_quantizer_kats_and_bit_exact(orc, ref):
    # tests/cpu/test_quantization.cpp:38-110
    W, B = 2, 17
    I = (1000 * np.arange(W)[:, None, None] + 10 * np.arange(F)[None, :, None]
         + np.arange(B)[None, None, :]).astype(np.float32)
    codes, params = orc.quantize(I, W, F, B)
    assert params.shape == (2, 21, 2, 2) and params.size // 2 == 84
    assert codes[0, 0, 0] == -127 and codes[0, 15, 15] == 127
    assert codes[0, 0, 16] == -127 and codes[0, 15, 16] == 127
    rc, rp = ref.ref_quantize(I, W, F, 32, B)
    assert np.array_equal(codes, rc) and np.array_equal(params, rp)
    # reconstruction within half a bin
    p = params[np.arange(W)[:, None, None], np.arange(F)[None, :, None] // 16,
               np.arange(B)[None, None, :] // 16]
    recon = p[..., 0] + p[..., 1] * codes.astype(np.float32)
    assert np.all(np.abs(recon - I) <= p[..., 1] * 0.5 + 5e-4)
    # degenerate chunk: scale 0, offset = value, codes 0
    const = np.full((1, F, 1), 42.0, np.float32)
    c, pp = orc.quantize(const, 1, F, 1)
    assert np.all(pp[..., 1] == 0.0) and np.all(pp[..., 0] == 42.0) and np.all(c == 0)
    # non-finite: code -128 and a zero parameter pair for its chunk
    nf = const.copy()
    nf[0, 0, 0] = np.nan
    c, pp = orc.quantize(nf, 1, F, 1)
    assert c[0, 0, 0] == -128 and pp[0, 0, 0, 0] == 0.0 and pp[0, 0, 0, 1] == 0.0
    rc, rp = ref.ref_quantize(nf, 1, F, 32, 1)
    assert np.array_equal(c, rc) and np.array_equal(pp, rp)
    # random data with inf entries
    rnd = np.random.default_rng(3).gamma(2.0, 50.0, size=(5, F, 40)).astype(np.float32)
    rnd[1, 3, 5] = np.inf
    c, pp = orc.quantize(rnd, 5, F, 40)
    rc, rp = ref.ref_quantize(rnd, 5, F, 32, 40)
    assert np.array_equal(c, rc) and np.array_equal(pp, rp)


def test_tracker_bit_exact_vs_reference(orc, ref):
    # beam_tracker.cpp:90-146 on the default geometry, drifting trajectory
    from beamform_project_b200 import api
    T, A, S = 40, 32, 16
    l0, m0, rl, rm = 0.01, -0.02, 2e-4, 1e-4
    pos, freq = api.default_positions(A), api.channelized_frequencies(F)
    v = ref.ref_make_moving_point_source(T, F, A, pos, freq, l0, m0, rl, rm, 4.0)
    dirs = api.tracker_window_directions(l0, m0, rl, rm, T, S)
    for w in range(len(dirs)):
        assert np.array_equal(dirs[w], ref.ref_tracker_window_direction(l0, m0, rl, rm, w, S))
    ww = orc.tracker_weights(dirs, pos, freq)
    ours = orc.tracker(v, ww, T, F, A, S)
    naive = ref.ref_tracker(v, T, F, A, l0, m0, rl, rm, S, variant=0)
    opt_v2 = ref.ref_tracker(v, T, F, A, l0, m0, rl, rm, S, variant=1)
    assert np.array_equal(ours, naive)
    assert np.array_equal(naive, opt_v2)  # tests/cpu/test_beam_tracker_opt_v2.cpp:50-79
    # constant trajectory equals the one-beam grid (tests/cpu/test_beam_tracker.cpp:121-139)
    still = ref.ref_tracker(v, T, F, A, l0, m0, 0.0, 0.0, S)
    w1 = orc.generate_weights(pos, freq, api.direction_from_lm(l0, m0)[None])
    assert np.array_equal(still, orc.beamform(v, w1, T, F, A, 1)[..., 0])


def test_generator_statistics_and_determinism(orc):
    from beamform_project_b200.api import generator_scale
    scale = generator_scale(2.0)
    a = orc.generate_voltage(1, 0, 64, F, 32, scale)
    b = orc.generate_voltage(1, 0, 64, F, 32, scale)
    c = orc.generate_voltage(2, 0, 64, F, 32, scale)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    re, im = orc.unpack(a)
    for x in (re, im):
        assert abs(float(x.mean())) < 0.02
        assert 1.9 < float(x.std()) < 2.1
    # offset: the sample counter continues across blocks
    whole = orc.generate_voltage(9, 0, 8, F, 32, scale)
    tail = orc.generate_voltage(9, 4 * F * 32, 4, F, 32, scale)
    assert np.array_equal(whole[4:], tail)
