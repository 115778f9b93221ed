"""DOA: exact block covariance on int8 tensor cores and the FP64 scan.

Covariance: bit-exact against the integer restatement (int64 sums of
x x^H).  Scan: against the FP64 oracle (orc_doa_scan) to 1e-6 relative
(the only freedom is the last bit of the float sin/cos of the reduced
phase).  The oracle itself is pinned to the reference's CpuOptBeamTracker
search on a source (CPU test below).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import rng, random_voltage

F = 336
C_LIGHT = 299_792_458.0


def geometry(A=64):
    lam = C_LIGHT / 800e6
    sp = 0.5 * lam
    cols = 32 if A >= 32 else A
    pos = np.zeros((A, 3), np.float32)
    for i in range(A):
        pos[i] = ((i % cols) * sp, (i // cols) * sp, 0.0)
    freq = (400e6 + np.arange(F) * (400e6 / 671)).astype(np.float32)
    kw = 2 * math.pi * freq.astype(np.float64) / C_LIGHT
    return pos, freq, kw


def source_voltage(T, A, sources, sigma=2.0, seed=0, multipath=None):
    """Complex Gaussian source waveforms (per spectrum and channel) along
    steering exp(-j k x l); coherent sources share a waveform; noise sigma per
    component; rounded half-to-even and clipped to int4."""
    pos, freq, kw = geometry(A)
    rng = np.random.default_rng(seed)
    g = (rng.normal(size=(T, F)) + 1j * rng.normal(size=(T, F))) / math.sqrt(2)
    x = (rng.normal(size=(T, F, A)) + 1j * rng.normal(size=(T, F, A))) * sigma
    for l, amp, phase in sources:
        st = np.exp(-1j * kw[:, None] * (pos[:, 0].astype(np.float64) * l)[None, :])
        x += amp * np.exp(1j * phase) * g[:, :, None] * st[None]
    if multipath is not None:
        l, amp, rho = multipath
        g3 = (rng.normal(size=(T, F)) + 1j * rng.normal(size=(T, F))) / math.sqrt(2)
        gm = rho * g + math.sqrt(1 - rho * rho) * g3
        st = np.exp(-1j * kw[:, None] * (pos[:, 0].astype(np.float64) * l)[None, :])
        x += amp * gm[:, :, None] * st[None]
    xr = np.clip(np.rint(x.real), -8, 7).astype(np.int64)
    xi = np.clip(np.rint(x.imag), -8, 7).astype(np.int64)
    return ((xr & 15) | ((xi & 15) << 4)).astype(np.uint8)


def test_oracle_doa_agrees_with_reference_search(ref):
    """One source: the FP64 1-D scan and the reference's 2-D coarse-to-fine
    Bartlett search (src/cpu_opt_beam_tracker.cpp:1619-2454) recover the
    same direction."""
    pos, freq, kw = geometry()
    K, B, l_true = 256, 2, 0.23
    v = source_voltage(K * B, 64, [(l_true, 2.0 * math.sqrt(2), 0.0)], seed=1)
    R = ref.covariance_blocks(v, K)
    _, cap, lest = ref.doa_scan(R, K, 8, 0.9, 1e-3, pos[:8], kw, -0.9, 0.001, 1801)
    dirs = ref.ref_doa_directions(v, pos, freq, K, capon=False, G=16, levels=2, fov_l=0.2, fov_m=0.05,
                                  subarray=0, lam=0.9, l0=0.2, m0=0.0)
    for w in range(B):
        assert abs(lest[w, 0] - l_true) < 0.01 and abs(lest[w, 1] - l_true) < 0.01
        assert abs(float(dirs[w, 0]) - l_true) < 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("A,K,B", [(64, 256, 3), (32, 128, 2), (64, 4096, 1)])
def test_covariance_bit_exact(cuda, orc, A, K, B):
    from beamform_project_b200 import api, native
    torch = cuda
    T = K * B
    v = random_voltage(T, F, A, seed=A + K)
    out = torch.full((B * F * A * A * 2,), 12345, dtype=torch.int32, device="cuda")
    api.doa_covariance_i32(None, torch.from_numpy(v).cuda(), out, api.Dimensions(T, F, A, 1), K)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    got = out.cpu().numpy().reshape(B, F, A, A, 2).astype(np.int64)
    exp = orc.covariance_blocks(v, K)
    assert np.array_equal(got, exp)


@pytest.mark.gpu
@pytest.mark.parametrize("fill", [0x88, 0x77, 0x78])
def test_covariance_extreme_components(cuda, orc, fill):
    """Constant -8 / +7 components (the largest block sums) and mixed signs."""
    from beamform_project_b200 import api, native
    torch = cuda
    A, K, B = 64, 128, 2
    v = np.full((K * B, F, A), fill, np.uint8)
    out = torch.full((B * F * A * A * 2,), 12345, dtype=torch.int32, device="cuda")
    api.doa_covariance_i32(None, torch.from_numpy(v).cuda(), out, api.Dimensions(K * B, F, A, 1), K)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    got = out.cpu().numpy().reshape(B, F, A, A, 2).astype(np.int64)
    assert np.array_equal(got, orc.covariance_blocks(v, K))


@pytest.mark.gpu
@pytest.mark.parametrize("A", [32, 64])
def test_covariance_long_block_is_sum_of_tiles(cuda, orc, A):
    """A block of 520 tiles (past the kernel's 512-tile flush of its component
    sums) of one repeated 128-spectrum tile is 520 times that tile's sums."""
    from beamform_project_b200 import api, native
    torch = cuda
    reps, K1 = 520, 128
    tile = random_voltage(K1, F, A, seed=11)
    out = torch.full((F * A * A * 2,), 12345, dtype=torch.int32, device="cuda")
    v = torch.from_numpy(tile).cuda().repeat(reps, 1, 1).contiguous()
    api.doa_covariance_i32(None, v, out, api.Dimensions(K1 * reps, F, A, 1), K1 * reps)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    got = out.cpu().numpy().reshape(F, A, A, 2).astype(np.int64)
    assert np.array_equal(got, reps * orc.covariance_blocks(tile, K1)[0])


@pytest.mark.gpu
def test_scan_matches_fp64_oracle_and_finds_sources(cuda, orc):
    from beamform_project_b200 import api, native
    torch = cuda
    A, K, B, M, n = 64, 512, 4, 8, 1801
    pos, freq, kw = geometry(A)
    amp = 2.0 * math.sqrt(2.0)
    v = source_voltage(K * B, A, [(-0.14, amp, 0.0), (0.14, amp, 1.1)], seed=3, multipath=(0.5, amp, 0.5))
    d = api.Dimensions(K * B, F, A, 1)
    cov = torch.empty(B * F * A * A * 2, dtype=torch.int32, device="cuda")
    api.doa_covariance_i32(None, torch.from_numpy(v).cuda(), cov, d, K)
    bart = torch.empty(B * n, dtype=torch.float64, device="cuda")
    cap = torch.empty(B * n, dtype=torch.float64, device="cuda")
    lest = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    ws = torch.empty(api.doa_workspace_bytes(d, K, M), dtype=torch.uint8, device="cuda")
    api.doa_scan(None, cov, torch.from_numpy(pos[:M]).cuda(), torch.from_numpy(kw).cuda(), d, K, M, 0.9, 1e-3,
                 -0.9, 0.001, n, 0.0, bart, cap, lest, ws)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    R = cov.cpu().numpy().reshape(B, F, A, A, 2).astype(np.int64)
    assert np.array_equal(R, orc.covariance_blocks(v, K))
    eb, ec, el = orc.doa_scan(R, K, M, 0.9, 1e-3, pos[:M], kw, -0.9, 0.001, n)
    gb = bart.cpu().numpy().reshape(B, n)
    gc = cap.cpu().numpy().reshape(B, n)
    assert np.allclose(gb, eb, rtol=1e-6, atol=0.0)
    assert np.allclose(gc, ec, rtol=1e-6, atol=0.0)
    assert np.allclose(lest.cpu().numpy().reshape(B, 2), el, atol=1e-6)
    # Capon's two largest local maxima: the coherent pair (0.7 beamwidth apart,
    # which smoothing along the element index of a 2 x 32 grid does not split)
    # between the two sources, and the multipath arrival at 0.5
    P = gc[-1]
    peaks = [i for i in range(1, n - 1) if P[i] > P[i - 1] and P[i] >= P[i + 1]]
    top = sorted(-0.9 + 0.001 * i for i in sorted(peaks, key=lambda i: -P[i])[:2])
    assert -0.14 < top[0] < 0.14 and abs(top[1] - 0.5) < 0.03, top


@pytest.mark.gpu
@pytest.mark.parametrize("M,jitter", [(3, 0.0), (13, 0.0), (14, 0.0), (16, 0.0), (8, 1e-3), (16, 1e-3), (2, 0.0)])
def test_scan_element_counts_match_fp64_oracle(cuda, orc, M, jitter):
    """Sub-array sizes across the scan's shared-memory layouts (four blocks
    per CTA up to 13 elements, two above) agree with the FP64 oracle, in the
    uniform sub-array form (a line of float positions) and, with the
    positions jittered by about a millimetre, in the general form."""
    from beamform_project_b200 import api, native
    torch = cuda
    A, K, B, n = 64, 128, 3, 301
    pos, freq, kw = geometry(A)
    if jitter:
        pos = pos.copy()
        pos[:M, :2] += (rng(M).standard_normal((M, 2)) * jitter).astype(np.float32)
    amp = 2.0 * math.sqrt(2.0)
    v = source_voltage(K * B, A, [(0.2, amp, 0.0)], seed=M)
    d = api.Dimensions(K * B, F, A, 1)
    cov = torch.empty(B * F * A * A * 2, dtype=torch.int32, device="cuda")
    api.doa_covariance_i32(None, torch.from_numpy(v).cuda(), cov, d, K)
    bart = torch.empty(B * n, dtype=torch.float64, device="cuda")
    cap = torch.empty(B * n, dtype=torch.float64, device="cuda")
    lest = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    ws = torch.empty(api.doa_workspace_bytes(d, K, M), dtype=torch.uint8, device="cuda")
    api.doa_scan(None, cov, torch.from_numpy(pos[:M]).cuda(), torch.from_numpy(kw).cuda(), d, K, M, 0.9, 1e-3,
                 -0.6, 0.004, n, 0.0, bart, cap, lest, ws)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    R = cov.cpu().numpy().reshape(B, F, A, A, 2).astype(np.int64)
    eb, ec, el = orc.doa_scan(R, K, M, 0.9, 1e-3, pos[:M], kw, -0.6, 0.004, n)
    assert np.allclose(bart.cpu().numpy().reshape(B, n), eb, rtol=1e-6, atol=0.0)
    assert np.allclose(cap.cpu().numpy().reshape(B, n), ec, rtol=1e-6, atol=0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("B,M,Fs", [(64, 8, 160), (65, 8, 160), (16, 8, 16), (64, 11, 160), (32, 16, 160),
                                    (33, 16, 160), (9, 12, 160), (1, 5, 16)])
def test_fold_schedules_match_fp64_oracle(cuda, orc, B, M, Fs):
    """The fold's two schedules on a channel slice against the FP64 oracle:
    one launch per channel over chunks of cells (at least as many channels
    as SMs; up to 64 blocks at 11 elements or fewer, 32 above; the
    forgetting recursion carried from chunk to chunk) and three launches
    for longer block sequences or fewer channels."""
    from beamform_project_b200 import api, native
    torch = cuda
    A, K, n, lam, load = 32, 128, 101, 0.9, 1e-3
    pos, freq, kw = geometry(A)
    kws = np.ascontiguousarray(kw[:Fs])
    v = rng(100 * B + M).integers(0, 256, size=(K * B, Fs, A), dtype=np.uint8)
    d = api.Dimensions(K * B, Fs, A, 1)
    cov = torch.empty(B * Fs * A * A * 2, dtype=torch.int32, device="cuda")
    api.doa_covariance_i32_slice(None, torch.from_numpy(v).cuda(), cov, d, K)
    bart = torch.empty(B * n, dtype=torch.float64, device="cuda")
    cap = torch.empty(B * n, dtype=torch.float64, device="cuda")
    lest = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    ws = torch.empty(api.doa_workspace_bytes(d, K, M), dtype=torch.uint8, device="cuda")
    api.doa_scan_slice(None, cov, torch.from_numpy(pos[:M]).cuda(), torch.from_numpy(kws).cuda(), d, K, M, lam,
                       load, -0.6, 0.012, n, 0.0, bart, cap, lest, ws)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    R = cov.cpu().numpy().reshape(B, Fs, A, A, 2).astype(np.int64)
    eb, ec, _ = orc.doa_scan(R, K, M, lam, load, pos[:M], kws, -0.6, 0.012, n)
    assert np.allclose(bart.cpu().numpy().reshape(B, n), eb, rtol=1e-6, atol=0.0)
    assert np.allclose(cap.cpu().numpy().reshape(B, n), ec, rtol=1e-6, atol=0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("A,capon,subarray,G,levels", [(32, False, 16, 16, 2), (64, False, 8, 12, 1),
                                                       (32, True, 8, 16, 2), (64, True, 8, 8, 0)])
def test_adaptive_tracker_follows_reference_search(cuda, ref, orc, A, capon, subarray, G, levels):
    """bf_doa_track against CpuOptBeamTracker::run_into on a drifting source:
    each window's direction within two final half-pitches of the reference's
    (the search compares FP64 powers where the reference compares FP32 ones,
    so a near-tie can pick the neighbouring candidate) and almost always
    within 1e-4; the emitted beam power equals the reference float32 chain
    along the GPU's own directions bit for bit, and the reference's emission
    wherever the directions agree to the last bit."""
    from beamform_project_b200 import api, native
    torch = cuda
    F, K, W = 336, 256, 8
    T = K * W
    pos = ref.ref_default_positions(A)
    freq = ref.ref_channelized_frequencies(F)
    l0, m0 = 0.06, -0.03
    v = ref.ref_make_moving_point_source(T, F, A, pos, freq, l0, m0, 1e-5, 5e-6, 3.0)
    fov = 0.15
    lam = 0.9
    ref_dirs, ref_I = ref.ref_doa_directions(v, pos, freq, K, capon=capon, G=G, levels=levels, fov_l=fov,
                                             fov_m=fov, subarray=subarray, lam=lam, load=1e-3, l0=0.0, m0=0.0,
                                             intensity=True)
    d = api.Dimensions(T, F, A, 1)
    cfg = api.doa_track_config(K, subarray=subarray, capon=capon, grid=G, levels=levels, fov_l=fov, fov_m=fov,
                               forgetting=lam, diag_load=1e-3)
    ws = torch.empty(api.doa_track_workspace_bytes(d, cfg), dtype=torch.uint8, device="cuda")
    dirs = torch.zeros(W * 3, dtype=torch.float32, device="cuda")
    inten = torch.zeros(T * F, dtype=torch.float32, device="cuda")
    api.doa_track(None, torch.from_numpy(v).cuda(), torch.from_numpy(pos).cuda(),
                  torch.from_numpy(api.wave_numbers(freq)).cuda(), d, cfg, dirs, inten, ws)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    got = dirs.cpu().numpy().reshape(W, 3)
    half = fov / G / (2 ** levels) if levels else 2 * fov / (G - 1)
    dl = np.abs(got[:, :2] - ref_dirs[:, :2])
    print(f"A={A} capon={capon} M={subarray} G={G} L={levels}: max |dir - reference| {dl.max():.2e} "
          f"(half-pitch {half:.2e}); median {np.median(dl):.2e}")
    assert dl.max() <= 2 * half
    assert np.median(dl) <= 1e-4
    got_I = inten.cpu().numpy().reshape(T, F)
    mine = orc.tracker(v, orc.tracker_weights(got, pos, freq), T, F, A, K)
    assert np.array_equal(got_I, mine)
    same = np.all(got == ref_dirs, axis=1)
    for w in np.nonzero(same)[0]:
        assert np.array_equal(got_I[w * K:(w + 1) * K], ref_I[w * K:(w + 1) * K])
