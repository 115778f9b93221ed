"""GPU parity on the benchmark workloads themselves (not random phases).

* The plain grid workload in full: a 32-element line array at half a
  wavelength of 600 MHz, 336 channels over 400-600 MHz, T = 1024, 16 beams at
  l = -0.5 + b/15, Gaussian sigma = 2, S = 10.  The reference-order kernel is
  bit-identical to the reference CPU core (src/cpu_beamformer.cpp:56-78,
  src/temporal_integration.cpp:79-110); the split-precision tensor path is
  within 1e-5 relative (1e-3 absolute floor) of the reference float32 output
  on its own, and of the FP64 sum.
* The full-band split-precision workload (2 x 32 grid, 2 shards x 336
  channels over 400-800 MHz, T = 32768, 128 beams on a 16 x 8 grid, a point
  source at SNR 5, S = 320, int8 chunk codes) run in full on the GPU and
  checked on windows {0, 1, 51, 102 (partial, 128 spectra)} of both shards:
  float32 within the same bar of the reference float32 chain and of FP64;
  int8 codes identical to the reference quantizer (src/quantization.cpp:61-161)
  applied to the kernel's own integrated values, and at most 1 LSB from the
  codes of the reference float32 chain, for at most 1e-4 of the codes (the
  count is printed; reference tests/cuda/test_cuda_quantization.cpp:26-45).
* The reference's own CUDA kernels (built for sm_100a from its sources) on
  the same inputs: its Tiled kernel within the reference CUDA tests'
  tolerance (tests/cuda/test_cuda_packed.cu:24-25) of the reference-order
  kernel, and its int8 quantizer within the reference CUDA test's bar of the
  B200 quantizer (which follows the reference CPU quantizer bit for bit).
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu
F = 336


def _bar(got, ref):
    """max of |got - ref| / (1e-3 + 1e-5 |ref|): at most 1 passes."""
    g = np.asarray(got, np.float64)
    r = np.asarray(ref, np.float64)
    return float(np.max(np.abs(g - r) / (1e-3 + 1e-5 * np.abs(r))))


@pytest.fixture(scope="module")
def c1(cuda):
    from beamform_project_b200 import api, native
    torch = cuda
    d, volt, w = bench.c1_inputs(torch.device("cuda"))
    w_host = w.cpu().numpy().reshape(bench.C1_B, F, bench.C1_A, 2)
    split = torch.empty(api.split_weight_bytes(d), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, w, split, d)
    W = api.integrated_time_count(bench.C1_T, bench.C1_S)
    out_t = torch.empty(W * F * bench.C1_B, dtype=torch.float32, device="cuda")
    out_x = torch.empty_like(out_t)
    wt = torch.from_numpy(bench.tiled_weights(w_host)).cuda()
    api.grid_tensor_integrated(None, volt, split, out_t, None, None, d, bench.C1_S)
    api.launch_packed_integrated_beamformer(api.CudaBeamformerKernel.Tiled, None, volt, wt, out_x, d, bench.C1_S)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    v = volt.cpu().numpy().reshape(bench.C1_T, F, bench.C1_A)
    shape = (W, F, bench.C1_B)
    return dict(v=v, w=w_host, wt=wt, volt=volt, tensor=out_t.cpu().numpy().reshape(shape),
                exact=out_x.cpu().numpy().reshape(shape))


def test_plain_grid_workload_exact_kernel_is_the_reference(c1, ref):
    T, A, B, S = bench.C1_T, bench.C1_A, bench.C1_B, bench.C1_S
    ref32 = ref.ref_integrate(ref.ref_beamform(c1["v"], c1["w"], T, F, A, B), T, F, A, B, S)
    assert np.array_equal(c1["exact"], ref32)


def test_plain_grid_workload_tensor_path_within_1e5_of_reference_fp32(c1, ref, orc):
    T, A, B, S = bench.C1_T, bench.C1_A, bench.C1_B, bench.C1_S
    ref32 = ref.ref_integrate(ref.ref_beamform(c1["v"], c1["w"], T, F, A, B), T, F, A, B, S)
    ref64 = orc.beamform_integrated(c1["v"], c1["w"], T, F, A, B, S, f64=True)
    b32, b64 = _bar(c1["tensor"], ref32), _bar(c1["tensor"], ref64)
    rel = float(np.max(np.abs(c1["tensor"] - ref32.astype(np.float64)) / np.abs(ref32)))
    print(f"plain grid workload: tensor vs reference fp32 {b32:.3f} of the bar (max rel {rel:.2e}), "
          f"vs FP64 {b64:.3f} of the bar")
    assert b32 <= 1.0
    assert b64 <= 1.0


def test_plain_grid_workload_reference_cuda_kernel(c1, cuda, orc):
    if not orc.reference_gpu_available():
        pytest.skip("reference CUDA kernels (oracle/_ref/libbfref_cuda.so) not built")
    torch = cuda
    g = orc.reference_gpu()
    T, A, B, S = bench.C1_T, bench.C1_A, bench.C1_B, bench.C1_S
    out = torch.empty(c1["exact"].size, dtype=torch.float32, device="cuda")
    orc.refgpu_check(g.refgpu_grid_integrated(1, torch.cuda.current_stream().cuda_stream, c1["volt"].data_ptr(),
                                              c1["wt"].data_ptr(), out.data_ptr(), T, F, A, B, S))
    torch.cuda.synchronize()
    assert _bar(out.cpu().numpy().reshape(c1["exact"].shape), c1["exact"]) <= 1.0


WINDOWS = (0, 1, 51, 102)


@pytest.fixture(scope="module")
def c2(cuda):
    """The full-band workload on the GPU: integrated values and codes of both
    shards, and the host voltages of the sampled windows."""
    from beamform_project_b200 import api, native
    torch = cuda
    T, A, B, S, NS = bench.T_SPECTRA, bench.N_ANT, bench.N_BEAMS, bench.S_INT, bench.N_SHARDS
    pos, freq, dirs = bench.workload_geometry()
    w_host = bench.workload_weights(pos, freq, dirs)
    _, mu = bench.workload_source(pos, freq, dirs)
    d = api.Dimensions(T, F, A, B)
    shard_bytes = T * F * A
    volt = torch.empty(NS * shard_bytes, dtype=torch.uint8, device="cuda")
    for s in range(NS):
        api.generate_voltage(None, bench.SEED, s * shard_bytes, bench.SIGMA, torch.from_numpy(mu[s]).cuda(), T,
                             volt[s * shard_bytes:(s + 1) * shard_bytes], d)
    wd = torch.from_numpy(w_host).cuda()
    split = torch.empty(api.split_weight_bytes(d, NS), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, wd, split, d, NS)
    W = api.integrated_time_count(T, S)
    n_out = NS * W * F * B
    integ = torch.empty(n_out, dtype=torch.float32, device="cuda")
    codes = torch.empty(n_out, dtype=torch.int8, device="cuda")
    qd = api.Dimensions(W, F, A, B)
    params = torch.empty(NS * 2 * api.quantization_parameter_count(qd), dtype=torch.float32, device="cuda")
    api.grid_tensor_integrated(None, volt, split, integ, codes, params, d, S, NS)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    vh = volt.view(NS, T, F, A)
    wins = {}
    for s in range(NS):
        for w in WINDOWS:
            a, b = w * S, min((w + 1) * S, T)
            wins[(s, w)] = np.ascontiguousarray(vh[s, a:b].cpu().numpy())
    yield dict(w=w_host, wins=wins, integ=integ.cpu().numpy().reshape(NS, W, F, B),
               codes=codes.cpu().numpy().reshape(NS, W, F, B), volt=volt, weights=wd, integ_dev=integ,
               codes_dev=codes, W=W)
    del volt, split, integ, codes, params
    torch.cuda.empty_cache()


def _per_window(fn, keys):
    with ThreadPoolExecutor(max_workers=8) as ex:
        return dict(zip(keys, ex.map(fn, keys)))


def test_full_band_workload_sampled_windows(c2, ref, orc):
    A, B, S = bench.N_ANT, bench.N_BEAMS, bench.S_INT
    keys = sorted(c2["wins"])

    def ref32(key):
        v = c2["wins"][key]
        Tw = len(v)
        return ref.ref_integrate(ref.ref_beamform(v, c2["w"][key[0]], Tw, F, A, B), Tw, F, A, B, S)[0]

    def ref64(key):
        v = c2["wins"][key]
        return orc.beamform_integrated(v, c2["w"][key[0]], len(v), F, A, B, S, f64=True)[0]

    r32 = _per_window(ref32, keys)
    r64 = _per_window(ref64, keys)
    assert len(c2["wins"][(0, 102)]) == 128  # the partial last window
    worst32 = worst64 = 0.0
    lsb_count = total = 0
    for key in keys:
        s, w = key
        got = c2["integ"][s, w]
        worst32 = max(worst32, _bar(got, r32[key]))
        worst64 = max(worst64, _bar(got, r64[key]))
        # codes: identical to the reference quantizer on the kernel's own values,
        # at most 1 LSB from the codes of the reference float32 chain
        own, _ = ref.ref_quantize(got[None], 1, F, A, B)
        assert np.array_equal(c2["codes"][s, w], own[0]), key
        chain, _ = ref.ref_quantize(r32[key][None], 1, F, A, B)
        diff = np.abs(c2["codes"][s, w].astype(np.int32) - chain[0].astype(np.int32))
        assert diff.max() <= 1, key
        lsb_count += int((diff > 0).sum())
        total += diff.size
    print(f"full-band workload, windows {WINDOWS} x 2 shards: vs reference fp32 {worst32:.3f} of the bar, "
          f"vs FP64 {worst64:.3f}; int8 codes 1 LSB from the reference chain: {lsb_count} of {total}")
    assert worst32 <= 1.0
    assert worst64 <= 1.0
    assert lsb_count <= 1e-4 * total


def test_full_band_workload_reference_cuda_quantizer(c2, cuda, orc):
    """The reference's int8 chunk quantizer (src/cuda_quantize_int8.cu:30-147,
    nvcc sm_100a) on the B200 path's integrated output.  The B200 quantizer
    reproduces the reference CPU quantizer bit for bit; the reference's own
    GPU kernel does not quite (nvcc contracts offset = min - (-127.5) * scale
    into one fused multiply-add), so against it the bar is the reference
    CUDA test's (tests/cuda/test_cuda_quantization.cpp:26-45): parameters
    within 1e-3 + 1e-6 |offset| and 1e-5 + 1e-6 |scale|, and codes at most
    1 LSB apart (the reference test wants them equal on its small cases;
    the count here is printed)."""
    if not orc.reference_gpu_available():
        pytest.skip("reference CUDA kernels (oracle/_ref/libbfref_cuda.so) not built")
    from beamform_project_b200 import api
    torch = cuda
    NS, W, B, A = bench.N_SHARDS, c2["W"], bench.N_BEAMS, bench.N_ANT
    qd = api.Dimensions(NS * W, F, A, B)
    n_par = 2 * api.quantization_parameter_count(qd)
    codes_b = torch.empty_like(c2["codes_dev"])
    params_b = torch.empty(n_par, dtype=torch.float32, device="cuda")
    api.launch_quantize_integrated_intensity(None, c2["integ_dev"], codes_b, params_b, qd)
    codes_r = torch.empty_like(codes_b)
    params_r = torch.empty_like(params_b)
    g = orc.reference_gpu()
    orc.refgpu_check(g.refgpu_quantize(torch.cuda.current_stream().cuda_stream, c2["integ_dev"].data_ptr(),
                                       codes_r.data_ptr(), params_r.data_ptr(), NS * W, F, A, B))
    torch.cuda.synchronize()
    diff = (codes_b.int() - codes_r.int()).abs()
    print(f"reference CUDA quantizer: {int((diff > 0).sum())} of {diff.numel()} codes 1 LSB apart")
    assert int(diff.max()) <= 1
    assert int((diff > 0).sum()) <= 1e-4 * diff.numel()
    pb, pr = params_b.view(-1, 2).double(), params_r.view(-1, 2).double()
    assert bool(((pb[:, 0] - pr[:, 0]).abs() <= 1e-3 + 1e-6 * pr[:, 0].abs()).all())
    assert bool(((pb[:, 1] - pr[:, 1]).abs() <= 1e-5 + 1e-6 * pr[:, 1].abs()).all())
