"""GPU parity: the tracker (reference beam_tracker.cpp:90-146).

mode 0 follows the reference float32 order; its only freedom is the last bit
of the FP64 sin/cos of the phase, so it must match the oracle to 1e-6
relative (and almost everywhere exactly).  mode 1 (tensor-pipe streaming
kernel, fp16 hi+lo weights, fp32 sums) must match within the reference's
CUDA tolerance |gpu - cpu| <= 1e-3 + 1e-5 |cpu| (tests/cuda/
test_cuda_packed.cu:24-25), and its per-window sums within 1e-5 relative of
the FP64 sum.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import random_voltage

pytestmark = pytest.mark.gpu
F = 336


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _run(torch, api, mode, v, pos, freq, dirs, T, A, S, want_int=True, want_integ=True):
    W = len(dirs)
    inten = torch.full((T * F,), -1.0, dtype=torch.float32, device="cuda") if want_int else None
    integ = torch.full((W * F,), -1.0, dtype=torch.float32, device="cuda") if want_integ else None
    api.tracker(None, mode, _dev(torch, v), _dev(torch, pos), _dev(torch, api.wave_numbers(freq)),
                _dev(torch, dirs), inten, integ, api.Dimensions(T, F, A, 1), S)
    torch.cuda.synchronize()
    return (None if inten is None else inten.cpu().numpy().reshape(T, F),
            None if integ is None else integ.cpu().numpy().reshape(W, F))


def _case(orc, api, T, A, S, seed, moving=True):
    pos, freq = api.default_positions(A), api.channelized_frequencies(F)
    l0, m0, rl, rm = (0.05, -0.03, 3e-5, -2e-5) if moving else (0.1, 0.0, 0.0, 0.0)
    dirs = api.tracker_window_directions(l0, m0, rl, rm, T, S)
    v = random_voltage(T, F, A, seed)
    ww = orc.tracker_weights(dirs, pos, freq)
    return pos, freq, dirs, v, orc.tracker(v, ww, T, F, A, S)


@pytest.mark.parametrize("A,T,S", [(32, 100, 16), (64, 257, 64), (128, 40, 10), (256, 33, 32)])
def test_mode0_reference_order(cuda, orc, A, T, S):
    from beamform_project_b200 import api
    pos, freq, dirs, v, ref = _case(orc, api, T, A, S, seed=A)
    inten, integ = _run(cuda, api, 0, v, pos, freq, dirs, T, A, S)
    assert np.allclose(inten, ref, rtol=1e-6, atol=1e-6)
    assert np.mean(inten == ref) > 0.99
    # per-window sums in increasing time (src/temporal_integration.cpp:95-109)
    exp = orc.integrate(ref[..., None], T, F, 1, S)[..., 0]
    assert np.allclose(integ, exp, rtol=1e-6, atol=1e-5)


@pytest.mark.parametrize("A,T,S", [(32, 100, 16), (64, 1024, 256), (64, 300, 320),
                                   (128, 50, 10), (256, 48, 32)])
def test_mode1_streaming_within_tolerance(cuda, orc, A, T, S):
    from beamform_project_b200 import api
    pos, freq, dirs, v, ref = _case(orc, api, T, A, S, seed=T)
    inten, integ = _run(cuda, api, 1, v, pos, freq, dirs, T, A, S)
    err = np.abs(inten.astype(np.float64) - ref)
    assert np.all(err <= 1e-3 + 1e-5 * np.abs(ref)), float(np.max(err - 1e-5 * np.abs(ref)))
    exp64 = orc.integrate(ref[..., None], T, F, 1, S)[..., 0].astype(np.float64)
    assert np.all(np.abs(integ - exp64) <= 1e-3 + 1e-5 * np.abs(exp64))


def test_mode1_integrated_only_and_point_source(cuda, orc, ref):
    """A source moving along the tracked trajectory stays in the beam: the
    tracked power is the coherent maximum and equals the oracle."""
    from beamform_project_b200 import api
    T, A, S = 128, 64, 32
    pos, freq = api.default_positions(A), api.channelized_frequencies(F)
    l0, m0, rl, rm = 0.02, 0.01, 1e-4, 0.0
    v = ref.ref_make_moving_point_source(T, F, A, pos, freq, l0, m0, rl, rm, 4.0)
    dirs = api.tracker_window_directions(l0, m0, rl, rm, T, S)
    exp = orc.tracker(v, orc.tracker_weights(dirs, pos, freq), T, F, A, S)
    _, integ = _run(cuda, api, 1, v, pos, freq, dirs, T, A, S, want_int=False)
    exp_w = exp.reshape(T // S, S, F).astype(np.float64).sum(axis=1)
    assert np.allclose(integ, exp_w, rtol=1e-5, atol=1e-3)
    # the tracked beam collects (close to) the full coherent power A^2 * 16
    assert float(np.median(exp)) > 0.5 * A * A * 16
