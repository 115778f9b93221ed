"""Loss-mask consumption (bf_apply_loss_mask): lost frames of the packed
voltage become zero in place, every other byte is untouched, and the valid
frames are counted per integration window and channel (numpy restatement)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import random_voltage, rng

F = 336


@pytest.mark.gpu
@pytest.mark.parametrize("T,A,S", [(1000, 64, 320), (37, 32, 10), (640, 128, 1)])
def test_lost_frames_zeroed_and_counted(cuda, T, A, S):
    from beamform_project_b200 import api
    torch = cuda
    v = random_voltage(T, F, A, seed=T + A)
    mask = (rng(S).random((T, F)) > 0.1).astype(np.uint8)
    mask[:, 5] = 0                       # a channel lost throughout
    mask[: min(T, S), 7] = 0             # a whole first window lost on one channel
    mask[3, :] = 2                       # nonzero bytes other than 1 count as valid
    dv = torch.from_numpy(v).cuda()
    W = -(-T // S)
    counts = torch.full((W * F,), 0xDEAD, dtype=torch.uint32, device="cuda")
    api.apply_loss_mask(None, dv, torch.from_numpy(mask).cuda(), api.Dimensions(T, F, A, 1), S, counts)
    torch.cuda.synchronize()
    exp = v.copy()
    exp[mask == 0] = 0
    assert np.array_equal(dv.cpu().numpy(), exp)
    valid = (mask != 0).astype(np.int64)
    pad = np.zeros((W * S - T, F), np.int64)
    exp_counts = np.concatenate([valid, pad]).reshape(W, S, F).sum(1)
    assert np.array_equal(counts.cpu().numpy().astype(np.int64).reshape(W, F), exp_counts)


@pytest.mark.gpu
def test_without_counts_and_argument_checks(cuda):
    from beamform_project_b200 import api, native
    torch = cuda
    T, A = 64, 32
    v = random_voltage(T, F, A, seed=3)
    mask = np.ones((T, F), np.uint8)
    mask[10, 100] = 0
    dv = torch.from_numpy(v).cuda()
    api.apply_loss_mask(None, dv, torch.from_numpy(mask).cuda(), api.Dimensions(T, F, A, 1), 320)
    torch.cuda.synchronize()
    got = dv.cpu().numpy()
    assert not got[10, 100].any() and np.array_equal(np.delete(got.reshape(-1, A), 10 * F + 100, 0),
                                                      np.delete(v.reshape(-1, A), 10 * F + 100, 0))
    with pytest.raises(native.InvalidArgument):
        api.apply_loss_mask(None, dv, torch.from_numpy(mask).cuda(), api.Dimensions(T, F, A, 1), 0)
