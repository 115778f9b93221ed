"""Channel-split DOA (beamform_project_b200.doa_channels): the path's one
exchange step.

CPU: the channel partition, and two gloo ranks that each scan their channel
slice with the FP64 oracle, sum the partial spectra with the module's
all-reduce and find the peaks: equal to one process scanning every channel
(the spectra up to the order of the sum over channels).
GPU: the slice entries (bf_doa_covariance_i32_slice, bf_doa_scan_slice) on
two and three slices of one job, summed on the device, then bf_doa_peak:
equal to bf_doa_scan over all channels.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from beamform_project_b200.doa_channels import channel_slice

F, A, K, B, M, N_PTS = 336, 64, 256, 3, 8, 301
L_FIRST, L_STEP, LAM, LOAD = -0.6, 0.004, 0.9, 1e-3


def _inputs(orc):
    rng = np.random.default_rng(7)
    v = rng.integers(0, 256, size=(K * B, F, A), dtype=np.uint8)
    R = orc.covariance_blocks(v, K)
    pos = np.zeros((A, 3), np.float32)
    pos[:, 0] = (np.arange(A) * 0.19).astype(np.float32)
    kw = (2 * np.pi * (400e6 + np.arange(F) * 1e6) / 299792458.0).astype(np.float64)
    return v, R, pos, kw


def _peaks(P: np.ndarray) -> np.ndarray:
    """argmax and the vertex of the parabola through it and its neighbours
    (concave case, offset clamped to half a step), per block."""
    out = np.zeros(P.shape[0])
    for b, row in enumerate(P):
        i = int(np.argmax(row))
        delta = 0.0
        if 0 < i < row.size - 1:
            den = row[i - 1] - 2 * row[i] + row[i + 1]
            if den < 0:
                delta = min(0.5, max(-0.5, 0.5 * (row[i - 1] - row[i + 1]) / den))
        out[b] = L_FIRST + (i + delta) * L_STEP
    return out


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7])
def test_channel_slices_cover_the_band_in_pairs(world):
    slices = [channel_slice(F, r, world) for r in range(world)]
    assert [f for s in slices for f in s] == list(range(F))
    assert all(s.start % 2 == 0 and len(s) % 2 == 0 for s in slices)
    assert max(len(s) for s in slices) - min(len(s) for s in slices) <= 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist

    from beamform_project_b200.doa_channels import reduce_spectra
    from oracle import loader as orc
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        _, R, pos, kw = _inputs(orc)
        sl = channel_slice(F, rank, world)
        bart, cap, _ = orc.doa_scan(R[:, sl.start:sl.stop], K, M, LAM, LOAD, pos[:M], kw[sl.start:sl.stop],
                                    L_FIRST, L_STEP, N_PTS)
        spectra = torch.from_numpy(np.stack([bart, cap]))
        reduce_spectra(spectra)
        out.put((rank, spectra.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_their_channel_slices(orc):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(world))
    _, R, pos, kw = _inputs(orc)
    bart, cap, lest = orc.doa_scan(R, K, M, LAM, LOAD, pos[:M], kw, L_FIRST, L_STEP, N_PTS)
    for r in range(world):
        assert np.allclose(res[r][0], bart, rtol=1e-12, atol=0.0)
        assert np.allclose(res[r][1], cap, rtol=1e-12, atol=0.0)
        assert np.allclose(_peaks(res[r][0]), lest[:, 0], rtol=0, atol=1e-9)
        assert np.allclose(_peaks(res[r][1]), lest[:, 1], rtol=0, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_slices_summed_on_the_device_equal_the_whole_scan(cuda, orc, world):
    from beamform_project_b200 import api, native
    from beamform_project_b200.doa_channels import scan_slice
    torch = cuda
    v, R, pos, kw = _inputs(orc)
    T = K * B
    d = api.Dimensions(T, F, A, 1)
    vd = torch.from_numpy(v).cuda()
    posd = torch.from_numpy(np.ascontiguousarray(pos[:M])).cuda()
    kwd = torch.from_numpy(kw).cuda()
    cov = torch.empty(B * F * A * A * 2, dtype=torch.int32, device="cuda")
    api.doa_covariance_i32(None, vd, cov, d, K)
    ws = torch.empty(api.doa_workspace_bytes(d, K, M), dtype=torch.uint8, device="cuda")
    bart = torch.empty(B * N_PTS, dtype=torch.float64, device="cuda")
    cap = torch.empty_like(bart)
    lest = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    api.doa_scan(None, cov, posd, kwd, d, K, M, LAM, LOAD, L_FIRST, L_STEP, N_PTS, 0.0, bart, cap, lest, ws)
    total = torch.zeros(2, B, N_PTS, dtype=torch.float64, device="cuda")
    for r in range(world):
        sl = channel_slice(F, r, world)
        vs = vd.view(T, F, A)[:, sl.start:sl.stop].contiguous()
        spectra, _ = scan_slice(vs, posd, kwd[sl.start:sl.stop].contiguous(), T, A, K, M, LAM, LOAD, L_FIRST,
                                L_STEP, N_PTS, 0.0, reduce=False)
        total += spectra
    le = torch.empty(B, 2, dtype=torch.float64, device="cuda")
    api.doa_peak(None, total[0], total[1], B, N_PTS, L_FIRST, L_STEP, le)
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    assert torch.allclose(total[0].reshape(-1), bart, rtol=1e-12, atol=0.0)
    assert torch.allclose(total[1].reshape(-1), cap, rtol=1e-12, atol=0.0)
    assert torch.allclose(le.reshape(-1), lest, rtol=0.0, atol=1e-9)
    # one slice holding every channel is the whole scan, bit for bit
    spectra, le1 = scan_slice(vd, posd, kwd, T, A, K, M, LAM, LOAD, L_FIRST, L_STEP, N_PTS, 0.0, reduce=False)
    torch.cuda.synchronize()
    assert torch.equal(spectra[0].reshape(-1), bart) and torch.equal(spectra[1].reshape(-1), cap)
    assert torch.equal(le1.reshape(-1), lest)
