"""Channel-split DOA across GPUs: the one exchange step of the path.

A DOA job's Bartlett and Capon spectra are sums over its frequency channels
(CpuOptBeamTracker splits the channels over its threads, each adding its
channels' powers into a private slab, then sums the slabs,
src/cpu_opt_beam_tracker.cpp:2046-2108), and everything before the sum --
the covariance, smoothing, forgetting and Cholesky of each channel -- is
independent per channel.  So N GPUs can each take a contiguous slice of the
channels (covariance, fold and scan on the slice: bf_doa_covariance_i32_slice,
bf_doa_scan_slice), one all-reduce of the partial spectra
(2 x blocks x points doubles) gives the job's spectra, and the peak search
(bf_doa_peak) runs on the sum.  One process per GPU under torchrun; the
default process group carries the all-reduce (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

from . import api
from .replicas import Replicas


def channel_slice(n_freq: int, rank: int, world: int) -> range:
    """Contiguous, balanced slice of the channels for `rank`: whole channel
    pairs (the covariance kernel reads channels in pairs), sizes differing by
    at most one pair."""
    pairs = Replicas.partition(n_freq // 2, rank, world)
    return range(2 * pairs.start, 2 * pairs.stop)


def reduce_spectra(spectra) -> None:
    """Sum a tensor of partial spectra over the ranks of the default process
    group, in place (no-op without one)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(spectra, op=dist.ReduceOp.SUM)


def scan_slice(volt_slice, positions, wave_numbers_slice, n_time: int, n_ant: int, block_len: int,
               subarray: int, forgetting: float, diag_load: float, l_first: float, l_step: float,
               n_points: int, m_fixed: float, reduce: bool = True):
    """Covariance, fold and scan of one channel slice ([T][slice][A] packed
    voltage on the current CUDA device, its wave numbers), the all-reduce of
    the partial spectra over the process group, and the peak search.
    Returns (spectra [2][blocks][n_points] double: Bartlett, Capon; l_est
    [blocks][2] double) as device tensors."""
    import torch
    n_slice = wave_numbers_slice.numel()
    d = api.Dimensions(n_time, n_slice, n_ant, 1)
    n_blocks = n_time // block_len
    dev = volt_slice.device
    cov = torch.empty(n_blocks * n_slice * n_ant * n_ant * 2, dtype=torch.int32, device=dev)
    ws = torch.empty(api.doa_workspace_bytes(d, block_len, subarray), dtype=torch.uint8, device=dev)
    spectra = torch.empty(2, n_blocks, n_points, dtype=torch.float64, device=dev)
    l_est = torch.empty(n_blocks, 2, dtype=torch.float64, device=dev)
    api.doa_covariance_i32_slice(None, volt_slice, cov, d, block_len)
    api.doa_scan_slice(None, cov, positions, wave_numbers_slice, d, block_len, subarray, forgetting, diag_load,
                       l_first, l_step, n_points, m_fixed, spectra[0], spectra[1], l_est, ws)
    if reduce:
        reduce_spectra(spectra)
    api.doa_peak(None, spectra[0], spectra[1], n_blocks, n_points, l_first, l_step, l_est)
    return spectra, l_est
