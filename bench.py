#!/usr/bin/env python3
"""Benchmark of the fixed-grid beamformer hot path on B200.

Workload (the full-band split-precision grid): 64 antennas on a 2 x 32 grid
at 0.5 wavelength spacing for 800 MHz; 672 channels over 400-800 MHz (end
points inclusive) as two shards of 336; T = 32768 spectra; 128 beams on a
16 x 8 direction-cosine grid; voltages complex int4 with Gaussian-like noise
sigma = 2.5 plus a point source at per-sample SNR 5 in a seeded on-grid
direction, generated on the device; weights complex64 (FP64 phase); output
float32 integrated over 320 spectra plus int8 chunk quantization.

One step = beamform + |.|^2 + integrate + quantize both shards.
Metric: beam-samples/s = T * F * B / step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--kernel tensor|tiled]
    python bench.py --impl reference ...   # the reference CPU implementation

Under torchrun (N > 1) every rank runs its own independent copy of the
workload (channel shards are independent; no collective on the data path):
weak scaling, value = all ranks' beam-samples / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from contextlib import nullcontext as _nullcontext
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

C_LIGHT = 299_792_458.0
T_SPECTRA = 32768
N_SHARDS = 2
F_SHARD = 336
N_ANT = 64
N_BEAMS = 128
S_INT = 320
SIGMA = 2.5
SNR = 5.0
SEED = 0
METRIC = "beam-samples/s (T*F*B)"

# DRAM bytes (read + write) per launch of each workload's dominant kernel, from
# one ncu capture each (dram__bytes_read.sum + dram__bytes_write.sum).  The
# grid figure was captured on one shard and the tracker figure on T = 32768;
# both are scaled to a full launch by the units processed.  The captures and
# their commands are summarised under profiles/.
NCU_TRAFFIC = {
    "grid": 2 * (768.05e6 + 19.96e6),
    "grid_cov": 2 * (767.84e6 + 19.31e6),
    "tracker": 8 * (704.715776e6 + 4.859392e6),
    "doa": 1.410263e9 + 162.521600e6,
}


# --------------------------------------------------------------------------
# workload definition (host side, FP64)
# --------------------------------------------------------------------------

def workload_geometry():
    lam = C_LIGHT / 800e6
    spacing = 0.5 * lam
    pos = np.zeros((N_ANT, 3), np.float32)
    for r in range(2):
        for c in range(32):
            pos[r * 32 + c] = (c * spacing, r * spacing, 0.0)
    F = N_SHARDS * F_SHARD
    freq = (400e6 + np.arange(F) * (400e6 / (F - 1))).astype(np.float32)
    ls = -0.45 + 0.06 * np.arange(16)
    ms = -0.21 + 0.06 * np.arange(8)
    dirs = np.zeros((N_BEAMS, 3), np.float32)
    for j in range(8):
        for i in range(16):
            l, m = np.float32(ls[i]), np.float32(ms[j])
            dirs[j * 16 + i] = (l, m, np.sqrt(np.float32(1) - (l * l + m * m)))
    return pos, freq, dirs


def steering_phase(pos, freq, dirs):
    """phase[b][f][a] = 2*pi*f/c * (p_a . d_b) in FP64 (src/weights.cpp:42-55)."""
    k = 2.0 * math.pi * freq.astype(np.float64) / C_LIGHT
    delay = dirs.astype(np.float64) @ pos.astype(np.float64).T  # [B][A]
    return k[None, :, None] * delay[:, None, :]


def workload_weights(pos, freq, dirs):
    ph = steering_phase(pos, freq, dirs)                          # [B][F][A]
    w = np.stack([np.cos(ph), np.sin(ph)], -1).astype(np.float32)  # [B][F][A][2]
    # per shard: [shard][B][336][A][2]
    return np.ascontiguousarray(np.stack([w[:, s * F_SHARD:(s + 1) * F_SHARD] for s in range(N_SHARDS)]))


def workload_source(pos, freq, dirs):
    """mu = A_s * exp(-i phase) of a point source at a seeded on-grid beam."""
    beam = int(np.random.default_rng(SEED).integers(0, N_BEAMS))
    amp = SIGMA * math.sqrt(SNR)
    ph = steering_phase(pos, freq, dirs[beam:beam + 1])[0]          # [F][A]
    mu = np.stack([amp * np.cos(ph), -amp * np.sin(ph)], -1).astype(np.float32)
    return beam, [np.ascontiguousarray(mu[s * F_SHARD:(s + 1) * F_SHARD]) for s in range(N_SHARDS)]


# --------------------------------------------------------------------------
# clocks sampled during the timed region (NVML)
# --------------------------------------------------------------------------

class ClockSampler:
    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
        0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown",
    }

    def __init__(self, device_index: int):
        self.samples: list[int] = []
        self.reasons: set[str] = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._ok = True
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._nv.nvmlDeviceGetClockInfo(self._h, self._nv.NVML_CLOCK_SM))
                r = self._nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.01)

    def __enter__(self):
        if self._ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._ok:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def measured_peaks():
    """(bf16 burst TFLOP/s, bf16 sustained TFLOP/s, HBM GB/s, source)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        burst = d.get("bf16_tflops") or d.get("bf16_tflops_sustained")
        return burst, d.get("bf16_tflops_sustained") or burst, d.get("hbm_gbs"), "measured"
    return 1590.0, 1400.0, 6650.0, "fallback"


def tensor_roofline(alg_flops: float, kernel_ms: float, timed_s: float, clocks: dict) -> dict:
    """Tensor roofline of one launch: algorithmic flop / CUDA-event duration.
    The divisor is the measured burst bf16 peak for a kernel timed in a short
    region, and the sustained (power-capped) one when the timed region lasts a
    second or more or the clocks show the power cap; both fractions are kept."""
    burst, sustained, _, src = measured_peaks()
    achieved = alg_flops / (kernel_ms / 1e3) / 1e12
    capped = timed_s >= 1.0 or "sw_power_cap" in (clocks.get("reasons") or [])
    peak = sustained if capped else burst
    return {"bound": "tensor", "achieved": round(achieved, 2), "peak": peak, "unit": "TFLOP/s",
            "frac": round(achieved / peak, 4),
            "peak_source": f"{src} bf16 dense, {'sustained' if capped else 'burst'}"
                           f" ({'timed region >= 1 s or power cap seen' if capped else 'short timed region, no power cap'})",
            "frac_of_burst": round(achieved / burst, 4), "frac_of_sustained": round(achieved / sustained, 4),
            "kernel_ms": round(kernel_ms, 4), "algorithmic_flop_per_launch": alg_flops}


def host_cpu_info() -> dict:
    """Host CPU description recorded beside every CPU figure."""
    info = {"threads_available": len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity")
            else os.cpu_count(), "omp_num_threads": os.environ.get("OMP_NUM_THREADS")}
    try:
        import subprocess
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        keys = {"Model name": "model", "Socket(s)": "sockets", "Core(s) per socket": "cores_per_socket",
                "Thread(s) per core": "threads_per_core", "NUMA node(s)": "numa_nodes", "CPU(s)": "cpus"}
        for line in out.splitlines():
            k, _, v = line.partition(":")
            if k.strip() in keys:
                info[keys[k.strip()]] = v.strip()
    except Exception:
        pass
    return info


def host_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


# --------------------------------------------------------------------------
# CPU baseline (reference CPU core, or the oracle port when it is absent)
# --------------------------------------------------------------------------

def cpu_baseline(v_host_shard0: np.ndarray, w_shard0: np.ndarray, budget_s: float = 12.0,
                 threads: int | None = None):
    """Time the reference CPU chain (cpu_beamform_packed_intensity_into ->
    cpu_integrate_intensity_into -> cpu_quantize_integrated_intensity) on
    whole 320-spectrum windows of shard 0, one window per host thread, in
    rounds until about budget_s of wall time.  The reference function is
    serial; the harness runs independent windows on separate threads."""
    from oracle import loader as orc
    kind = "reference" if orc.reference_available() else "port"
    threads = threads or host_threads()
    F, A, B = F_SHARD, N_ANT, N_BEAMS
    W_total = len(v_host_shard0) // S_INT

    def one_window(widx: int):
        t0 = widx * S_INT
        v = np.ascontiguousarray(v_host_shard0[t0:t0 + S_INT])
        if kind == "reference":
            I = orc.ref_beamform(v, w_shard0, S_INT, F, A, B)
            integ = orc.ref_integrate(I, S_INT, F, A, B, S_INT)
            orc.ref_quantize(integ, 1, F, A, B)
        else:
            integ = orc.beamform_integrated(v, w_shard0, S_INT, F, A, B, S_INT)
            orc.quantize(integ, 1, F, B)

    done = 0
    with orc.perf_build():
        t_start = time.perf_counter()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            while True:
                list(ex.map(one_window, [(done + i) % W_total for i in range(threads)]))
                done += threads
                if time.perf_counter() - t_start > budget_s:
                    break
        el = time.perf_counter() - t_start
    value = done * S_INT * F * B / el
    return {"value": value, "unit": "beam-samples/s", "cores": threads, "kind": kind,
            "sample": f"{done} whole windows of {S_INT} spectra x {F} channels x {B} beams x {A} "
                      f"antennas (shard 0, one window per thread, {threads} threads), "
                      f"beamform+integrate+quantize, {el:.1f} s",
            "build": orc.reference_perf_flags() if kind == "reference" else "oracle port",
            "host": host_cpu_info()}


# --------------------------------------------------------------------------
# the reference's own CUDA kernels on the same GPU (oracle/_ref/libbfref_cuda.so,
# compiled by oracle/build.py from the reference checkout for sm_100a)
# --------------------------------------------------------------------------

def tiled_weights(w: np.ndarray) -> np.ndarray:
    """Canonical [B][F][A][2] -> the reference's tiled [F][ceil(B/32)][A][32][2]
    (include/beamformer/indexing.hpp:54-61), zero padded."""
    B, F, A, _ = w.shape
    bt = -(-B // 32)
    pad = np.zeros((bt * 32, F, A, 2), np.float32)
    pad[:B] = w
    return np.ascontiguousarray(pad.reshape(bt, 32, F, A, 2).transpose(2, 0, 3, 1, 4))


def event_time(stream, fn, steps: int, flush=None) -> float:
    """Mean CUDA-event time (ms) of fn() on `stream` over `steps` launches;
    flush() (an L2 flush) runs between launches outside the events."""
    import torch
    times = []
    for _ in range(steps):
        if flush is not None:
            flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    return statistics.mean(a.elapsed_time(b) for a, b in times)


def reference_gpu_grid(volt, w_host, integ_t, codes_t, shard_bytes, n_out, W, S, steps, stream,
                       flush=None) -> dict:
    """Time the reference's Tiled integrated grid kernel
    (src/cuda_beamformer.cu:263-354 via launch_packed_integrated_beamformer,
    :488-543) and its int8 chunk quantizer (src/cuda_quantize_int8.cu:30-147)
    on the same voltages as the B200 path, one launch per 336-channel shard
    (the reference's dimension check), and compare their products."""
    import torch
    from oracle import loader as orc
    if not orc.reference_gpu_available():
        return {"unavailable": "oracle/_ref/libbfref_cuda.so was not built (no reference checkout at build time)"}
    g = orc.reference_gpu()
    n_shards, B, F, A = w_host.shape[0], w_host.shape[1], w_host.shape[2], w_host.shape[3]
    T = shard_bytes // (F * A)
    wt = torch.from_numpy(np.stack([tiled_weights(w_host[s]) for s in range(n_shards)])).to(volt.device)
    wt_stride = wt[0].numel()
    integ_r = torch.empty_like(integ_t)
    codes_r = torch.empty_like(codes_t)
    ft, bt = -(-F // 16), -(-B // 16)
    params_r = torch.empty(n_shards * W * ft * bt * 2, dtype=torch.float32, device=volt.device)
    h = stream.cuda_stream

    def step():
        for sh in range(n_shards):
            orc.refgpu_check(g.refgpu_grid_integrated(1, h, volt.data_ptr() + sh * shard_bytes,
                                                      wt.data_ptr() + sh * wt_stride * 4,
                                                      integ_r.data_ptr() + sh * n_out * 4, T, F, A, B, S))
        orc.refgpu_check(g.refgpu_quantize(h, integ_r.data_ptr(), codes_r.data_ptr(), params_r.data_ptr(),
                                           n_shards * W, F, A, B))

    step()
    torch.cuda.synchronize()
    ms = event_time(stream, step, steps, flush)
    ref = integ_r.double()
    rel = ((integ_t.double() - ref).abs() / (1e-3 + ref.abs())).max().item()
    lsb = (codes_t.int() - codes_r.int()).abs()
    return {"kernel": "reference tiled_packed_integrated_voltage_beamformer_kernel + "
                      "quantize_integrated_intensity_kernel (reference sources, nvcc sm_100a)",
            "ms_per_step": ms, "value": T * n_shards * F * B / (ms / 1e3), "steps": steps,
            "launches_per_step": n_shards + 1,
            "max_diff_vs_b200_over_1e-3_plus_abs": rel,
            "int8_codes_differing": int((lsb > 0).sum().item()), "int8_max_lsb": int(lsb.max().item())}


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------

def run_gpu(args):
    import torch
    from beamform_project_b200 import api, native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()

    pos, freq, dirs = workload_geometry()
    w_host = workload_weights(pos, freq, dirs)
    beam, mu_host = workload_source(pos, freq, dirs)
    d = api.Dimensions(T_SPECTRA, F_SHARD, N_ANT, N_BEAMS)
    W = api.integrated_time_count(T_SPECTRA, S_INT)
    qd = api.Dimensions(W, F_SHARD, N_ANT, N_BEAMS)
    n_out = W * F_SHARD * N_BEAMS
    n_par = 2 * api.quantization_parameter_count(qd)

    N_SHARDS = args.shards  # noqa: N806  (the full band is 2; fewer for small profiling cases)
    w_host = np.ascontiguousarray(w_host[:N_SHARDS])
    volt = torch.empty(N_SHARDS * T_SPECTRA * F_SHARD * N_ANT, dtype=torch.uint8, device=dev)
    shard_bytes = T_SPECTRA * F_SHARD * N_ANT
    for s in range(N_SHARDS):
        api.generate_voltage(None, SEED + 1000 * rank, s * shard_bytes, SIGMA,
                             torch.from_numpy(mu_host[s]).to(dev), T_SPECTRA,
                             volt[s * shard_bytes:(s + 1) * shard_bytes], d)
    weights = torch.from_numpy(w_host).to(dev)
    integ = torch.empty(N_SHARDS * n_out, dtype=torch.float32, device=dev)
    codes = torch.empty(N_SHARDS * n_out, dtype=torch.int8, device=dev)
    params = torch.empty(N_SHARDS * n_par, dtype=torch.float32, device=dev)
    kernel = args.kernel
    tensor_path = kernel in ("tensor", "auto")
    split = None
    tune = None
    if tensor_path:
        split = torch.empty(api.split_weight_bytes(d, N_SHARDS), dtype=torch.uint8, device=dev)
        api.prepare_split_weights(None, weights, split, d, N_SHARDS)
        workspace = torch.empty(api.grid_tensor_workspace_bytes(d, S_INT, N_SHARDS), dtype=torch.uint8,
                                device=dev)
    if kernel == "auto":
        # the checked covariance form, with the grid path's launch choices
        # tuned for this class first (every candidate timed, parity-gated)
        auto_w = torch.empty(api.auto_weight_bytes(d, N_SHARDS), dtype=torch.uint8, device=dev)
        api.prepare_auto_weights(None, weights, auto_w, d, N_SHARDS)
        auto_ws = torch.zeros(max(256, api.grid_auto_workspace_bytes(d, S_INT, N_SHARDS)), dtype=torch.uint8,
                              device=dev)
        if args.tune:
            t_tune = time.perf_counter()
            tune = api.autotune_grid(None, d, S_INT, N_SHARDS)
            tune["wall_s"] = round(time.perf_counter() - t_tune, 2)
    torch.cuda.synchronize()

    main_events = []  # CUDA events around the dominant kernel of each timed step
    qd_all = api.Dimensions(N_SHARDS * W, F_SHARD, N_ANT, N_BEAMS)  # [shard][W] == [shard * W + w]

    def step(record=False):
        if record:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        if kernel == "auto":
            # checked form (covariance form + recomputed units), then the int8 chunk quantizer
            api.grid_auto_integrated(None, volt, auto_w, integ, None, None, auto_ws, d, S_INT, N_SHARDS)
            if record:
                e1.record(stream)
                main_events.append((e0, e1))
            api.launch_quantize_integrated_intensity(None, integ, codes, params, qd_all)
            return 3 if tune is None or tune["chosen"]["form"] != "split" else 2
        if kernel == "tensor":
            if args.fused_quant:
                # one kernel: beamform, |.|^2, integration and int8 quantization fused
                api.grid_tensor_quantized(None, volt, split, integ, codes, params, workspace, d, S_INT,
                                          N_SHARDS)
                if record:
                    e1.record(stream)
                launches = 1
            else:
                # tensor kernel (beamform, |.|^2, integration), then the int8 chunk quantizer
                api.grid_tensor_integrated(None, volt, split, integ, None, None, d, S_INT, N_SHARDS)
                if record:
                    e1.record(stream)
                api.launch_quantize_integrated_intensity(None, integ, codes, params, qd_all)
                launches = 2
            if record:
                main_events.append((e0, e1))
            return launches
        else:
            launches = 0
            for s in range(N_SHARDS):
                api.launch_packed_integrated_beamformer(
                    api.CudaBeamformerKernel.Direct, None, volt[s * shard_bytes:],
                    weights[s], integ[s * n_out:], d, S_INT)
                launches += 1
            for s in range(N_SHARDS):
                api.launch_quantize_integrated_intensity(None, integ[s * n_out:], codes[s * n_out:],
                                                         params[s * n_par:], qd)
                launches += 1
        if record:
            e1.record(stream)
            main_events.append((e0, e1))
        return launches

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    launches = 0
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for _ in range(args.steps):
            launches += step(record=True)
        t1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    main_ms = statistics.mean(a.elapsed_time(b) for a, b in main_events)
    if dist:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_per_step = ms / args.steps
    samples_per_step = T_SPECTRA * N_SHARDS * F_SHARD * N_BEAMS
    value = samples_per_step * world / (ms_per_step / 1e3)

    # end to end through the public API: pinned host voltage in, results out
    host_v = torch.empty(volt.numel(), dtype=torch.uint8, pin_memory=True)
    host_v.copy_(volt)
    host_i = torch.empty(integ.numel(), dtype=torch.float32, pin_memory=True)
    host_c = torch.empty(codes.numel(), dtype=torch.int8, pin_memory=True)
    host_p = torch.empty(params.numel(), dtype=torch.float32, pin_memory=True)
    e2e_steps = max(1, args.e2e_steps)

    def e2e_step():
        volt.copy_(host_v, non_blocking=True)
        step()
        host_i.copy_(integ, non_blocking=True)
        host_c.copy_(codes, non_blocking=True)
        host_p.copy_(params, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    a1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = a0.elapsed_time(a1) / e2e_steps
    e2e_path = "torch copies + device-pointer C-ABI calls, one phase after the other"
    serial_ms, e2e_chunk, e2e_match = None, None, None
    if tensor_path and not args.fused_quant:
        # the host-buffer C-ABI pipeline: the same products, with each time
        # chunk's copy-in, kernels and copy-out overlapped on three streams
        serial_ms = e2e_ms
        pipe = api.GridHostPipeline(d, S_INT, N_SHARDS, checked=kernel == "auto")
        pipe.upload_weights(w_host)
        e2e_chunk = pipe.chunk_spectra
        pipe.run(host_v, host_i, host_c, host_p)
        e2e_match = bool(torch.equal(host_i, integ.cpu()) and torch.equal(host_c, codes.cpu())
                         and torch.equal(host_p, params.cpu()))
        if dist:
            dist.barrier()
        e2e_ms = statistics.mean(pipe.run(host_v, host_i, host_c, host_p) for _ in range(e2e_steps))
        pipe.close()
        e2e_path = ("bf_grid_pipeline_run" + (" (checked form)" if kernel == "auto" else "") +
                    ": pinned host buffers, chunked copy-in / kernels / copy-out overlap")
    if dist:
        tt = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e_value = samples_per_step * world / (e2e_ms / 1e3)

    # sanity: the injected source beam is the brightest beam of the band
    prof = integ.view(N_SHARDS, W, F_SHARD, N_BEAMS).double().sum(dim=(0, 1, 2))
    peak_ok = int(torch.argmax(prof).item()) == beam

    # the plain drop-in beside it: the reference-order float32 kernel (Direct,
    # bit-identical to the reference CPU core) and the quantizer, same inputs
    plain = None
    if tensor_path and args.plain_steps > 0:
        integ_p = torch.empty_like(integ)
        codes_p = torch.empty_like(codes)
        params_p = torch.empty_like(params)

        def plain_step():
            for s in range(N_SHARDS):
                api.launch_packed_integrated_beamformer(api.CudaBeamformerKernel.Direct, None,
                                                        volt[s * shard_bytes:], weights[s], integ_p[s * n_out:],
                                                        d, S_INT)
            api.launch_quantize_integrated_intensity(None, integ_p, codes_p, params_p, qd_all)
        plain_step()
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.plain_steps):
            plain_step()
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = p0.elapsed_time(p1) / args.plain_steps
        ref = integ_p.double()
        rel = ((integ.double() - ref).abs() / ref.abs().clamp_min(1e-30)).max().item()
        lsb = (codes.int() - codes_p.int()).abs()
        plain = {"kernel": "grid_exact_kernel (Direct, reference float32 order) + quantize_kernel",
                 "ms_per_step": plain_ms, "value": samples_per_step / (plain_ms / 1e3),
                 "tensor_speedup": plain_ms / ms_per_step, "max_rel_diff_vs_tensor": rel,
                 "int8_codes_differing": int((lsb > 0).sum().item()), "int8_max_lsb": int(lsb.max().item())}

    # the covariance form beside it (opt-in kernel, same inputs): time and
    # distance from the reference-order float32 output
    cov = None
    if tensor_path and args.cov_steps > 0 and plain is not None:
        covw = torch.empty(api.cov_weight_bytes(d, N_SHARDS), dtype=torch.uint8, device=dev)
        api.prepare_cov_weights(None, weights, covw, d, N_SHARDS)
        integ_c = torch.empty_like(integ)
        codes_c = torch.empty_like(codes)
        params_c = torch.empty_like(params)

        def cov_step():
            api.grid_cov_integrated(None, volt, covw, integ_c, None, None, d, S_INT, N_SHARDS)

        cov_step()
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(args.cov_steps):
            cov_step()
        c1.record(stream)
        torch.cuda.synchronize()
        assert native.take_device_error() == 0
        cov_ms = c0.elapsed_time(c1) / args.cov_steps
        api.launch_quantize_integrated_intensity(None, integ_c, codes_c, params_c, qd_all)
        torch.cuda.synchronize()
        ref = integ_p.double()
        rel = ((integ_c.double() - ref).abs() / ref.abs().clamp_min(1e-30)).max().item()
        lsb = (codes_c.int() - codes_p.int()).abs()
        cov = {"kernel": "grid_cov_kernel (covariance form, opt-in)", "kernel_ms": cov_ms,
               "value": samples_per_step / (cov_ms / 1e3),
               "algorithmic_tflops": (8 * T_SPECTRA * N_SHARDS * F_SHARD * N_ANT * N_BEAMS
                                      + 3 * samples_per_step) / (cov_ms / 1e3) / 1e12,
               "max_rel_diff_vs_plain": rel, "int8_codes_differing": int((lsb > 0).sum().item()),
               "int8_max_lsb": int(lsb.max().item())}
        del covw, integ_c, codes_c, params_c

        # the checked form (covariance form + split-kernel recomputation of
        # every unit whose error estimate is above the calibrated limit)
        aw = torch.empty(api.auto_weight_bytes(d, N_SHARDS), dtype=torch.uint8, device=dev)
        api.prepare_auto_weights(None, weights, aw, d, N_SHARDS)
        aws = torch.zeros(max(256, api.grid_auto_workspace_bytes(d, S_INT, N_SHARDS)), dtype=torch.uint8,
                          device=dev)
        integ_a = torch.empty_like(integ)

        def auto_step():
            api.grid_auto_integrated(None, volt, aw, integ_a, None, None, aws, d, S_INT, N_SHARDS)

        auto_step()
        torch.cuda.synchronize()
        a_ms = event_time(stream, auto_step, args.cov_steps)
        assert native.take_device_error() == 0
        n_units = int(aws[:4].view(torch.int32).item())
        rel = ((integ_a.double() - integ_p.double()).abs() / integ_p.double().abs().clamp_min(1e-30)).max().item()
        if kernel == "auto":
            def split_step():
                api.grid_tensor_integrated(None, volt, split, integ_p2, None, None, d, S_INT, N_SHARDS)
            integ_p2 = torch.empty_like(integ)
            split_step()
            cov["split_form_ms"] = event_time(stream, split_step, args.cov_steps)
            del integ_p2
        cov["checked_form"] = {
            "kernel": "grid_cov_kernel with error estimates + grid_tensor_kernel over the listed units",
            "ms_per_step": a_ms, "value": samples_per_step / (a_ms / 1e3),
            "algorithmic_tflops": (8 * T_SPECTRA * N_SHARDS * F_SHARD * N_ANT * N_BEAMS
                                   + 3 * samples_per_step) / (a_ms / 1e3) / 1e12,
            "units_recomputed": n_units, "max_rel_diff_vs_plain": rel}
        del aw, aws, integ_a

    # the reference's own CUDA kernels (Tiled + int8 quantizer) on the same GPU and inputs
    ref_gpu = None
    if tensor_path and args.ref_gpu_steps > 0:
        ref_gpu = reference_gpu_grid(volt, w_host, integ, codes, shard_bytes, n_out, W, S_INT,
                                     args.ref_gpu_steps, stream)
        if "ms_per_step" in ref_gpu:
            ref_gpu["b200_speedup"] = ref_gpu["ms_per_step"] / ms_per_step

    cmac = T_SPECTRA * N_SHARDS * F_SHARD * N_ANT * N_BEAMS
    alg_flops = 8 * cmac + 3 * samples_per_step
    csum = clocks.summary()
    roofline = tensor_roofline(alg_flops, main_ms, ms / 1e3, csum)
    if kernel == "auto":
        roofline["traffic"] = round(NCU_TRAFFIC["grid_cov"]) if N_SHARDS == 2 and "grid_cov" in NCU_TRAFFIC \
            else None
        roofline["kernel"] = ("grid_cov_kernel + grid_tensor_kernel over recomputed units (checked form)"
                              if tune is None or tune["chosen"]["form"] != "split" else "grid_tensor_kernel")
    else:
        roofline["traffic"] = (round(NCU_TRAFFIC["grid"]) if kernel == "tensor" and N_SHARDS == 2
                               and not args.fused_quant else None)
        roofline["kernel"] = "grid_tensor_kernel" if kernel == "tensor" else "grid_exact_kernel+quantize"

    line = {
        "metric": METRIC, "value": value, "unit": "beam-samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int4xfp16->fp32",
        "data": "synthetic (seeded on-device int4 generator, point source at beam %d)" % beam,
        "config": {"workload": "full-band split-precision grid: A=64 (2x32), F=672 (2 shards x 336), "
                               "T=32768, B=128 (16x8), S=320, float32 + int8 chunk codes",
                   "kernel": kernel, "parallelism": f"independent replicas x{world}",
                   "l2": "inputs (1.41 GB voltage) exceed L2; no flush"},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "beam-samples/s",
                "h2d_bytes_per_step": host_v.numel(),
                "d2h_bytes_per_step": host_i.numel() * 4 + host_c.numel() + host_p.numel() * 4,
                "ms_per_step": e2e_ms, "path": e2e_path, "chunk_spectra": e2e_chunk,
                "serial_ms_per_step": serial_ms, "products_match_device_run": e2e_match},
        "gpu_launches": launches,
        "clocks": csum,
        "source_peak_ok": peak_ok,
        "plain_dropin": plain,
        "covariance_form": cov,
        "reference_gpu": ref_gpu,
        "autotune": tune,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v0 = volt[:shard_bytes].cpu().numpy().reshape(T_SPECTRA, F_SHARD, N_ANT)
        line["cpu_baseline"] = cpu_baseline(v0, w_host[0], budget_s=args.cpu_seconds)
    if world == 1 and args.configs and tensor_path:
        # the other workloads, each measured the same way (CUDA-event kernel
        # time, roofline, CPU baseline, end to end, clocks), as sub-records
        del volt, weights, integ, codes, params, split, workspace, host_v, host_i, host_c, host_p
        torch.cuda.empty_cache()
        line["configs"] = run_configs(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_configs(args) -> dict:
    """Plain grid, tracker, DOA and served-mix records beside the headline
    (one GPU).  Each gets a few steps and a shorter CPU sample so that the
    whole default run stays within a few minutes."""
    import copy
    import torch
    sub = copy.copy(args)
    sub.steps = max(3, min(args.steps, 20))
    sub.warmup = max(3, min(args.warmup, 5))
    sub.e2e_steps = min(args.e2e_steps, 3)
    sub.cpu_seconds = args.config_cpu_seconds
    sub.plain_steps = min(args.plain_steps, 2)
    sub.kernel = "tensor"
    sub.t_spectra = TR_T
    out = {}
    for name, fn in (("c1_plain_grid", measure_c1), ("c3_tracker", lambda a: run_tracker(a, emit=False)),
                     ("c4_doa", lambda a: run_doa(a, emit=False)),
                     ("c5_served_mix", lambda a: run_serve(a, emit=False))):
        t0 = time.perf_counter()
        try:
            rec = fn(sub)
        except Exception as exc:  # a failed sub-record must not hide the headline
            rec = {"error": f"{type(exc).__name__}: {exc}"}
        if isinstance(rec, dict):
            rec["wall_s"] = round(time.perf_counter() - t0, 1)
        out[name] = rec
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------------
# plain fixed-grid workload (CPU-runnable): 32-element line array at 0.5
# wavelength of 600 MHz, F=336 over 400-600 MHz (end points inclusive),
# T=1024, Gaussian sigma=2 (seed 0), 16 beams at l = -0.5 + b/15, m = 0,
# complex64 weights, float32 power integrated over 10 spectra
# --------------------------------------------------------------------------
C1_T, C1_A, C1_B, C1_S, C1_SIGMA = 1024, 32, 16, 10, 2.0


def c1_geometry():
    lam = C_LIGHT / 600e6
    pos = np.zeros((C1_A, 3), np.float32)
    pos[:, 0] = (np.arange(C1_A) * (0.5 * lam)).astype(np.float32)
    freq = (400e6 + np.arange(F_SHARD) * (200e6 / (F_SHARD - 1))).astype(np.float32)
    dirs = np.zeros((C1_B, 3), np.float32)
    for b in range(C1_B):
        l = np.float32(-0.5 + b / 15.0)
        dirs[b] = (l, 0.0, np.sqrt(np.float32(1) - l * l))
    return pos, freq, dirs


def c1_inputs(dev):
    """Device voltages, canonical and tiled weights of the plain-grid workload."""
    import torch
    from beamform_project_b200 import api
    pos, freq, dirs = c1_geometry()
    d = api.Dimensions(C1_T, F_SHARD, C1_A, C1_B)
    volt = torch.empty(C1_T * F_SHARD * C1_A, dtype=torch.uint8, device=dev)
    api.generate_voltage(None, SEED, 0, C1_SIGMA, None, C1_T, volt, d)
    w = torch.empty(C1_B * F_SHARD * C1_A * 2, dtype=torch.float32, device=dev)
    api.generate_weights(None, torch.from_numpy(pos).to(dev), torch.from_numpy(freq).to(dev),
                         torch.from_numpy(dirs).to(dev), w, d)
    return d, volt, w


def measure_c1(args) -> dict:
    """The plain fixed-grid workload: split-precision tensor path, the
    reference-order Tiled kernel (bit-identical to the reference CPU core), the
    reference's own Tiled kernel on the same GPU, and the reference CPU core.
    Its 11 MB of voltage fit in L2, so every timed launch follows an L2 flush
    (a 256 MB write) outside its events."""
    import torch
    from beamform_project_b200 import api, native
    from oracle import loader as orc
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    d, volt, w = c1_inputs(dev)
    W = api.integrated_time_count(C1_T, C1_S)
    n_out = W * F_SHARD * C1_B
    w_host = w.cpu().numpy().reshape(C1_B, F_SHARD, C1_A, 2)
    wt = torch.from_numpy(tiled_weights(w_host)).to(dev)
    split = torch.empty(api.split_weight_bytes(d), dtype=torch.uint8, device=dev)
    api.prepare_split_weights(None, w, split, d)
    out_t = torch.empty(n_out, dtype=torch.float32, device=dev)
    out_x = torch.empty(n_out, dtype=torch.float32, device=dev)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    steps = max(3, min(args.steps, 50))

    def flush():
        flush_buf.zero_()

    def tensor_step():
        api.grid_tensor_integrated(None, volt, split, out_t, None, None, d, C1_S)

    def exact_step():
        api.launch_packed_integrated_beamformer(api.CudaBeamformerKernel.Tiled, None, volt, wt, out_x, d, C1_S)

    for _ in range(3):
        tensor_step()
        exact_step()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        t_ms = event_time(stream, tensor_step, steps, flush)
        x_ms = event_time(stream, exact_step, steps, flush)
    assert native.take_device_error() == 0
    ref_gpu = None
    if args.ref_gpu_steps > 0 and orc.reference_gpu_available():
        g = orc.reference_gpu()
        out_r = torch.empty_like(out_t)

        def ref_step():
            orc.refgpu_check(g.refgpu_grid_integrated(1, stream.cuda_stream, volt.data_ptr(), wt.data_ptr(),
                                                      out_r.data_ptr(), C1_T, F_SHARD, C1_A, C1_B, C1_S))
        ref_step()
        r_ms = event_time(stream, ref_step, steps, flush)
        ref_gpu = {"kernel": "reference tiled_packed_integrated_voltage_beamformer_kernel (nvcc sm_100a)",
                   "kernel_ms": r_ms, "value": C1_T * F_SHARD * C1_B / (r_ms / 1e3),
                   "b200_tensor_speedup": r_ms / t_ms,
                   "max_diff_vs_exact_over_1e-3_plus_abs":
                       ((out_r.double() - out_x.double()).abs() / (1e-3 + out_x.double().abs())).max().item()}
    # parity on the whole workload against the reference CPU core
    v_host = volt.cpu().numpy().reshape(C1_T, F_SHARD, C1_A)
    parity = None
    if orc.reference_available():
        ref32 = orc.ref_integrate(orc.ref_beamform(v_host, w_host, C1_T, F_SHARD, C1_A, C1_B),
                                  C1_T, F_SHARD, C1_A, C1_B, C1_S)
        gt = out_t.cpu().numpy().reshape(ref32.shape).astype(np.float64)
        parity = {"exact_kernel_bit_identical_to_reference_cpu": bool(np.array_equal(
                      out_x.cpu().numpy().reshape(ref32.shape), ref32)),
                  "tensor_max_rel_vs_reference_fp32": float((np.abs(gt - ref32) / np.abs(ref32)).max()),
                  "tensor_within_1e-3_plus_1e-5_rel": bool(np.all(np.abs(gt - ref32) <= 1e-3 + 1e-5 * np.abs(ref32)))}
    # end to end: pinned host voltage in, integrated powers out, every step
    host_v = torch.empty(volt.numel(), dtype=torch.uint8, pin_memory=True)
    host_v.copy_(volt)
    host_o = torch.empty(n_out, dtype=torch.float32, pin_memory=True)

    def e2e_step():
        volt.copy_(host_v, non_blocking=True)
        tensor_step()
        host_o.copy_(out_t, non_blocking=True)
    e2e_step()
    e2e_ms = event_time(stream, e2e_step, max(3, args.e2e_steps), flush)
    samples = C1_T * F_SHARD * C1_B
    _, _, hbm_gbs, peak_src = measured_peaks()
    alg_bytes = C1_T * F_SHARD * C1_A + n_out * 4
    # CPU: the reference core (performance build) on the whole workload, one
    # thread, and the same split into time blocks on all host threads
    cpu = None
    if not args.no_cpu_baseline and orc.reference_available():
        threads = host_threads()
        with orc.perf_build():
            t0 = time.perf_counter()
            n1 = 0
            while True:
                orc.ref_integrate(orc.ref_beamform(v_host, w_host, C1_T, F_SHARD, C1_A, C1_B),
                                  C1_T, F_SHARD, C1_A, C1_B, C1_S)
                n1 += 1
                if time.perf_counter() - t0 > args.cpu_seconds / 2:
                    break
            one = n1 * samples / (time.perf_counter() - t0)
            blocks = [(b * C1_T // threads // C1_S * C1_S, (b + 1) * C1_T // threads // C1_S * C1_S)
                      for b in range(threads)]
            blocks[-1] = (blocks[-1][0], C1_T)

            def block(i):
                a, b = blocks[i]
                if b > a:
                    vv = np.ascontiguousarray(v_host[a:b])
                    orc.ref_integrate(orc.ref_beamform(vv, w_host, b - a, F_SHARD, C1_A, C1_B),
                                      b - a, F_SHARD, C1_A, C1_B, C1_S)
            t0 = time.perf_counter()
            nt = 0
            with ThreadPoolExecutor(max_workers=threads) as ex:
                while True:
                    list(ex.map(block, range(threads)))
                    nt += 1
                    if time.perf_counter() - t0 > args.cpu_seconds / 2:
                        break
            many = nt * samples / (time.perf_counter() - t0)
        cpu = {"value": many, "unit": "beam-samples/s", "cores": threads, "kind": "reference",
               "single_thread_value": one,
               "sample": f"the whole workload: {n1} runs on 1 thread (cpu_beamform_packed_intensity_into + "
                         f"cpu_integrate_intensity_into, serial), {nt} runs split into {threads} time blocks "
                         f"on {threads} threads",
               "build": orc.reference_perf_flags(), "host": host_cpu_info()}
    csum = clocks.summary()
    return {
        "workload": "plain grid: A=32 line array (0.5 lambda at 600 MHz), F=336 over 400-600 MHz, T=1024, "
                    "B=16 (l = -0.5 + b/15, m = 0), Gaussian sigma=2 seed 0, complex64 weights, S=10, float32",
        "value": samples / (t_ms / 1e3), "unit": "beam-samples/s", "kernel": "grid_tensor_kernel (S=10 form)",
        "kernel_ms": t_ms, "steps": steps, "l2": "11 MB input fits L2: 256 MB flush before every timed launch",
        "plain_dropin": {"kernel": "grid_exact_kernel (Tiled, reference float32 order)", "kernel_ms": x_ms,
                         "value": samples / (x_ms / 1e3)},
        "reference_gpu": ref_gpu, "parity": parity,
        "roofline": {"bound": "hbm", "achieved": round(alg_bytes / (t_ms / 1e3) / 1e9, 1), "peak": hbm_gbs,
                     "unit": "GB/s", "frac": round(alg_bytes / (t_ms / 1e3) / 1e9 / hbm_gbs, 4),
                     "traffic": None, "peak_source": peak_src + " (copy bandwidth)",
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "note": "a 13 MB launch: launch latency and the kernel ramp, not HBM, set its time"},
        "e2e": {"value": samples / (e2e_ms / 1e3), "unit": "beam-samples/s", "h2d_bytes_per_step": host_v.numel(),
                "d2h_bytes_per_step": n_out * 4, "ms_per_step": e2e_ms},
        "cpu_baseline": cpu, "clocks": csum, "gpu_launches": 2 * steps,
    }


# --------------------------------------------------------------------------
# tracker workload: A=64 (2 x 32), F=336 (400-600 MHz), T=262144 spectra,
# one steering direction per 1024-spectrum window (W=256), noise sigma=2 plus
# a source at SNR 3 drifting 0.02 in direction cosine over the run
# --------------------------------------------------------------------------
TR_T = 262144
TR_S = 1024
TR_SIGMA = 2.0
TR_SNR = 3.0
TR_L0, TR_M0 = 0.10, -0.05
TR_DRIFT = 0.02


def tracker_inputs(T: int = TR_T):
    pos, freq_full, _ = workload_geometry()
    freq = np.ascontiguousarray(freq_full[:F_SHARD])
    rate_l = TR_DRIFT * math.cos(math.radians(30.0)) / T
    rate_m = TR_DRIFT * math.sin(math.radians(30.0)) / T
    from beamform_project_b200 import api
    dirs = api.tracker_window_directions(TR_L0, TR_M0, rate_l, rate_m, T, TR_S)
    # the source sits at each window's mid point (the beam points at its start)
    W = len(dirs)
    mids = np.stack([api.direction_from_lm(TR_L0 + (w + 0.5) * TR_S * rate_l,
                                           TR_M0 + (w + 0.5) * TR_S * rate_m) for w in range(W)])
    k = 2.0 * math.pi * freq.astype(np.float64) / C_LIGHT
    ph = k[None, :, None] * (mids.astype(np.float64) @ pos.astype(np.float64).T)[:, None, :]
    amp = TR_SIGMA * math.sqrt(TR_SNR)
    mu = np.stack([amp * np.cos(ph), -amp * np.sin(ph)], -1).astype(np.float32)  # [W][F][A][2]
    return pos, freq, dirs, mu, (rate_l, rate_m)


def run_tracker(args, emit: bool = True):
    if args.impl == "reference":
        return run_tracker_reference(args)
    import torch
    from beamform_project_b200 import api, native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    TR_T = args.t_spectra  # noqa: N806
    pos, freq, dirs, mu, _ = tracker_inputs(TR_T)
    d = api.Dimensions(TR_T, F_SHARD, N_ANT, 1)
    W = len(dirs)
    volt = torch.empty(TR_T * F_SHARD * N_ANT, dtype=torch.uint8, device=dev)
    api.generate_voltage(None, SEED + 77 + 1000 * rank, 0, TR_SIGMA, torch.from_numpy(mu).to(dev), TR_S,
                         volt, d)
    pos_d = torch.from_numpy(pos).to(dev)
    k_d = torch.from_numpy(api.wave_numbers(freq)).to(dev)
    dirs_d = torch.from_numpy(dirs).to(dev)
    integ = torch.empty(W * F_SHARD, dtype=torch.float32, device=dev)
    inten = torch.empty(TR_T * F_SHARD, dtype=torch.float32, device=dev)
    mode = api.TrackerMode.Streaming if args.kernel in ("auto", "tensor", "stream") else api.TrackerMode.ReferenceOrder

    def step(per_spectrum=False):
        api.tracker(None, mode, volt, pos_d, k_d, dirs_d, inten if per_spectrum else None, integ, d, TR_S)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    events = []
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 100))
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            events.append((e0, e1))
        t1.record(stream)
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    kern_ms = statistics.mean(a.elapsed_time(b) for a, b in events)
    if dist:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    # per-spectrum (drop-in [T][F][1]) variant, timed separately
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    step(True)
    s0.record(stream)
    for _ in range(5):
        step(True)
    s1.record(stream)
    torch.cuda.synchronize()
    ps_ms = s0.elapsed_time(s1) / 5

    # the plain drop-in beside it: the reference-order tracker (mode 0, float32
    # order of the reference CPU tracker), same inputs, same outputs
    plain = None
    if mode == api.TrackerMode.Streaming and args.plain_steps > 0:
        integ_p = torch.empty_like(integ)
        inten_p = torch.empty_like(inten)

        def plain_step():
            api.tracker(None, api.TrackerMode.ReferenceOrder, volt, pos_d, k_d, dirs_d, inten_p, integ_p, d, TR_S)
        plain_step()
        torch.cuda.synchronize()
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(args.plain_steps):
            plain_step()
        q1.record(stream)
        torch.cuda.synchronize()
        plain_ms = q0.elapsed_time(q1) / args.plain_steps
        step(True)
        torch.cuda.synchronize()
        ref = inten_p.double()
        rel = ((inten.double() - ref).abs() / (1e-3 + ref.abs())).max().item()
        plain = {"kernel": "tracker_exact_kernel (reference float32 order), per-spectrum + integrated",
                 "ms_per_step": plain_ms, "value": TR_T * F_SHARD / (plain_ms / 1e3),
                 "streaming_speedup_per_spectrum_output": plain_ms / ps_ms,
                 "max_diff_vs_streaming_over_1e-3_plus_abs": rel}

    # the reference's own CUDA tracker (v5, device resident) on the same GPU and
    # voltages; it hard-codes its default geometry, so the B200 tracker runs
    # once more on that geometry to compare products
    ref_gpu = None
    if mode == api.TrackerMode.Streaming and args.ref_gpu_steps > 0:
        ref_gpu = reference_gpu_tracker(volt, inten, TR_T, args.ref_gpu_steps, stream, ps_ms)

    # end to end: pinned host voltage in, integrated powers out
    host_v = torch.empty(volt.numel(), dtype=torch.uint8, pin_memory=True)
    host_v.copy_(volt)
    host_i = torch.empty(integ.numel(), dtype=torch.float32, pin_memory=True)
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    n_e2e = max(1, args.e2e_steps)
    a0.record(stream)
    for _ in range(n_e2e):
        volt.copy_(host_v, non_blocking=True)
        step()
        host_i.copy_(integ, non_blocking=True)
    a1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = a0.elapsed_time(a1) / n_e2e

    samples = TR_T * F_SHARD
    in_bytes = TR_T * F_SHARD * N_ANT
    alg_bytes = in_bytes + W * F_SHARD * 4
    _, _, hbm_gbs, peak_src = measured_peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": samples * world / (ms / 1e3), "unit": "beam-samples/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int4xfp16->fp32",
        "data": "synthetic (seeded on-device int4 generator, source drifting along the track)",
        "config": {"workload": "tracker: A=64 (2x32), F=336, T=262144, window 1024 (W=256), "
                               "float32 integrated power per window per channel",
                   "kernel": "tracker_stream_kernel" if mode == 1 else "tracker_exact_kernel",
                   "parallelism": f"independent replicas x{world}",
                   "l2": "inputs (5.64 GB voltage) exceed L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_gbs, "unit": "GB/s",
                     "frac": round(achieved / hbm_gbs, 4),
                     "traffic": round(NCU_TRAFFIC["tracker"]) if mode == 1 and TR_T == 262144 else None,
                     "peak_source": peak_src + " (copy bandwidth)", "kernel_ms": round(kern_ms, 4),
                     "algorithmic_bytes_per_launch": alg_bytes},
        "plain_dropin": plain,
        "reference_gpu": ref_gpu,
        "per_spectrum_output": {"ms_per_step": ps_ms, "value": samples / (ps_ms / 1e3),
                                "bytes_per_launch": in_bytes + TR_T * F_SHARD * 4,
                                "achieved_gbs": (in_bytes + TR_T * F_SHARD * 4) / (ps_ms / 1e3) / 1e9},
        "e2e": {"value": samples * world / (e2e_ms / 1e3), "unit": "beam-samples/s",
                "h2d_bytes_per_step": host_v.numel(), "d2h_bytes_per_step": host_i.numel() * 4,
                "ms_per_step": e2e_ms},
        "gpu_launches": steps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v0 = volt[: 64 * TR_S * F_SHARD * N_ANT].cpu().numpy().reshape(-1, F_SHARD, N_ANT)
        line["cpu_baseline"] = tracker_cpu_baseline(v0, budget_s=args.cpu_seconds)
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


def reference_gpu_tracker(volt, inten, T, steps, stream, b200_ps_ms) -> dict:
    """Time cuda_beam_tracker_v5_device_resident (src/cuda_beam_tracker_v5.cu:383-420;
    per-spectrum [T][F][1] output, its default time_chunk_size 80 and unroll 8,
    V5ExecutionConfig in include/beamformer/cuda_beam_tracker_v5.hpp:45-49) on
    the same voltages, and compare it with the B200 streaming tracker run on
    the reference's default geometry and the same trajectory."""
    import torch
    from beamform_project_b200 import api
    from oracle import loader as orc
    if not orc.reference_gpu_available():
        return {"unavailable": "oracle/_ref/libbfref_cuda.so was not built (no reference checkout at build time)"}
    g = orc.reference_gpu()
    dev = volt.device
    rate_l = TR_DRIFT * math.cos(math.radians(30.0)) / T
    rate_m = TR_DRIFT * math.sin(math.radians(30.0)) / T
    out_r = torch.empty_like(inten)
    h = stream.cuda_stream

    def step():
        orc.refgpu_check(g.refgpu_tracker_v5(volt.data_ptr(), out_r.data_ptr(), T, F_SHARD, N_ANT, TR_L0, TR_M0,
                                             rate_l, rate_m, TR_S, 80, 8, h))
    step()
    torch.cuda.synchronize()
    ms = event_time(stream, step, steps)
    # the B200 tracker on the reference's default geometry (8 x 8 at 0.6 m, 300 MHz + ch * 300 kHz)
    pos = torch.from_numpy(api.default_positions(N_ANT)).to(dev)
    k = torch.from_numpy(api.wave_numbers(api.channelized_frequencies(F_SHARD))).to(dev)
    dirs = torch.from_numpy(api.tracker_window_directions(TR_L0, TR_M0, rate_l, rate_m, T, TR_S)).to(dev)
    d = api.Dimensions(T, F_SHARD, N_ANT, 1)
    mine = torch.empty_like(inten)
    integ = torch.empty(api.tracker_window_count(T, TR_S) * F_SHARD, dtype=torch.float32, device=dev)
    api.tracker(None, api.TrackerMode.Streaming, volt, pos, k, dirs, mine, integ, d, TR_S)
    torch.cuda.synchronize()
    ref = out_r.double()
    rel = ((mine.double() - ref).abs() / (1e-3 + ref.abs())).max().item()
    in_bytes = T * F_SHARD * N_ANT
    return {"kernel": "reference tracker_v5_kernel<64,8> via cuda_beam_tracker_v5_device_resident "
                      "(reference sources, nvcc sm_100a), per-spectrum output",
            "ms_per_step": ms, "value": T * F_SHARD / (ms / 1e3), "steps": steps,
            "achieved_gbs": (in_bytes + T * F_SHARD * 4) / (ms / 1e3) / 1e9,
            "b200_per_spectrum_speedup": ms / b200_ps_ms,
            "max_diff_vs_b200_over_1e-3_plus_abs": rel,
            "compared_on": "reference default geometry, same voltages and trajectory"}


def tracker_cpu_baseline(v: np.ndarray, budget_s: float):
    """beam_tracker_opt_v2 (the reference's OpenMP tracker, all host threads)
    on whole 1024-spectrum windows.  The reference API hard-codes its own
    default geometry, so the timed work matches but the steering geometry is
    the reference's (the oracle port is used when the reference core is
    absent)."""
    from oracle import loader as orc
    kind = "reference" if orc.reference_available() else "port"
    threads = host_threads()
    T = v.shape[0]
    done = 0
    vc = np.ascontiguousarray(v)
    with orc.perf_build() if kind == "reference" else _nullcontext():
        t_start = time.perf_counter()
        while True:
            if kind == "reference":
                orc.reference_perf().ref_set_threads(threads)
                orc.ref_tracker(vc, T, F_SHARD, N_ANT, 0.1, -0.05, 0.0, 0.0, TR_S, variant=1)
            else:
                from beamform_project_b200 import api
                pos, freq = api.default_positions(N_ANT), api.channelized_frequencies(F_SHARD)
                dirs = api.tracker_window_directions(0.1, -0.05, 0.0, 0.0, T, TR_S)
                orc.tracker(v, orc.tracker_weights(dirs, pos, freq), T, F_SHARD, N_ANT, TR_S)
            done += T
            if time.perf_counter() - t_start > budget_s:
                break
        el = time.perf_counter() - t_start
    return {"value": done * F_SHARD / el, "unit": "beam-samples/s",
            "cores": threads if kind == "reference" else 1, "kind": kind,
            "sample": f"{done // TR_S} windows of {TR_S} spectra x {F_SHARD} channels x {N_ANT} antennas "
                      f"(beam_tracker_opt_v2, OpenMP), {el:.1f} s",
            "build": orc.reference_perf_flags() if kind == "reference" else "oracle port",
            "host": host_cpu_info()}


def run_tracker_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import loader as orc
    from beamform_project_b200.api import generator_scale
    pos, freq, dirs, mu, _ = tracker_inputs()
    n_win = 16
    v = orc.generate_voltage(SEED + 77, 0, n_win * TR_S, F_SHARD, N_ANT, generator_scale(TR_SIGMA),
                             mu[:n_win], TR_S)
    times = []
    base = None
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        base = tracker_cpu_baseline(v, budget_s=0.0)
        if i >= args.warmup:
            times.append(time.perf_counter() - t)
    value = n_win * TR_S * F_SHARD / statistics.mean(times)
    base["value"] = value
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "beam-samples/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "impl": "reference",
        "data": "synthetic (same seeded voltages, first 16 windows)",
        "config": {"workload": "tracker: A=64 (2x32), F=336, T=262144, window 1024 (W=256)",
                   "sample": f"{n_win} windows x {TR_S} spectra per step"},
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "beam-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------------------
# DOA workload: A=64 (2 x 32), F=336 (400-600 MHz), blocks of K=4096 spectra,
# 16 blocks, forgetting 0.9; noise sigma=2 plus two coherent sources 0.7
# beamwidth apart at SNR 2 and a 50 %-correlated multipath copy; 8-element
# smoothing, Bartlett and Capon (load 1e-3 tr/M, FP64 Cholesky) on a
# 1801-point grid with parabolic peak refinement
# --------------------------------------------------------------------------
DOA_K = 4096
DOA_BLOCKS = 16
DOA_SIGMA = 2.0
DOA_SNR = 2.0
DOA_SUB = 8
DOA_GRID = (-0.9, 0.001, 1801)
DOA_EPOCH = 64   # source waveforms change every 64 spectra


def doa_inputs(T: int):
    pos, freq_full, _ = workload_geometry()
    freq = np.ascontiguousarray(freq_full[:F_SHARD])
    k = 2.0 * math.pi * freq.astype(np.float64) / C_LIGHT
    # beamwidth of the 8-element sub-array at the band centre: lambda / aperture
    bw = (C_LIGHT / float(freq.mean())) / (DOA_SUB * float(pos[1, 0] - pos[0, 0]))
    l1, l2, l3 = -0.35 * bw, 0.35 * bw, 0.5
    amp = DOA_SIGMA * math.sqrt(DOA_SNR)
    U = T // DOA_EPOCH
    rng = np.random.default_rng(SEED + 4)
    g1 = (rng.normal(size=(U, F_SHARD)) + 1j * rng.normal(size=(U, F_SHARD))) / math.sqrt(2)
    g3 = (rng.normal(size=(U, F_SHARD)) + 1j * rng.normal(size=(U, F_SHARD))) / math.sqrt(2)
    gm = 0.5 * g1 + math.sqrt(0.75) * g3
    mu = np.zeros((U, F_SHARD, N_ANT), np.complex128)
    for l, g, ph in ((l1, g1, 0.0), (l2, g1, 1.1), (l3, gm, 0.0)):
        st = np.exp(-1j * k[:, None] * (pos[:, 0].astype(np.float64) * l)[None, :])  # [F][A]
        mu += amp * np.exp(1j * ph) * g[:, :, None] * st[None]
    mu32 = np.stack([mu.real, mu.imag], -1).astype(np.float32)
    return pos, freq, k, mu32, (l1, l2, l3)


def run_doa(args, emit: bool = True):
    import torch
    from beamform_project_b200 import api, native
    if args.impl == "reference":
        return run_doa_reference(args)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    T = DOA_K * DOA_BLOCKS
    pos, freq, k, mu, truth = doa_inputs(T)
    d = api.Dimensions(T, F_SHARD, N_ANT, 1)
    volt = torch.empty(T * F_SHARD * N_ANT, dtype=torch.uint8, device=dev)
    api.generate_voltage(None, SEED + 5, 0, DOA_SIGMA, torch.from_numpy(mu).to(dev), DOA_EPOCH, volt, d)
    l0, dl, n = DOA_GRID
    cov = torch.empty(DOA_BLOCKS * F_SHARD * N_ANT * N_ANT * 2, dtype=torch.int32, device=dev)
    bart = torch.empty(DOA_BLOCKS * n, dtype=torch.float64, device=dev)
    cap = torch.empty_like(bart)
    lest = torch.empty(2 * DOA_BLOCKS, dtype=torch.float64, device=dev)
    ws = torch.empty(api.doa_workspace_bytes(d, DOA_K, DOA_SUB), dtype=torch.uint8, device=dev)
    pos_d = torch.from_numpy(np.ascontiguousarray(pos[:DOA_SUB])).to(dev)
    k_d = torch.from_numpy(k).to(dev)
    cov_ev, scan_ev = [], []

    def step(record=False):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if record else None
        if record:
            e[0].record(stream)
        api.doa_covariance_i32(None, volt, cov, d, DOA_K)
        if record:
            e[1].record(stream)
        api.doa_scan(None, cov, pos_d, k_d, d, DOA_K, DOA_SUB, 0.9, 1e-3, l0, dl, n, 0.0, bart, cap, lest, ws)
        if record:
            e[2].record(stream)
            cov_ev.append((e[0], e[1]))
            scan_ev.append((e[1], e[2]))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert native.take_device_error() == 0
    steps = max(1, min(args.steps, 50))
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for _ in range(steps):
            step(record=True)
        t1.record(stream)
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    cov_ms = statistics.mean(a.elapsed_time(b) for a, b in cov_ev)
    scan_ms = statistics.mean(a.elapsed_time(b) for a, b in scan_ev)
    # end to end: pinned host voltage in, spectra and estimates out
    host_v = torch.empty(volt.numel(), dtype=torch.uint8, pin_memory=True)
    host_v.copy_(volt)
    host_b = torch.empty(bart.numel(), dtype=torch.float64, pin_memory=True)
    host_c = torch.empty_like(host_b, pin_memory=True)
    host_l = torch.empty(lest.numel(), dtype=torch.float64, pin_memory=True)
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(max(1, args.e2e_steps)):
        volt.copy_(host_v, non_blocking=True)
        step()
        host_b.copy_(bart, non_blocking=True)
        host_c.copy_(cap, non_blocking=True)
        host_l.copy_(lest, non_blocking=True)
    a1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = a0.elapsed_time(a1) / max(1, args.e2e_steps)
    samples = T * F_SHARD
    in_bytes = T * F_SHARD * N_ANT
    alg_bytes = in_bytes + DOA_BLOCKS * F_SHARD * N_ANT * N_ANT * 8
    _, _, hbm_gbs, peak_src = measured_peaks()
    achieved = alg_bytes / (cov_ms / 1e3) / 1e9
    est = host_l.numpy().reshape(DOA_BLOCKS, 2)
    line = {
        "metric": METRIC, "value": samples / (ms / 1e3), "unit": "beam-samples/s", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int4xint8->int32, fp64",
        "data": "synthetic (seeded on-device generator; coherent pair + multipath)",
        "config": {"workload": "DOA: A=64 (2x32), F=336, K=4096 x 16 blocks, forgetting 0.9, 8-element "
                               "smoothing, Bartlett + Capon on 1801 points (one direction stream: B=1)",
                   "l2": "inputs (1.41 GB voltage) exceed L2; no flush",
                   "sources_l": [round(x, 4) for x in truth]},
        "roofline": {"bound": "hbm", "kernel": "doa_cov_kernel", "achieved": round(achieved, 1),
                     "peak": hbm_gbs, "unit": "GB/s", "frac": round(achieved / hbm_gbs, 4),
                     "traffic": round(NCU_TRAFFIC["doa"]),
                     "peak_source": peak_src + " (copy bandwidth)", "kernel_ms": round(cov_ms, 4),
                     "algorithmic_bytes_per_launch": alg_bytes},
        "scan_ms": scan_ms,
        "l_est_last_block": {"bartlett": float(est[-1, 0]), "capon": float(est[-1, 1])},
        "e2e": {"value": samples / (e2e_ms / 1e3), "unit": "beam-samples/s", "h2d_bytes_per_step": host_v.numel(),
                "d2h_bytes_per_step": (host_b.numel() + host_c.numel() + host_l.numel()) * 8, "ms_per_step": e2e_ms},
        "gpu_launches": 4 * steps,
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = doa_cpu_baseline(volt[: 2 * DOA_K * F_SHARD * N_ANT].cpu().numpy()
                                                .reshape(-1, F_SHARD, N_ANT), pos, freq, args.cpu_seconds)
    if emit:
        print(json.dumps(line), flush=True)
    return line


def doa_cpu_baseline(v: np.ndarray, pos, freq, budget_s: float):
    """CpuOptBeamTracker (Capon, coarse grid 16, 2 refinements, 8-element
    smoothing, forgetting 0.9; OpenMP over frequencies) on whole blocks."""
    from oracle import loader as orc
    threads = host_threads()
    T = v.shape[0]
    done = 0
    kind = "reference" if orc.reference_available() else "port"
    with orc.perf_build() if kind == "reference" else _nullcontext():
        t0 = time.perf_counter()
        while True:
            if kind == "reference":
                orc.reference_perf().ref_set_threads(threads)
                orc.ref_doa_directions(v, pos, freq, DOA_K, capon=True, G=16, levels=2, fov_l=0.4, fov_m=0.05,
                                       subarray=DOA_SUB, lam=0.9, load=1e-3, l0=0.0, m0=0.0)
            else:
                R = orc.covariance_blocks(v, DOA_K)
                orc.doa_scan(R, DOA_K, DOA_SUB, 0.9, 1e-3, pos[:DOA_SUB],
                             2 * math.pi * freq.astype(np.float64) / C_LIGHT, *DOA_GRID)
            done += T
            if time.perf_counter() - t0 > budget_s:
                break
        el = time.perf_counter() - t0
    return {"value": done * F_SHARD / el, "unit": "beam-samples/s", "cores": threads if kind == "reference" else 1,
            "kind": kind, "sample": f"{done // DOA_K} blocks of {DOA_K} spectra x {F_SHARD} channels "
                                    f"(CpuOptBeamTracker Capon, G=16, 2 refinements), {el:.1f} s",
            "build": orc.reference_perf_flags() if kind == "reference" else "oracle port",
            "host": host_cpu_info()}


def run_doa_split(args):
    """The DOA step of one job split across the GPUs by channel (the path's one
    exchange step): each rank takes a contiguous slice of the 336 channels
    (covariance, fold and scan of the slice), one NCCL all-reduce sums the
    partial spectra (2 x 16 x 1801 doubles), then the peak search.  Strong
    scaling: the whole job's samples over the max-over-ranks step time."""
    import datetime
    import torch
    from beamform_project_b200 import api, native
    from beamform_project_b200.doa_channels import channel_slice, scan_slice
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    T = DOA_K * DOA_BLOCKS
    pos, freq, k, mu, truth = doa_inputs(T)
    d = api.Dimensions(T, F_SHARD, N_ANT, 1)
    volt = torch.empty(T * F_SHARD * N_ANT, dtype=torch.uint8, device=dev)
    api.generate_voltage(None, SEED + 5, 0, DOA_SIGMA, torch.from_numpy(mu).to(dev), DOA_EPOCH, volt, d)
    sl = channel_slice(F_SHARD, rank, world)
    vs = volt.view(T, F_SHARD, N_ANT)[:, sl.start:sl.stop].contiguous()
    del volt
    pos_d = torch.from_numpy(np.ascontiguousarray(pos[:DOA_SUB])).to(dev)
    k_d = torch.from_numpy(np.ascontiguousarray(k[sl.start:sl.stop])).to(dev)
    l0, dl, n = DOA_GRID

    def step():
        return scan_slice(vs, pos_d, k_d, T, N_ANT, DOA_K, DOA_SUB, 0.9, 1e-3, l0, dl, n, 0.0)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if native.take_device_error() != 0:
        raise RuntimeError("device error word set")
    steps = max(1, min(args.steps, 50))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        spectra, l_est = step()
    t1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = t0.elapsed_time(t1) / steps
    if dist:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    est = l_est.cpu().numpy()
    line = {
        "metric": METRIC, "value": T * F_SHARD / (ms / 1e3), "unit": "beam-samples/s", "n_gpus": world,
        "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "int4xint8->int32, fp64",
        "data": "synthetic (seeded on-device generator; coherent pair + multipath)",
        "config": {"workload": "DOA, one job split by channel: A=64 (2x32), F=336, K=4096 x 16 blocks, "
                               "Bartlett + Capon on 1801 points",
                   "parallelism": f"channel split x{world} (NCCL all-reduce of the partial spectra)",
                   "channels_on_rank0": len(channel_slice(F_SHARD, 0, world))},
        "l_est_last_block": {"bartlett": float(est[-1, 0]), "capon": float(est[-1, 1])},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_doa_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import loader as orc
    from beamform_project_b200.api import generator_scale
    T = 2 * DOA_K
    pos, freq, k, mu, _ = doa_inputs(DOA_K * DOA_BLOCKS)
    v = orc.generate_voltage(SEED + 5, 0, T, F_SHARD, N_ANT, generator_scale(DOA_SIGMA),
                             mu[: T // DOA_EPOCH], DOA_EPOCH)
    times = []
    base = None
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        base = doa_cpu_baseline(v, pos, freq, budget_s=0.0)
        if i >= args.warmup:
            times.append(time.perf_counter() - t)
    value = T * F_SHARD / statistics.mean(times)
    base["value"] = value
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "beam-samples/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "impl": "reference",
        "data": "synthetic (same seeded voltages, first 2 blocks)",
        "config": {"workload": "DOA: A=64 (2x32), F=336, K=4096 x 16 blocks", "sample": "2 blocks per step"},
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "beam-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------------------
# served mix: Poisson arrivals, HBM-budget admission, one graph per window
# --------------------------------------------------------------------------

SERVE_SEED = 1
SERVE_RATE = 200.0
SERVE_POOL = 20480
SERVE_SIGMA = 2.0


def serve_jobs(seconds: float):
    from beamform_project_b200 import serve
    return serve.poisson_mix(seed=SERVE_SEED, rate_hz=SERVE_RATE, duration_s=seconds, pool_spectra=SERVE_POOL)


def serve_cpu_baseline(jobs, budget_s: float):
    """The reference CPU path per job class, timed on small samples of each
    class on the host cores and combined over the mix's beam-samples:
    grid jobs (A, B) by the reference chain beamform -> integrate (S) ->
    quantize on one 320-spectrum window of 336 channels (windows on
    independent threads); tracker jobs (A, S) by beam_tracker_opt_v2
    (OpenMP) once per source on 320 x k spectra."""
    from oracle import loader as orc
    from beamform_project_b200 import api, serve
    kind = "reference" if orc.reference_available() else "port"
    threads = host_threads()
    classes = {}
    for j in jobs:
        key = (j.kind, j.n_ant, j.n_beams if j.kind == serve.GRID else 1, j.integration_spectra)
        classes[key] = classes.get(key, 0) + j.beam_samples()
    per = max(0.2, budget_s / max(1, len(classes)))
    rng = np.random.default_rng(0)
    rates = {}
    with orc.perf_build() if kind == "reference" else _nullcontext():
        _serve_class_rates(classes, rates, per, rng, kind, threads)
    total = sum(classes.values())
    cpu_s = sum(classes[k] / rates[k] for k in classes)
    return {"value": total / cpu_s, "unit": "beam-samples/s", "cores": threads, "kind": kind,
            "sample": f"{len(classes)} job classes (grid A x B x S, tracker A x S), about {per:.1f} s each, "
                      f"combined over the mix's {total:.3e} beam-samples",
            "build": orc.reference_perf_flags() if kind == "reference" else "oracle port",
            "host": host_cpu_info()}


def _serve_class_rates(classes, rates, per, rng, kind, threads):
    from oracle import loader as orc
    from beamform_project_b200 import api, serve
    for key in sorted(classes):
        k, A, B, S = key
        v = rng.integers(0, 256, size=(320 * 4, F_SHARD, A), dtype=np.uint8)
        t0 = time.perf_counter()
        n = 0
        if k == serve.GRID:
            w = np.ascontiguousarray(orc.generate_weights(serve.array_positions(A),
                                                          serve.band_frequencies(F_SHARD),
                                                          np.tile(np.array([[0, 0, 1]], np.float32), (B, 1))))

            def one(i):
                vv = np.ascontiguousarray(v[320 * (i % 4):320 * (i % 4 + 1)])
                if kind == "reference":
                    I = orc.ref_beamform(vv, w, 320, F_SHARD, A, B)
                    integ = orc.ref_integrate(I, 320, F_SHARD, A, B, S)
                    orc.ref_quantize(integ, 320 // S, F_SHARD, A, B)
                else:
                    integ = orc.beamform_integrated(vv, w, 320, F_SHARD, A, B, S)
                    orc.quantize(integ, 320 // S, F_SHARD, B)
            with ThreadPoolExecutor(max_workers=threads) as ex:
                while True:
                    list(ex.map(one, range(threads)))
                    n += threads * 320 * F_SHARD * B
                    if time.perf_counter() - t0 > per:
                        break
        else:
            while True:
                if kind == "reference":
                    orc.reference_perf().ref_set_threads(threads)
                    orc.ref_tracker(v, len(v), F_SHARD, A, 0.1, -0.05, 0.0, 0.0, S, variant=1)
                else:
                    pos, freq = api.default_positions(A), api.channelized_frequencies(F_SHARD)
                    dirs = api.tracker_window_directions(0.1, -0.05, 0.0, 0.0, len(v), S)
                    orc.tracker(v, orc.tracker_weights(dirs, pos, freq), len(v), F_SHARD, A, S)
                n += len(v) * F_SHARD
                if time.perf_counter() - t0 > per:
                    break
        rates[key] = n / (time.perf_counter() - t0)


def serve_latency(jobs, run, infos, step_ms, step_offset: int) -> dict:
    """Real-time view of a served stream.  realtime_factor: the stream's
    length (first arrival to the end of the last job's data, as if every job
    ran from its arrival) over the device time of all its windows; at or above
    1 the GPU keeps up with the stream.  The steps are replayed on the stream
    clock (serve.realtime_replay): window latency is a step's finish minus the
    time its data was complete, admission wait a job's first window minus its
    arrival, completion latency its last window's finish minus the end of its
    data."""
    from beamform_project_b200 import serve
    k = run.get("windows_per_step", 1)
    rep = serve.realtime_replay(step_ms, run["step_windows"], windows_per_step=k)
    w_s = 320 * serve.SPECTRUM_S
    t0 = min(j.arrival_s for j in jobs)
    t1 = max(j.arrival_s + j.n_spectra * serve.SPECTRUM_S for j in jobs)
    waits, done_lat = [], []
    for j, jid in zip(jobs, run["job_ids"]):
        info = infos.get(jid)
        if info is None or info["admit_step"] is None or info["last_step"] is None:
            continue
        a, b = info["admit_step"] - step_offset, info["last_step"] - step_offset
        if a < 0 or b >= len(rep["end_s"]):
            continue
        waits.append(rep["ready_s"][a] - k * w_s - j.arrival_s)
        done_lat.append(rep["end_s"][b] - (j.arrival_s + j.n_spectra * serve.SPECTRUM_S))
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None  # noqa: E731
    lat_ms = rep["latency_s"] * 1e3
    return {"realtime_factor": (t1 - t0) / rep["device_s"] if rep["device_s"] else None,
            "stream_s": t1 - t0, "device_s": rep["device_s"],
            "replayed_window_latency_ms_p50": pct(lat_ms, 50), "replayed_window_latency_ms_p99": pct(lat_ms, 99),
            "admission_wait_s_p50": pct(waits, 50), "admission_wait_s_p99": pct(waits, 99),
            "completion_latency_s_p50": pct(done_lat, 50), "completion_latency_s_p99": pct(done_lat, 99),
            "virtual_stream_s": len(run["step_windows"]) and (run["step_windows"][-1] + k) * w_s,
            "windows_per_step": k}


def run_serve(args, emit: bool = True):
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        jobs = serve_jobs(args.serve_seconds)
        t = time.perf_counter()
        base = serve_cpu_baseline(jobs, budget_s=args.cpu_seconds)
        el = time.perf_counter() - t
        print(json.dumps({
            "metric": METRIC, "value": base["value"], "unit": "beam-samples/s", "n_gpus": 0, "steps": 1,
            "warmup": 0, "ms_per_step": el * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "impl": "reference",
            "data": "synthetic (served mix classes; random int4 samples)",
            "config": {"workload": f"served mix: Poisson {SERVE_RATE:g} jobs/s for {args.serve_seconds:g} s, "
                                   f"seed {SERVE_SEED}", "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "beam-samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }), flush=True)
        return
    import torch
    from beamform_project_b200 import native, serve
    from beamform_project_b200.replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    reps = Replicas("nccl", timeout_s=600)
    world, rank = reps.world, reps.rank
    jobs = serve_jobs(args.serve_seconds)
    budget = int(args.serve_budget_gb * 1e9)
    srv = serve.Server(budget, max_jobs=args.serve_max_jobs, pool_spectra=SERVE_POOL, pool_seed=SERVE_SEED + rank,
                       pool_sigma=SERVE_SIGMA, window_budget_us=args.serve_window_us)
    stream = torch.cuda.ExternalStream(srv.stream_handle())
    # warm-up: one job of every class of the mix, served to completion
    seen, warm = set(), []
    for j in jobs:
        key = (j.kind, j.n_ant, j.n_beams, j.integration_spectra)
        if key not in seen:
            seen.add(key)
            w = serve.JobSpec(**{**j.__dict__, "n_spectra": 320 * max(1, args.warmup), "_keep": []})
            warm.append(w)
    serve.run_stream(srv, warm)
    srv.sync()
    st0 = srv.stats()
    n_warm_steps = len(srv.step_times())

    reps.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    infos = {}

    def record_info(jid):
        infos[jid] = srv.job_info(jid)
    with ClockSampler(local) as clocks:
        e0.record(stream)
        r = serve.run_stream(srv, jobs, on_done=record_info)
        e1.record(stream)
        srv.sync()
        torch.cuda.synchronize()
    el_ms = e0.elapsed_time(e1)
    assert native.take_device_error() == 0
    st = srv.stats()
    times = srv.step_times()[n_warm_steps:]
    latency = serve_latency(jobs, r, infos, times, n_warm_steps)
    samples = st["beam_samples"] - st0["beam_samples"]
    steps = st["steps"] - st0["steps"]
    el_ms = reps.max(el_ms)
    value = reps.sum(samples) / (el_ms / 1e3)

    # algorithmic bytes: every job window reads its voltage once and writes its outputs
    vbytes = 0
    obytes = 0
    flops = 0
    for j in jobs:
        ch = j.n_shards * F_SHARD
        vbytes += j.n_spectra * ch * j.n_ant
        W = j.n_spectra // j.integration_spectra
        obytes += W * ch * j.n_beams * (5 if j.kind == serve.GRID else 4)
        flops += 8 * j.n_spectra * ch * j.n_ant * j.n_beams
    _, peak_tflops, hbm_gbs, peak_src = measured_peaks()
    achieved = (vbytes + obytes) / (el_ms / 1e3) / 1e9

    # e2e: a shorter stream through the same public calls, with every finished
    # job's results copied to pinned host memory inside the timed region
    e2e = None
    if args.serve_e2e_seconds > 0:
        ejobs = serve_jobs(args.serve_e2e_seconds)
        d2h = [0]

        def fetch(jid):
            integ, codes, params = srv.result(jid, floats=False)
            d2h[0] += sum(a.nbytes for a in (integ, codes, params) if a is not None)
        s0 = srv.stats()["beam_samples"]
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e2.record(stream)
        serve.run_stream(srv, ejobs, on_done=fetch)
        srv.sync()
        e3.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        es = srv.stats()["beam_samples"] - s0
        h2d = sum(12 * j.n_ant + 4 * j.n_shards * F_SHARD + 16 * j.n_beams for j in ejobs)
        e2e = {"value": es * world / wall, "unit": "beam-samples/s",
               "h2d_bytes_per_step": int(h2d / max(1, len(ejobs))),
               "d2h_bytes_per_step": int(d2h[0] / max(1, len(ejobs))),
               "step": "one job (inputs uploaded at admission, results read back when done)",
               "wall_s": wall, "seconds_of_arrivals": args.serve_e2e_seconds}
    srv.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "beam-samples/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": el_ms / max(1, steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int4xfp16->fp32",
            "data": "synthetic (device voltage pools from the seeded generator; seeded job stream)",
            "config": {"workload": f"served mix: Poisson {SERVE_RATE:g} jobs/s for {args.serve_seconds:g} s "
                                   f"(seed {SERVE_SEED}), A in {{32,64}}, 1-4 shards of 336, grid B in "
                                   f"{{1,8,32,128}} or tracker 1-16 sources, 0.1-2 s at 2.56 us/spectrum, "
                                   f"S in {{10,320}}, {args.serve_budget_gb:g} GB admission budget, "
                                   f"320-spectrum served windows, window-time admission bound "
                                   f"{args.serve_window_us:g} us",
                       "jobs": len(jobs), "parallelism": f"independent replicas x{world}",
                       "l2": "voltage pools (2.6 GB) exceed L2; no flush"},
            "serve": {"window_ms_p50": float(np.percentile(times, 50)) if len(times) else None,
                      "window_ms_p99": float(np.percentile(times, 99)) if len(times) else None,
                      "window_ms_max": float(times.max()) if len(times) else None,
                      "window_budget_ms": 0.5, "windows_over_budget": int((times > 0.5).sum()),
                      "job_windows": st["job_windows"] - st0["job_windows"],
                      "jobs_done": st["jobs_done"] - st0["jobs_done"],
                      "arena_peak_gb": st["arena_bytes_peak"] / 1e9, "graph_captures": st["graph_captures"],
                      "mean_live_jobs": (st["job_windows"] - st0["job_windows"]) / max(1, steps),
                      "gpu_busy_frac": float(times.sum()) / el_ms if el_ms else None,
                      "window_bound_us": args.serve_window_us, **latency},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_gbs, "unit": "GB/s",
                         "frac": round(achieved / hbm_gbs, 4), "traffic": None,
                         "peak_source": peak_src + " (copy bandwidth)",
                         "algorithmic_bytes": vbytes + obytes,
                         "tensor_tflops_algorithmic": round(flops / (el_ms / 1e3) / 1e12, 2),
                         "note": "aggregate over the mix; the tensor-bound grid classes sit under the "
                                 "tensor roofline instead"},
            "e2e": e2e,
            "gpu_launches": int(st["kernel_launches"] - st0["kernel_launches"]),
            "clocks": clocks.summary(),
        }
        if args.serve_throughput_k > 1:
            line["serve"]["throughput_mode"] = serve_throughput_mode(args, jobs, budget, rank)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = serve_cpu_baseline(jobs, budget_s=args.cpu_seconds)
        if emit:
            print(json.dumps(line), flush=True)
    reps.close()
    return line if rank == 0 else None


def serve_throughput_mode(args, jobs, budget: int, rank: int) -> dict:
    """The same stream with each step serving args.serve_throughput_k windows
    per live job and admission by memory and slots only: each grid channel's
    weights load once per k windows and a step's fixed costs spread over k
    windows, at the price of latency (the setting for a server that has
    fallen behind its stream)."""
    import torch
    from beamform_project_b200 import native, serve
    k = args.serve_throughput_k
    srv = serve.Server(budget, max_jobs=args.serve_max_jobs, pool_spectra=SERVE_POOL, pool_seed=SERVE_SEED + rank,
                       pool_sigma=SERVE_SIGMA, window_budget_us=0.0, windows_per_step=k)
    stream = torch.cuda.ExternalStream(srv.stream_handle())
    seen, warm = set(), []
    for j in jobs:
        key = (j.kind, j.n_ant, j.n_beams, j.integration_spectra)
        if key not in seen:
            seen.add(key)
            warm.append(serve.JobSpec(**{**j.__dict__, "n_spectra": 320 * k, "_keep": []}))
    serve.run_stream(srv, warm)
    srv.sync()
    st0 = srv.stats()
    n_warm = len(srv.step_times())
    infos = {}

    def record_info(jid):
        infos[jid] = srv.job_info(jid)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r = serve.run_stream(srv, jobs, on_done=record_info)
    e1.record(stream)
    srv.sync()
    torch.cuda.synchronize()
    el_ms = e0.elapsed_time(e1)
    assert native.take_device_error() == 0
    st = srv.stats()
    times = srv.step_times()[n_warm:]
    lat = serve_latency(jobs, r, infos, times, n_warm)
    srv.close()
    steps = st["steps"] - st0["steps"]
    return {"windows_per_step": k, "value": (st["beam_samples"] - st0["beam_samples"]) / (el_ms / 1e3),
            "unit": "beam-samples/s", "steps": steps, "step_ms_p50": float(np.percentile(times, 50)),
            "step_ms_p99": float(np.percentile(times, 99)),
            "mean_live_jobs": (st["job_windows"] - st0["job_windows"]) / max(1, steps) / k,
            "arena_peak_gb": st["arena_bytes_peak"] / 1e9, **lat}



def run_reference(args):
    """The reference's own CPU implementation on the host cores, same metric."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pos, freq, dirs = workload_geometry()
    w_host = workload_weights(pos, freq, dirs)
    beam, mu_host = workload_source(pos, freq, dirs)
    from oracle import loader as orc
    from beamform_project_b200.api import generator_scale
    # a bounded slice of the same seeded voltages (the oracle generator is
    # byte-identical to the device generator): one window per host thread
    threads = os.cpu_count() or 1
    n_win = min(threads, T_SPECTRA // S_INT)
    v0 = orc.generate_voltage(SEED, 0, n_win * S_INT, F_SHARD, N_ANT, generator_scale(SIGMA),
                              mu_host[0][None], T_SPECTRA)
    vfull = np.zeros((T_SPECTRA, F_SHARD, N_ANT), np.uint8)
    vfull[:n_win * S_INT] = v0
    times = []
    base = None
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        base = cpu_baseline(vfull[:n_win * S_INT], w_host[0], budget_s=0.0, threads=threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t)
    value = base["value"]
    per_step_samples = n_win * S_INT * F_SHARD * N_BEAMS
    value = per_step_samples / statistics.mean(times)
    base["value"] = value
    line = {"metric": METRIC, "value": value, "unit": "beam-samples/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "impl": "reference",
            "data": "synthetic (same seeded voltages, first windows of shard 0)",
            "config": {"workload": "full-band split-precision grid: A=64 (2x32), F=672 (2 shards x 336), "
                                   "T=32768, B=128 (16x8), S=320, float32 + int8 chunk codes",
                       "sample": f"{n_win} windows x 320 spectra of shard 0 per step"},
            "cpu_baseline": base,
            "e2e": {"value": value, "unit": "beam-samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# profiling workloads: one grid shape on random inputs, one served job class
# --------------------------------------------------------------------------

def run_shape(args):
    """The split-precision grid path on one shard of seeded random voltages
    and unit-modulus weights of a given shape (--shape-ant, --shape-beams,
    --shape-spectra, T = --t-spectra), timed with CUDA events, beside the
    reference-order kernel on the same inputs."""
    import torch
    from beamform_project_b200 import api, native
    T, F, A, B, S = args.t_spectra, F_SHARD, args.shape_ant, args.shape_beams, args.shape_spectra
    d = api.Dimensions(T, F, A, B)
    W = -(-T // S)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    volt = torch.randint(0, 256, (T * F * A,), dtype=torch.uint8, device="cuda", generator=g)
    ph = torch.rand(B * F * A, device="cuda", generator=g) * (2 * math.pi)
    w = torch.stack([torch.cos(ph), torch.sin(ph)], -1).contiguous()
    split = torch.empty(api.split_weight_bytes(d), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, w, split, d)
    out = torch.empty(W * F * B, dtype=torch.float32, device="cuda")

    def step():
        api.grid_tensor_integrated(None, volt, split, out, None, None, d, S)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for e0, e1 in ev:
        e0.record()
        step()
        e1.record()
    torch.cuda.synchronize()
    ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in ev)
    line = {"workload": f"grid shape A={A} B={B} S={S} T={T} F={F} (one shard, random inputs)",
            "kernel_ms": ms, "algorithmic_tflops": (8.0 * T * F * A * B + 3.0 * T * F * B) / (ms / 1e3) / 1e12}
    if args.plain_steps > 0:
        ref = torch.empty_like(out)
        api.launch_packed_integrated_beamformer(api.CudaBeamformerKernel.Direct, None, volt, w, ref, d, S)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        api.launch_packed_integrated_beamformer(api.CudaBeamformerKernel.Direct, None, volt, w, ref, d, S)
        e1.record()
        torch.cuda.synchronize()
        r, o = ref.double(), out.double()
        line["plain_dropin_ms"] = e0.elapsed_time(e1)
        line["max_diff_vs_plain_over_1e-3_plus_abs"] = float(((o - r).abs() / (1e-3 + r.abs())).max())
    if native.take_device_error() != 0:
        raise RuntimeError("device error word set")
    print(json.dumps(line), flush=True)


def run_serve_job(args):
    """One served job of a class alone (--job-kind grid or tracker, --shape-ant,
    --shape-beams (sources), --shape-spectra, --job-shards) in a small
    server (2 GB arena, 1920-spectrum pool): the median device time of its
    windows."""
    import numpy as np
    import torch  # noqa: F401  (CUDA context for the server)
    from beamform_project_b200 import serve
    A, B, S, ns = args.shape_ant, args.shape_beams, args.shape_spectra, args.job_shards
    pos = serve.array_positions(A)
    freq = serve.band_frequencies(ns * F_SHARD)
    rng = np.random.default_rng(1)
    if args.job_kind == "tracker":
        tr = np.zeros((B, 4), np.float32)
        tr[:, :2] = rng.uniform(-0.3, 0.3, size=(B, 2))
        tr[:, 2:] = 1e-8
        spec = serve.JobSpec(serve.TRACKER, A, ns, B, 320 * 5, S, pos, freq, trajectories=tr)
    else:
        lm = rng.uniform(-0.3, 0.3, size=(B, 2)).astype(np.float32)
        n = np.sqrt(1 - (lm ** 2).sum(1)).astype(np.float32)
        spec = serve.JobSpec(serve.GRID, A, ns, B, 320 * 5, S, pos, freq, directions=np.c_[lm, n].astype(np.float32))
    srv = serve.Server(int(2e9), max_jobs=8, pool_spectra=1920, pool_seed=1, pool_sigma=2.0)
    try:
        srv.submit(spec)
        while srv.step() > 0:
            pass
        srv.sync()
        t = srv.step_times()
    finally:
        srv.close()
    print(json.dumps({"workload": f"served {args.job_kind} job alone: A={A} B={B} S={S} shards={ns}",
                      "windows": len(t), "window_ms_median": float(np.median(t[1:])) if len(t) > 1 else None}),
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="grid", choices=["grid", "tracker", "doa", "doa-split", "serve", "shape", "serve-job"],
                    help="doa-split: one DOA job split across the GPUs by channel (strong scaling); shape / "
                         "serve-job: profiling workloads (one grid shape on random inputs; one served job class alone)")
    ap.add_argument("--shape-ant", type=int, default=128)
    ap.add_argument("--shape-beams", type=int, default=64)
    ap.add_argument("--shape-spectra", type=int, default=320)
    ap.add_argument("--job-kind", default="tracker", choices=["tracker", "grid"])
    ap.add_argument("--job-shards", type=int, default=4)
    ap.add_argument("--cov-steps", type=int, default=20,
                    help="grid: time the opt-in covariance-form kernel beside the split kernel")
    ap.add_argument("--kernel", default="auto", choices=["auto", "tensor", "tiled", "stream", "exact"],
                    help="grid: auto = the checked covariance form, autotuned; tensor = the split kernel")
    ap.add_argument("--shards", type=int, default=N_SHARDS, choices=[1, 2])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--fused-quant", action="store_true",
                    help="quantize inside the tensor kernel's epilogue (measured slower than the separate kernel)")
    ap.add_argument("--t-spectra", type=int, default=TR_T, help="tracker workload length (profiling)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="steps of the plain drop-in (reference-order) kernel timed beside the tensor path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune", type=int, default=1,
                    help="grid --kernel auto: run the autotuner for the class first (0: the default choice)")
    ap.add_argument("--configs", type=int, default=1,
                    help="grid: also measure the plain-grid, tracker, DOA and served workloads as sub-records")
    ap.add_argument("--config-cpu-seconds", type=float, default=5.0,
                    help="CPU-baseline sample length of each sub-record")
    ap.add_argument("--ref-gpu-steps", type=int, default=3,
                    help="steps of the reference's own CUDA kernels timed beside the B200 path (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="seconds of Poisson arrivals (the full stream is 10)")
    ap.add_argument("--serve-e2e-seconds", type=float, default=0.2)
    ap.add_argument("--serve-window-us", type=float, default=480.0,
                    help="admission bound on the predicted device time of a window (0: memory only)")
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-max-jobs", type=int, default=512)
    ap.add_argument("--serve-throughput-k", type=int, default=8,
                    help="serve: also run the stream with this many windows per step (0 or 1: skip)")
    args = ap.parse_args()
    if args.workload == "shape":
        run_shape(args)
    elif args.workload == "serve-job":
        run_serve_job(args)
    elif args.workload == "doa-split":
        run_doa_split(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "tracker":
        run_tracker(args)
    elif args.workload == "doa":
        run_doa(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
