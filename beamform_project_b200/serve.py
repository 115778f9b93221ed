"""Served, continuously batched mode (bf_serve_* in include/bf_b200.h).

A :class:`Server` owns an HBM arena for per-job state, device voltage pools
(the seeded generator's output standing in for the ingest buffers) and one
CUDA stream.  Jobs are submitted at any time; every :meth:`Server.step`
admits queued jobs first-in first-out while their state fits the arena, then
runs one served window (``window_spectra`` spectra) of every live job as one
CUDA-graph replay.  :func:`poisson_mix` builds the seeded request stream of
the served benchmark (Poisson arrivals; a mix of antenna counts, shards,
beam counts, tracker sources, durations and integration lengths).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import native

GRID, TRACKER = 0, 1
QUEUED, LIVE, RUNNING, DONE, CANCELLED, UNKNOWN = range(6)
SPECTRUM_S = 2.56e-6
C_LIGHT = 299_792_458.0


@dataclass
class JobSpec:
    kind: int
    n_ant: int
    n_shards: int
    n_beams: int                  # grid beams or tracker sources
    n_spectra: int
    integration_spectra: int
    positions: np.ndarray         # [A][3] float32
    frequencies: np.ndarray       # [n_shards * shard_channels] float32
    directions: np.ndarray | None = None     # grid [B][3] float32
    trajectories: np.ndarray | None = None   # tracker [S][4] float32 (l0, m0, dl, dm per spectrum)
    pool_offset: int = 0
    quantize: bool = True
    arrival_s: float = 0.0        # request-stream time (informational)
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> native.ServeJob:
        arrs = [np.ascontiguousarray(self.positions, np.float32),
                np.ascontiguousarray(self.frequencies, np.float32)]
        d = np.ascontiguousarray(self.directions, np.float32) if self.directions is not None else None
        t = np.ascontiguousarray(self.trajectories, np.float32) if self.trajectories is not None else None
        self._keep = [a for a in arrs + [d, t] if a is not None]
        ptr = (lambda a: a.ctypes.data if a is not None else None)
        return native.ServeJob(self.kind, self.n_ant, self.n_shards, self.n_beams, self.n_spectra,
                               self.integration_spectra, self.pool_offset, ptr(arrs[0]), ptr(arrs[1]),
                               ptr(d), ptr(t), int(bool(self.quantize)), 0)

    def beam_samples(self, shard_channels: int = 336) -> int:
        return self.n_spectra * self.n_shards * shard_channels * self.n_beams


class _DeviceArray:
    """__cuda_array_interface__ view of device memory owned by the server."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class Server:
    def __init__(self, hbm_budget_bytes: int, max_jobs: int = 512, window_spectra: int = 320,
                 pool_spectra: int = 20480, shard_channels: int = 336, max_shards: int = 4,
                 pool_seed: int = 1, pool_sigma: float = 2.0, window_budget_us: float = 0.0,
                 host_only: bool = False, windows_per_step: int = 1):
        from .api import generator_scale
        self.config = native.ServeConfig(int(hbm_budget_bytes), int(max_jobs), int(window_spectra),
                                         int(pool_spectra), int(shard_channels), int(max_shards), int(pool_seed),
                                         float(generator_scale(pool_sigma)), float(window_budget_us),
                                         int(windows_per_step))
        self.windows_per_step = max(1, int(windows_per_step))
        self.host_only = host_only
        self._h = C.c_void_p()
        fn = native.lib().bf_serve_create_host_only if host_only else native.lib().bf_serve_create
        native.check(fn(C.byref(self.config), C.byref(self._h)))
        self.specs: dict[int, JobSpec] = {}

    # -- lifetime
    def close(self) -> None:
        if self._h:
            native.check(native.lib().bf_serve_destroy(self._h))
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    # -- requests
    def job_bytes(self, spec: JobSpec) -> int:
        job = spec.to_c()
        return int(native.lib().bf_serve_job_bytes(C.byref(self.config), C.byref(job)))

    def submit(self, spec: JobSpec) -> int:
        job = spec.to_c()
        jid = C.c_uint64(0)
        native.check(native.lib().bf_serve_submit(self._h, C.byref(job), C.byref(jid)))
        self.specs[int(jid.value)] = spec
        return int(jid.value)

    def step(self) -> int:
        n = C.c_uint32(0)
        native.check(native.lib().bf_serve_step(self._h, C.byref(n)))
        return int(n.value)

    def poll(self, job_id: int) -> int:
        st = C.c_int32(0)
        native.check(native.lib().bf_serve_poll(self._h, int(job_id), C.byref(st)))
        return int(st.value)

    def job_info(self, job_id: int) -> dict:
        """Server steps at which the job was submitted, ran its first and its
        last window (None when not reached), and its windows launched."""
        info = native.ServeJobInfo()
        native.check(native.lib().bf_serve_job_info_get(self._h, int(job_id), C.byref(info)))
        none = (1 << 64) - 1
        return {"state": int(info.state), "submit_step": int(info.submit_step),
                "admit_step": None if info.admit_step == none else int(info.admit_step),
                "last_step": None if info.last_step == none else int(info.last_step),
                "windows_launched": int(info.windows_launched)}

    def cancel(self, job_id: int) -> None:
        native.check(native.lib().bf_serve_cancel(self._h, int(job_id)))

    def checkpoint(self, job_id: int) -> bytes:
        """Self-contained image of a job (description, windows served, their
        results); waits for the job's launched windows.  See restore()."""
        n = C.c_uint64(0)
        native.check(native.lib().bf_serve_checkpoint(self._h, int(job_id), None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        native.check(native.lib().bf_serve_checkpoint(self._h, int(job_id), buf, n.value, C.byref(n)))
        return buf.raw[: n.value]

    def restore(self, image: bytes) -> int:
        """Queue the job of a checkpoint image (from a server with the same
        window, shard and pool settings); it resumes at its next window.  Its
        results equal an uninterrupted run's when this server's pool holds the
        same rows as the source's: the image records the pool offset, not the
        pool's contents."""
        jid = C.c_uint64(0)
        buf = C.create_string_buffer(bytes(image), len(image))
        native.check(native.lib().bf_serve_restore(self._h, buf, len(image), C.byref(jid)))
        self.specs[jid.value] = spec_of_checkpoint(image)
        return jid.value

    def release(self, job_id: int) -> None:
        native.check(native.lib().bf_serve_release(self._h, int(job_id)))
        self.specs.pop(int(job_id), None)

    def take_done(self, capacity: int = 4096) -> list[int]:
        """Jobs that became DONE since the last call (a completion queue)."""
        buf = (C.c_uint64 * capacity)()
        n = C.c_uint64(0)
        native.check(native.lib().bf_serve_take_done(self._h, buf, capacity, C.byref(n)))
        return [int(buf[i]) for i in range(n.value)]

    def sync(self) -> None:
        native.check(native.lib().bf_serve_sync(self._h))

    def stream_handle(self) -> int:
        return int(native.lib().bf_serve_stream(self._h) or 0)

    def pool(self, n_ant: int):
        """The device voltage pool that jobs of n_ant antennas read, as a torch
        uint8 tensor [pool_spectra][pool_channels][n_ant] (a view, no copy).
        The ingest hook: write captured rows into it on the server's stream
        (torch.cuda.ExternalStream(server.stream_handle())) before the step
        whose windows read them."""
        import torch
        ptr, sp, ch = C.c_void_p(), C.c_uint64(0), C.c_uint64(0)
        native.check(native.lib().bf_serve_pool(self._h, int(n_ant), C.byref(ptr), C.byref(sp), C.byref(ch)))
        shape = (int(sp.value), int(ch.value), int(n_ant))
        return torch.as_tensor(_DeviceArray(int(ptr.value), shape, "|u1"), device="cuda")

    def result_pointers(self, job_id: int) -> tuple[int, int, int, int]:
        i, c, p = C.c_void_p(), C.c_void_p(), C.c_void_p()
        n = C.c_uint64(0)
        native.check(native.lib().bf_serve_result(self._h, int(job_id), C.byref(i), C.byref(c), C.byref(p),
                                                  C.byref(n)))
        return int(i.value or 0), int(c.value or 0), int(p.value or 0), int(n.value)

    def result(self, job_id: int, floats: bool = True):
        """Host copies of a DONE job's results: integrated (grid [shard][W][F][B],
        tracker [W][F_total][sources]) and, for quantized grid jobs, codes and
        the (offset, scale) parameters.  floats=False skips a quantized grid
        job's float output (its product is the int8 codes).  A DONE job's
        results are complete, so the copies run on the caller's current
        stream (into pinned host memory), never on the server's own stream,
        which the server destroys when it closes."""
        import torch
        spec = self.specs[int(job_id)]
        ip, cp, pp, W = self.result_pointers(job_id)
        F = self.config.shard_channels
        if spec.kind == GRID:
            shape = (spec.n_shards, W, F, spec.n_beams)
        else:
            shape = (W, spec.n_shards * F, spec.n_beams)
        views = []
        if floats or not cp:
            views.append((ip, shape, "<f4", torch.float32))
        if cp:
            npar = spec.n_shards * W * ((F + 15) // 16) * ((spec.n_beams + 15) // 16) * 2
            views += [(cp, shape, "|i1", torch.int8), (pp, (npar,), "<f4", torch.float32)]
        out = []
        for ptr, shp, ts, dt in views:
            dev = torch.as_tensor(_DeviceArray(ptr, shp, ts), device="cuda")
            host = torch.empty(shp, dtype=dt, pin_memory=True)
            host.copy_(dev, non_blocking=True)
            out.append(host)
        torch.cuda.current_stream().synchronize()
        arrs = [h.numpy() for h in out]
        if not (floats or not cp):
            arrs = [None] + arrs
        if not cp:
            arrs += [None, None]
        return tuple(arrs)

    # -- reporting
    def stats(self) -> dict:
        st = native.ServeStats()
        native.check(native.lib().bf_serve_stats_get(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in native.ServeStats._fields_}

    def step_times(self) -> np.ndarray:
        n = C.c_uint64(0)
        native.check(native.lib().bf_serve_step_times(self._h, None, 0, C.byref(n)))
        out = np.zeros(int(n.value), np.float32)
        if out.size:
            native.check(native.lib().bf_serve_step_times(
                self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size, C.byref(n)))
        return out


# --------------------------------------------------------------------------
# the served benchmark's request stream
# --------------------------------------------------------------------------

def array_positions(n_ant: int) -> np.ndarray:
    """64 antennas: 2 x 32 grid at half a wavelength of 800 MHz; 32: a line
    at half a wavelength of 600 MHz."""
    if n_ant == 64:
        sp = 0.5 * C_LIGHT / 800e6
        return np.array([((a % 32) * sp, (a // 32) * sp, 0.0) for a in range(64)], np.float32)
    sp = 0.5 * C_LIGHT / 600e6
    return np.array([(a * sp, 0.0, 0.0) for a in range(n_ant)], np.float32)


def band_frequencies(n_channels: int) -> np.ndarray:
    """n_channels over 400-800 MHz, end points included."""
    return (400e6 + np.arange(n_channels) * (400e6 / max(1, n_channels - 1))).astype(np.float32)


def spec_of_checkpoint(image: bytes) -> JobSpec:
    """The job description carried by a checkpoint image (bf_serve_checkpoint):
    "BFSRVCK1", u32 version, u32 kind, n_ant, n_shards, n_beams, quantize,
    u64 n_spectra, integration_spectra, pool_offset, windows served, u32
    window_spectra, shard_channels, max_shards, pool-scale bits, u64
    pool_spectra, pool_seed, then float32 positions, frequencies and
    directions (grid) or trajectories (tracker)."""
    b = bytes(image)
    if b[:8] != b"BFSRVCK1":
        raise ValueError("not a served-job checkpoint image")
    u32 = np.frombuffer(b, np.uint32, 6, 8)
    _, kind, A, ns, B, quant = (int(x) for x in u32)
    u64 = np.frombuffer(b, np.uint64, 4, 32)
    n_spectra, S, pool_offset = int(u64[0]), int(u64[1]), int(u64[2])
    shard_ch = int(np.frombuffer(b, np.uint32, 1, 68)[0])
    at = 96
    pos = np.frombuffer(b, np.float32, 3 * A, at).reshape(A, 3).copy()
    at += 12 * A
    freq = np.frombuffer(b, np.float32, ns * shard_ch, at).copy()
    at += 4 * ns * shard_ch
    if kind == GRID:
        dirs = np.frombuffer(b, np.float32, 3 * B, at).reshape(B, 3).copy()
        return JobSpec(GRID, A, ns, B, n_spectra, S, pos, freq, directions=dirs, pool_offset=pool_offset,
                       quantize=bool(quant))
    traj = np.frombuffer(b, np.float32, 4 * B, at).reshape(B, 4).copy()
    return JobSpec(TRACKER, A, ns, B, n_spectra, S, pos, freq, trajectories=traj, pool_offset=pool_offset)


def poisson_mix(seed: int = 1, rate_hz: float = 200.0, duration_s: float = 10.0, window_spectra: int = 320,
                pool_spectra: int = 20480, shard_channels: int = 336, max_shards: int = 4) -> list[JobSpec]:
    """Seeded request stream: Poisson arrivals at rate_hz for duration_s.
    Each job: 32 or 64 antennas, 1-4 shards of shard_channels, either a grid
    of 1, 8, 32 or 128 beams (int8 quantized) or a tracker with 1-16 drifting
    sources; 0.1-2 s of data at 2.56 us per spectrum (rounded up to whole
    served windows); integration over 10 or 320 spectra."""
    rng = np.random.default_rng(seed)
    jobs: list[JobSpec] = []
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t >= duration_s:
            break
        A = int(rng.choice([32, 64]))
        ns = int(rng.integers(1, max_shards + 1))
        kind = int(rng.integers(0, 2))
        dur = float(rng.uniform(0.1, 2.0))
        n_spectra = int(math.ceil(dur / SPECTRUM_S / window_spectra)) * window_spectra
        S = int(rng.choice([10, 320]))
        pos = array_positions(A)
        freq = band_frequencies(ns * shard_channels)
        offset = int(rng.integers(0, pool_spectra // window_spectra)) * window_spectra
        if kind == GRID:
            B = int(rng.choice([1, 8, 32, 128]))
            lm = rng.uniform(-0.3, 0.3, size=(B, 2)).astype(np.float32)
            n = np.sqrt(np.float32(1) - (lm[:, 0] * lm[:, 0] + lm[:, 1] * lm[:, 1])).astype(np.float32)
            dirs = np.concatenate([lm, n[:, None]], axis=1).astype(np.float32)
            jobs.append(JobSpec(GRID, A, ns, B, n_spectra, S, pos, freq, directions=dirs, pool_offset=offset,
                                quantize=True, arrival_s=t))
        else:
            n_src = int(rng.integers(1, 17))
            tr = np.zeros((n_src, 4), np.float32)
            tr[:, :2] = rng.uniform(-0.3, 0.3, size=(n_src, 2))
            tr[:, 2:] = rng.uniform(-0.02, 0.02, size=(n_src, 2)) / n_spectra
            jobs.append(JobSpec(TRACKER, A, ns, n_src, n_spectra, S, pos, freq, trajectories=tr,
                                pool_offset=offset, arrival_s=t))
    return jobs


def run_stream(server: Server, jobs: list[JobSpec], window_spectra: int = 320, release: bool = True,
               max_steps: int | None = None, on_done=None) -> dict:
    """Virtual-time request loop: job i is submitted before the first served
    window whose start (step * window_spectra * 2.56 us) is at or after its
    arrival; one server step per window; finished jobs (the server's
    completion queue) are handed to on_done(job_id) and released.  When
    nothing is live the loop waits for the GPU (queued jobs need the memory
    of finished ones) or jumps to the next arrival.  Returns counts."""
    k = getattr(server, "windows_per_step", 1)
    step_s = window_spectra * k * SPECTRUM_S
    order = sorted(range(len(jobs)), key=lambda i: jobs[i].arrival_s)
    i = 0
    step_idx = 0
    steps_run = 0
    outstanding = 0
    step_windows = []   # stream window index of every server step that launched work
    ids = [None] * len(jobs)
    while True:
        while i < len(order) and jobs[order[i]].arrival_s <= step_idx * step_s:
            ids[order[i]] = server.submit(jobs[order[i]])
            outstanding += 1
            i += 1
        n_live = server.step()
        if n_live:
            steps_run += 1
            step_windows.append(step_idx * k)
        step_idx += 1
        if n_live == 0 or step_idx % 8 == 0:
            for jid in server.take_done():
                outstanding -= 1
                if on_done is not None:
                    on_done(jid)
                if release:
                    server.release(jid)
        if max_steps is not None and steps_run >= max_steps:
            break
        if n_live == 0:
            if outstanding == 0:
                if i >= len(order):
                    break
                step_idx = max(step_idx, int(math.ceil(jobs[order[i]].arrival_s / step_s)))
            else:
                server.sync()
    return {"steps": steps_run, "submitted": i, "step_windows": step_windows, "job_ids": ids,
            "windows_per_step": k}


def realtime_replay(step_ms, step_windows, window_spectra: int = 320, windows_per_step: int = 1) -> dict:
    """Replays the served steps against the stream clock.  Step i serves the
    stream windows from step_windows[i] on (windows_per_step of them), whose
    data is complete at (step_windows[i] + windows_per_step) * window time;
    the GPU starts a step when its data is complete and the previous step has
    finished, and takes step_ms[i] (its measured device time).  Returns per-step
    ready and finish times (s) and the real-time factor (stream seconds served /
    device seconds)."""
    import numpy as np
    w_s = window_spectra * SPECTRUM_S
    ready = (np.asarray(step_windows, np.float64) + float(windows_per_step)) * w_s
    dur = np.asarray(step_ms, np.float64) / 1e3
    n = min(len(ready), len(dur))
    ready, dur = ready[:n], dur[:n]
    end = np.empty(n)
    t = 0.0
    for k in range(n):
        t = max(t, ready[k]) + dur[k]
        end[k] = t
    span = (ready[-1] - ready[0] + windows_per_step * w_s) if n else 0.0
    return {"ready_s": ready, "end_s": end, "latency_s": end - ready,
            "realtime_factor": span / dur.sum() if n and dur.sum() > 0 else None,
            "stream_s": span, "device_s": float(dur.sum())}
