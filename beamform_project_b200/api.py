"""Python host mirror of the reference's beamformer interface for the hot path.

Names, argument meaning and error behaviour follow the reference's
include/beamformer headers:

  cuda_stage_api.hpp:21-42   launch_packed_beamformer,
                             launch_packed_integrated_beamformer,
                             launch_quantize_integrated_intensity
  cuda_beamformer.hpp:98-123 cuda_beamform_packed_intensity,
                             cuda_beamform_packed_integrated_intensity,
                             cuda_beamform_packed_quantized_integrated_intensity
  beam_tracker.hpp:60-100    tracker_window_count / tracker_window_direction /
                             the per-spectrum tracker
  config.hpp:74-94           Dimensions / validate_dimensions
  quantization.hpp:16-43     chunk layout

Device-stage functions take torch CUDA tensors and a stream (None = torch's
current stream) and launch one kernel through the C ABI; they do not
allocate or synchronise.  Buffer sizes are checked here (the C ABI only sees
raw pointers), so an undersized tensor is an InvalidArgument, never an
out-of-bounds access.  Host one-shot functions take numpy arrays and copy in
and out, like the reference's wrappers.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from enum import IntEnum

import numpy as np

from . import native
from .native import (BeamformerError, CudaError, DeviceTimeout, InvalidArgument, LogicError,  # noqa: F401
                     OutOfRange, Unsupported, check)

SPEED_OF_LIGHT = 299_792_458.0
TWO_PI = 6.283185307179586476925286766559
LOCAL_FREQUENCY_CHANNELS = 336
MAXIMUM_BEAMS = 128
QUANT_CHUNK_FREQ = 16
QUANT_CHUNK_BEAM = 16
INTEGRATION_AFTER_UPCHAN = 10
INTEGRATION_DIRECT = 320


class CudaBeamformerKernel(IntEnum):
    Direct = native.BF_KERNEL_DIRECT
    Tiled = native.BF_KERNEL_TILED
    Tensor = native.BF_KERNEL_TENSOR


class TrackerMode(IntEnum):
    ReferenceOrder = 0
    Streaming = 1


@dataclass(frozen=True)
class Dimensions:
    n_time: int = 15360
    n_freq: int = LOCAL_FREQUENCY_CHANNELS
    n_ant: int = 64
    n_beams: int = 64

    def c(self) -> native.Dims:
        return native.dims(self.n_time, self.n_freq, self.n_ant, self.n_beams)


def validate_dimensions(dims: Dimensions) -> None:
    """config.hpp:81-94 (raises InvalidArgument with the reference's text)."""
    d = dims.c()
    check(native.lib().bf_validate_dimensions(C.byref(d)))


def integrated_time_count(n_time: int, integration_spectra: int) -> int:
    """temporal_integration.cpp:16-26."""
    if integration_spectra == 0:
        raise InvalidArgument(1, "integration_spectra must be positive")
    if n_time == 0:
        raise InvalidArgument(1, "n_time must be positive")
    return -(-n_time // integration_spectra)


def quantization_layout(integrated_dims: Dimensions) -> tuple[int, int, int]:
    """quantization.cpp:34-47: (time_tiles, frequency_tiles, beam_tiles)."""
    validate_dimensions(integrated_dims)
    return (integrated_dims.n_time, -(-integrated_dims.n_freq // QUANT_CHUNK_FREQ),
            -(-integrated_dims.n_beams // QUANT_CHUNK_BEAM))


def quantization_parameter_count(integrated_dims: Dimensions) -> int:
    t, f, b = quantization_layout(integrated_dims)
    return t * f * b


# --------------------------------------------------------------------------
# device helpers
# --------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _stream_handle(stream) -> int:
    torch = _torch()
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _dev(t, name: str, dtype, min_elems: int) -> int:
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise InvalidArgument(1, f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise InvalidArgument(1, f"{name} must have dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise InvalidArgument(1, f"{name} must be contiguous")
    if t.numel() < min_elems:
        raise InvalidArgument(1, f"{name} is smaller than dimensions ({t.numel()} < {min_elems})")
    return t.data_ptr()


def _weight_count(kernel: int, d: Dimensions) -> int:
    if kernel == CudaBeamformerKernel.Tiled:
        return d.n_freq * (-(-d.n_beams // 32)) * d.n_ant * 32 * 2
    return d.n_beams * d.n_freq * d.n_ant * 2


# --------------------------------------------------------------------------
# device-stage API (cuda_stage_api.hpp:21-42)
# --------------------------------------------------------------------------

def launch_packed_beamformer(kernel, stream, packed_voltage, weights, intensity,
                             dims: Dimensions) -> None:
    torch = _torch()
    validate_dimensions(dims)
    k = int(kernel)
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    w = _dev(weights, "weights", torch.float32, _weight_count(k, dims))
    o = _dev(intensity, "intensity", torch.float32, dims.n_time * dims.n_freq * dims.n_beams)
    d = dims.c()
    check(native.lib().bf_launch_packed_beamformer(k, _stream_handle(stream), v, w, o, C.byref(d)))


def launch_packed_integrated_beamformer(kernel, stream, packed_voltage, weights,
                                        integrated_intensity, dims: Dimensions,
                                        integration_spectra: int) -> None:
    torch = _torch()
    validate_dimensions(dims)
    k = int(kernel)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    w = _dev(weights, "weights", torch.float32, _weight_count(k, dims))
    o = _dev(integrated_intensity, "integrated_intensity", torch.float32,
             nw * dims.n_freq * dims.n_beams)
    d = dims.c()
    check(native.lib().bf_launch_packed_integrated_beamformer(
        k, _stream_handle(stream), v, w, o, C.byref(d), int(integration_spectra)))


def launch_quantize_integrated_intensity(stream, integrated_intensity, codes, params,
                                         integrated_dims: Dimensions) -> None:
    torch = _torch()
    n = integrated_dims.n_time * integrated_dims.n_freq * integrated_dims.n_beams
    i = _dev(integrated_intensity, "integrated_intensity", torch.float32, n)
    c = _dev(codes, "codes", torch.int8, n)
    p = _dev(params, "params", torch.float32, 2 * quantization_parameter_count(integrated_dims))
    d = integrated_dims.c()
    check(native.lib().bf_launch_quantize_integrated_intensity(_stream_handle(stream), i, c, p,
                                                               C.byref(d)))


# --------------------------------------------------------------------------
# split-precision tensor-core grid
# --------------------------------------------------------------------------

def split_weight_bytes(dims: Dimensions, n_shards: int = 1) -> int:
    d = dims.c()
    return int(native.lib().bf_split_weight_bytes(C.byref(d), int(n_shards)))


def prepare_split_weights(stream, weights, split_weights, dims: Dimensions, n_shards: int = 1) -> None:
    torch = _torch()
    validate_dimensions(dims)
    w = _dev(weights, "weights", torch.float32, n_shards * dims.n_beams * dims.n_freq * dims.n_ant * 2)
    s = _dev(split_weights, "split_weights", torch.uint8, split_weight_bytes(dims, n_shards))
    d = dims.c()
    check(native.lib().bf_prepare_split_weights(_stream_handle(stream), w, s, C.byref(d),
                                                int(n_shards)))


def grid_tensor_integrated(stream, packed_voltage, split_weights, integrated, codes, params,
                           dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> None:
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    n_out = n_shards * nw * dims.n_freq * dims.n_beams
    v = _dev(packed_voltage, "packed_voltage", torch.uint8,
             n_shards * dims.n_time * dims.n_freq * dims.n_ant)
    s = _dev(split_weights, "split_weights", torch.uint8, split_weight_bytes(dims, n_shards))
    o = _dev(integrated, "integrated", torch.float32, n_out)
    c = p = None
    if codes is not None or params is not None:
        qd = Dimensions(nw, dims.n_freq, dims.n_ant, dims.n_beams)
        c = _dev(codes, "codes", torch.int8, n_out)
        p = _dev(params, "params", torch.float32, 2 * n_shards * quantization_parameter_count(qd))
    d = dims.c()
    check(native.lib().bf_grid_tensor_integrated(_stream_handle(stream), v, s, o, c, p,
                                                 C.byref(d), int(integration_spectra),
                                                 int(n_shards)))


def cov_weight_bytes(dims: Dimensions, n_shards: int = 1) -> int:
    d = dims.c()
    return int(native.lib().bf_cov_weight_bytes(C.byref(d), int(n_shards)))


def prepare_cov_weights(stream, weights, cov_weights, dims: Dimensions, n_shards: int = 1) -> None:
    """Canonical complex64 weights ([shard][B][F][A][2], device) -> the
    covariance-form grid's per-channel image (bf_prepare_cov_weights)."""
    torch = _torch()
    validate_dimensions(dims)
    w = _dev(weights, "weights", torch.float32, 2 * n_shards * dims.n_beams * dims.n_freq * dims.n_ant)
    o = _dev(cov_weights, "cov_weights", torch.uint8, cov_weight_bytes(dims, n_shards))
    d = dims.c()
    check(native.lib().bf_prepare_cov_weights(_stream_handle(stream), w, o, C.byref(d), int(n_shards)))


def grid_cov_integrated(stream, packed_voltage, cov_weights, integrated, codes, params,
                        dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> None:
    """The grid beamformer in covariance form (bf_grid_cov_integrated): the
    integrated power of each window from its exact INT32 array covariance on
    int8 tensor cores and a split-fp16 quadratic form.  n_ant 64, integration
    a multiple of 64 spectra; same outputs and layouts as grid_tensor_integrated."""
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    n_out = n_shards * nw * dims.n_freq * dims.n_beams
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, n_shards * dims.n_time * dims.n_freq * dims.n_ant)
    s = _dev(cov_weights, "cov_weights", torch.uint8, cov_weight_bytes(dims, n_shards))
    o = _dev(integrated, "integrated", torch.float32, n_out)
    c = p = None
    if codes is not None or params is not None:
        qd = Dimensions(nw, dims.n_freq, dims.n_ant, dims.n_beams)
        c = _dev(codes, "codes", torch.int8, n_out)
        p = _dev(params, "params", torch.float32, 2 * n_shards * quantization_parameter_count(qd))
    d = dims.c()
    check(native.lib().bf_grid_cov_integrated(_stream_handle(stream), v, s, o, c, p, C.byref(d),
                                              int(integration_spectra), int(n_shards)))


def grid_cov_estimate(stream, packed_voltage, cov_weights, integrated, estimate, dims: Dimensions,
                      integration_spectra: int, n_shards: int = 1) -> None:
    """grid_cov_integrated that also writes each value's relative error
    estimate 2^-23 |v_b|^2 tr(E) / I (float32, same layout as integrated)."""
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    n_out = n_shards * nw * dims.n_freq * dims.n_beams
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, n_shards * dims.n_time * dims.n_freq * dims.n_ant)
    s = _dev(cov_weights, "cov_weights", torch.uint8, cov_weight_bytes(dims, n_shards))
    o = _dev(integrated, "integrated", torch.float32, n_out)
    e = _dev(estimate, "estimate", torch.float32, n_out)
    d = dims.c()
    check(native.lib().bf_grid_cov_estimate(_stream_handle(stream), v, s, o, e, C.byref(d),
                                            int(integration_spectra), int(n_shards)))


def auto_weight_bytes(dims: Dimensions, n_shards: int = 1) -> int:
    d = dims.c()
    return int(native.lib().bf_auto_weight_bytes(C.byref(d), int(n_shards)))


def prepare_auto_weights(stream, weights, auto_weights, dims: Dimensions, n_shards: int = 1) -> None:
    """Canonical complex64 weights -> the checked grid's operand (covariance
    image, where the form applies, then the split image)."""
    torch = _torch()
    validate_dimensions(dims)
    w = _dev(weights, "weights", torch.float32, 2 * n_shards * dims.n_beams * dims.n_freq * dims.n_ant)
    o = _dev(auto_weights, "auto_weights", torch.uint8, auto_weight_bytes(dims, n_shards))
    d = dims.c()
    check(native.lib().bf_prepare_auto_weights(_stream_handle(stream), w, o, C.byref(d), int(n_shards)))


def grid_auto_workspace_bytes(dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> int:
    d = dims.c()
    return int(native.lib().bf_grid_auto_workspace_bytes(C.byref(d), int(integration_spectra), int(n_shards)))


def grid_auto_integrated(stream, packed_voltage, auto_weights, integrated, codes, params, workspace,
                         dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> None:
    """The checked grid beamformer (bf_grid_auto_integrated): the covariance
    form with per-value error estimates where it applies, the split kernel
    over every unit whose estimate exceeds the calibrated limit, and the split
    kernel alone elsewhere; every value within 1e-5 relative of FP64.  The
    workspace's first int32 is the number of units recomputed."""
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    n_out = n_shards * nw * dims.n_freq * dims.n_beams
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, n_shards * dims.n_time * dims.n_freq * dims.n_ant)
    s = _dev(auto_weights, "auto_weights", torch.uint8, auto_weight_bytes(dims, n_shards))
    o = _dev(integrated, "integrated", torch.float32, n_out)
    c = p = None
    if codes is not None or params is not None:
        qd = Dimensions(nw, dims.n_freq, dims.n_ant, dims.n_beams)
        c = _dev(codes, "codes", torch.int8, n_out)
        p = _dev(params, "params", torch.float32, 2 * n_shards * quantization_parameter_count(qd))
    wsb = grid_auto_workspace_bytes(dims, integration_spectra, n_shards)
    ws = _dev(workspace, "workspace", torch.uint8, wsb) if wsb > 0 else None
    d = dims.c()
    check(native.lib().bf_grid_auto_integrated(_stream_handle(stream), v, s, o, c, p, ws, C.byref(d),
                                               int(integration_spectra), int(n_shards)))


# --------------------------------------------------------------------------
# autotuner of the grid path (bf_autotune_grid, bf_tune_*)
# --------------------------------------------------------------------------

GRID_FORMS = {0: "split", 1: "checked covariance"}


def _cfg_dict(c) -> dict:
    return {"form": GRID_FORMS[int(c.form)], "group_mult": int(c.group_mult), "paired": bool(c.paired)}


def autotune_grid(stream, dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> dict:
    """Time every launch choice of the grid path for this class (n_ant,
    padded beams, integration) on seeded synthetic data, keep those whose
    products agree with the default's, record the fastest in the tuning
    table (used by later untuned calls) and return the candidates."""
    validate_dimensions(dims)
    cap = 16
    cands = (native.GridConfig * cap)()
    ms = (C.c_float * cap)()
    ok = (C.c_uint8 * cap)()
    n = C.c_uint32(0)
    best = C.c_uint32(0)
    d = dims.c()
    check(native.lib().bf_autotune_grid(_stream_handle(stream), C.byref(d), int(integration_spectra), int(n_shards),
                                        cands, ms, ok, cap, C.byref(n), C.byref(best)))
    rows = [{**_cfg_dict(cands[i]), "ms": float(ms[i]), "ok": bool(ok[i])} for i in range(n.value)]
    return {"candidates": rows, "best": int(best.value), "chosen": rows[best.value]}


def tune_get(n_ant: int, nb_pad: int, integration_spectra: int, device: str | None = None) -> dict | None:
    c = native.GridConfig()
    found = C.c_int32(0)
    check(native.lib().bf_tune_get(device.encode() if device else None, int(n_ant), int(nb_pad),
                                   int(integration_spectra), C.byref(c), C.byref(found)))
    return _cfg_dict(c) if found.value else None


def tune_set(n_ant: int, nb_pad: int, integration_spectra: int, form: int, group_mult: int, paired: bool,
             ms: float = 0.0, device: str | None = None) -> None:
    c = native.GridConfig(int(form), int(group_mult), int(bool(paired)), 0)
    check(native.lib().bf_tune_set(device.encode() if device else None, int(n_ant), int(nb_pad),
                                   int(integration_spectra), C.byref(c), float(ms)))


def tune_save(path: str | None = None) -> None:
    check(native.lib().bf_tune_save(path.encode() if path else None))


def tune_load(path: str | None = None) -> None:
    check(native.lib().bf_tune_load(path.encode() if path else None))


def tune_clear() -> None:
    check(native.lib().bf_tune_clear())


def tune_cache_path() -> str:
    buf = C.create_string_buffer(4096)
    native.lib().bf_tune_cache_path(buf, len(buf))
    return buf.value.decode()


def grid_auto_integrated_with(stream, packed_voltage, auto_weights, integrated, codes, params, workspace,
                              dims: Dimensions, integration_spectra: int, n_shards: int, form: int,
                              group_mult: int = 1, paired: bool = True) -> None:
    """grid_auto_integrated with an explicit launch choice."""
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    n_out = n_shards * nw * dims.n_freq * dims.n_beams
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, n_shards * dims.n_time * dims.n_freq * dims.n_ant)
    s = _dev(auto_weights, "auto_weights", torch.uint8, auto_weight_bytes(dims, n_shards))
    o = _dev(integrated, "integrated", torch.float32, n_out)
    c = p = None
    if codes is not None or params is not None:
        qd = Dimensions(nw, dims.n_freq, dims.n_ant, dims.n_beams)
        c = _dev(codes, "codes", torch.int8, n_out)
        p = _dev(params, "params", torch.float32, 2 * n_shards * quantization_parameter_count(qd))
    wsb = grid_auto_workspace_bytes(dims, integration_spectra, n_shards)
    ws = _dev(workspace, "workspace", torch.uint8, wsb) if wsb > 0 else None
    cfg = native.GridConfig(int(form), int(group_mult), int(bool(paired)), 0)
    d = dims.c()
    check(native.lib().bf_grid_auto_integrated_with(_stream_handle(stream), v, s, o, c, p, ws, C.byref(d),
                                                    int(integration_spectra), int(n_shards), C.byref(cfg)))


def grid_tensor_workspace_bytes(dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> int:
    d = dims.c()
    return int(native.lib().bf_grid_tensor_workspace_bytes(C.byref(d), int(integration_spectra), int(n_shards)))


def grid_tensor_quantized(stream, packed_voltage, split_weights, integrated, codes, params, workspace,
                          dims: Dimensions, integration_spectra: int, n_shards: int = 1) -> None:
    """Tensor-core grid with the int8 quantizer fused into its epilogue;
    `workspace` (uint8, grid_tensor_workspace_bytes) is the kernel's scratch."""
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    n_out = n_shards * nw * dims.n_freq * dims.n_beams
    qd = Dimensions(nw, dims.n_freq, dims.n_ant, dims.n_beams)
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, n_shards * dims.n_time * dims.n_freq * dims.n_ant)
    s = _dev(split_weights, "split_weights", torch.uint8, split_weight_bytes(dims, n_shards))
    o = _dev(integrated, "integrated", torch.float32, n_out)
    c = _dev(codes, "codes", torch.int8, n_out)
    p = _dev(params, "params", torch.float32, 2 * n_shards * quantization_parameter_count(qd))
    w = _dev(workspace, "workspace", torch.uint8, grid_tensor_workspace_bytes(dims, integration_spectra, n_shards))
    d = dims.c()
    check(native.lib().bf_grid_tensor_quantized(_stream_handle(stream), v, s, o, c, p, w, C.byref(d),
                                                int(integration_spectra), int(n_shards)))


# --------------------------------------------------------------------------
# tracker
# --------------------------------------------------------------------------

def _host(a, name: str, dtype, min_elems: int) -> int:
    """Address of a contiguous host buffer (numpy array or CPU tensor)."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.dtype(dtype) or not a.flags.c_contiguous:
            raise InvalidArgument(1, f"{name} must be a contiguous {np.dtype(dtype)} array")
        if a.size < min_elems:
            raise InvalidArgument(1, f"{name} is smaller than dimensions ({a.size} < {min_elems})")
        return a.ctypes.data
    torch = _torch()
    tdt = {np.uint8: torch.uint8, np.int8: torch.int8, np.float32: torch.float32}[dtype]
    if not isinstance(a, torch.Tensor) or a.is_cuda or a.dtype != tdt or not a.is_contiguous():
        raise InvalidArgument(1, f"{name} must be a contiguous host {tdt} tensor or numpy array")
    if a.numel() < min_elems:
        raise InvalidArgument(1, f"{name} is smaller than dimensions ({a.numel()} < {min_elems})")
    return a.data_ptr()


def grid_pipeline_chunk_spectra(dims: Dimensions, integration_spectra: int, n_shards: int = 1,
                                chunk_spectra: int = 0) -> int:
    d = dims.c()
    return int(native.lib().bf_grid_pipeline_chunk_spectra(C.byref(d), int(integration_spectra), int(n_shards),
                                                           int(chunk_spectra)))


class GridHostPipeline:
    """The tensor-core grid fed from host buffers (bf_grid_pipeline_*): the
    counterpart of CudaBeamformerWorkspace.run_quantized_integrated_pipeline
    (include/beamformer/cuda_beamformer.hpp:66-76) with weights resident and,
    per block, the voltage streamed in and the products streamed out in time
    chunks that overlap the kernels.  Host layouts: voltage
    [shard][T][F][A] uint8, integrated [shard][W][F][B] float32, codes
    [shard][W][F][B] int8, params [shard][W][F/16][B/16][2] float32.  Pinned
    host tensors give PCIe-rate copies; numpy arrays work through the
    driver's staging."""

    def __init__(self, dims: Dimensions, integration_spectra: int, n_shards: int = 1, chunk_spectra: int = 0,
                 checked: bool = False):
        """checked=True runs the checked covariance form
        (bf_grid_pipeline_create_checked) instead of the split kernel."""
        validate_dimensions(dims)
        self.dims, self.spectra, self.n_shards = dims, int(integration_spectra), int(n_shards)
        self.n_windows = integrated_time_count(dims.n_time, integration_spectra)
        self.chunk_spectra = grid_pipeline_chunk_spectra(dims, integration_spectra, n_shards, chunk_spectra)
        h = C.c_void_p()
        d = dims.c()
        create = native.lib().bf_grid_pipeline_create_checked if checked else native.lib().bf_grid_pipeline_create
        check(create(C.byref(d), self.spectra, self.n_shards, int(chunk_spectra), C.byref(h)))
        self._h = h

    def upload_weights(self, weights) -> None:
        """Canonical complex64 weights [shard][B][F][A] (or float32 [..][2])."""
        w = np.asarray(weights)
        w = np.ascontiguousarray(w, dtype=np.complex64).view(np.float32) if np.iscomplexobj(w) \
            else np.ascontiguousarray(w, dtype=np.float32)
        n = 2 * self.n_shards * self.dims.n_beams * self.dims.n_freq * self.dims.n_ant
        check(native.lib().bf_grid_pipeline_upload_weights(self._handle(), _host(w.reshape(-1), "weights",
                                                                                 np.float32, n)))

    def run(self, voltage, integrated=None, codes=None, params=None) -> float:
        """One block; returns the device milliseconds from first copy-in to last copy-out."""
        d = self.dims
        n_out = self.n_shards * self.n_windows * d.n_freq * d.n_beams
        n_par = 2 * self.n_shards * quantization_parameter_count(
            Dimensions(self.n_windows, d.n_freq, d.n_ant, d.n_beams))
        v = _host(voltage, "voltage", np.uint8, self.n_shards * d.n_time * d.n_freq * d.n_ant)
        i = None if integrated is None else _host(integrated, "integrated", np.float32, n_out)
        c = None if codes is None else _host(codes, "codes", np.int8, n_out)
        p = None if params is None else _host(params, "params", np.float32, n_par)
        ms = C.c_float(0.0)
        check(native.lib().bf_grid_pipeline_run(self._handle(), v, i, c, p, C.byref(ms)))
        return float(ms.value)

    def _handle(self):
        if self._h is None:
            raise LogicError(2, "the pipeline has been closed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            native.lib().bf_grid_pipeline_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may be gone already
            pass


def tracker(stream, mode, packed_voltage, positions, wave_numbers, window_directions,
            intensity, integrated, dims: Dimensions, integration_spectra: int) -> None:
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    pp = _dev(positions, "positions", torch.float32, 3 * dims.n_ant)
    k = _dev(wave_numbers, "wave_numbers", torch.float64, dims.n_freq)
    dd = _dev(window_directions, "window_directions", torch.float32, 3 * nw)
    i = _dev(intensity, "intensity", torch.float32, dims.n_time * dims.n_freq) if intensity is not None else None
    g = _dev(integrated, "integrated", torch.float32, nw * dims.n_freq) if integrated is not None else None
    d = dims.c()
    check(native.lib().bf_tracker(_stream_handle(stream), int(mode), v, pp, k, dd, i, g,
                                  C.byref(d), int(integration_spectra)))


# --------------------------------------------------------------------------
# DOA (CpuOptBeamTracker's covariance and scan, cpu_opt_beam_tracker.hpp:91-169)
# --------------------------------------------------------------------------

def doa_covariance_i32(stream, packed_voltage, covariance, dims: Dimensions, block_len: int) -> None:
    """Exact int32 block covariance [blocks][F][A][A][2] on int8 tensor cores."""
    torch = _torch()
    validate_dimensions(dims)
    B = dims.n_time // block_len if block_len else 0
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    c = _dev(covariance, "covariance", torch.int32, B * dims.n_freq * dims.n_ant * dims.n_ant * 2)
    d = dims.c()
    check(native.lib().bf_doa_covariance_i32(_stream_handle(stream), v, c, C.byref(d), int(block_len)))


def doa_workspace_bytes(dims: Dimensions, block_len: int, subarray: int) -> int:
    d = dims.c()
    return int(native.lib().bf_doa_workspace_bytes(C.byref(d), int(block_len), int(subarray)))


def doa_scan(stream, covariance, positions, wave_numbers, dims: Dimensions, block_len: int, subarray: int,
             forgetting: float, diag_load: float, l_first: float, l_step: float, n_points: int,
             m_fixed: float, bartlett, capon, l_est, workspace) -> None:
    torch = _torch()
    validate_dimensions(dims)
    B = dims.n_time // block_len if block_len else 0
    M = subarray if 0 < subarray < dims.n_ant else dims.n_ant
    c = _dev(covariance, "covariance", torch.int32, B * dims.n_freq * dims.n_ant * dims.n_ant * 2)
    pp = _dev(positions, "positions", torch.float32, 3 * M)
    k = _dev(wave_numbers, "wave_numbers", torch.float64, dims.n_freq)
    b = _dev(bartlett, "bartlett", torch.float64, B * n_points)
    cp = _dev(capon, "capon", torch.float64, B * n_points)
    le = _dev(l_est, "l_est", torch.float64, 2 * B)
    w = _dev(workspace, "workspace", torch.uint8, doa_workspace_bytes(dims, block_len, subarray))
    d = dims.c()
    check(native.lib().bf_doa_scan(_stream_handle(stream), c, pp, k, C.byref(d), int(block_len), int(subarray),
                                   float(forgetting), float(diag_load), float(l_first), float(l_step),
                                   int(n_points), float(m_fixed), b, cp, le, w))


def _slice_dims(dims: Dimensions) -> None:
    if not (2 <= dims.n_freq <= 336 and dims.n_freq % 2 == 0):
        raise InvalidArgument(1, "a channel slice holds an even count of 2 to 336 channels")


def doa_covariance_i32_slice(stream, packed_voltage, covariance, dims: Dimensions, block_len: int) -> None:
    """bf_doa_covariance_i32_slice: doa_covariance_i32 on a contiguous slice of
    a job's channels (dims.n_freq = the slice's channels), one GPU's share of a
    channel-split DOA job."""
    torch = _torch()
    _slice_dims(dims)
    B = dims.n_time // block_len if block_len else 0
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    c = _dev(covariance, "covariance", torch.int32, B * dims.n_freq * dims.n_ant * dims.n_ant * 2)
    d = dims.c()
    check(native.lib().bf_doa_covariance_i32_slice(_stream_handle(stream), v, c, C.byref(d), int(block_len)))


def doa_scan_slice(stream, covariance, positions, wave_numbers, dims: Dimensions, block_len: int, subarray: int,
                   forgetting: float, diag_load: float, l_first: float, l_step: float, n_points: int,
                   m_fixed: float, bartlett, capon, l_est, workspace) -> None:
    """bf_doa_scan_slice: doa_scan over a channel slice; bartlett and capon
    are the slice's partial sums over frequency (sum them over the slices,
    then doa_peak)."""
    torch = _torch()
    _slice_dims(dims)
    B = dims.n_time // block_len if block_len else 0
    M = subarray if 0 < subarray < dims.n_ant else dims.n_ant
    c = _dev(covariance, "covariance", torch.int32, B * dims.n_freq * dims.n_ant * dims.n_ant * 2)
    pp = _dev(positions, "positions", torch.float32, 3 * M)
    k = _dev(wave_numbers, "wave_numbers", torch.float64, dims.n_freq)
    b = _dev(bartlett, "bartlett", torch.float64, B * n_points)
    cp = _dev(capon, "capon", torch.float64, B * n_points)
    le = _dev(l_est, "l_est", torch.float64, 2 * B)
    w = _dev(workspace, "workspace", torch.uint8, doa_workspace_bytes(dims, block_len, subarray))
    d = dims.c()
    check(native.lib().bf_doa_scan_slice(_stream_handle(stream), c, pp, k, C.byref(d), int(block_len),
                                         int(subarray), float(forgetting), float(diag_load), float(l_first),
                                         float(l_step), int(n_points), float(m_fixed), b, cp, le, w))


def doa_peak(stream, bartlett, capon, n_blocks: int, n_points: int, l_first: float, l_step: float, l_est) -> None:
    """bf_doa_peak: each block's argmax and parabolic peak of the Bartlett and
    Capon spectra ([blocks][n_points] double), as doa_scan finds them."""
    torch = _torch()
    b = _dev(bartlett, "bartlett", torch.float64, n_blocks * n_points)
    cp = _dev(capon, "capon", torch.float64, n_blocks * n_points)
    le = _dev(l_est, "l_est", torch.float64, 2 * n_blocks)
    check(native.lib().bf_doa_peak(_stream_handle(stream), b, cp, int(n_blocks), int(n_points), float(l_first),
                                   float(l_step), le))


def doa_track_config(block_len: int, subarray: int = 0, capon: bool = False, grid: int = 16, levels: int = 2,
                     interp: bool = True, fov_l: float = 0.2, fov_m: float = 0.2, forgetting: float = 1.0,
                     diag_load: float = 1e-3, prior_l: float = 0.0, prior_m: float = 0.0):
    """bf_doa_track_config; fields and defaults follow CpuOptTrackerConfig
    (include/beamformer/cpu_opt_beam_tracker.hpp:45-86) with the scan on."""
    return native.DoaTrackConfig(int(block_len), int(subarray), int(bool(capon)), int(grid), int(levels),
                                 int(bool(interp)), float(fov_l), float(fov_m), float(forgetting), float(diag_load),
                                 float(prior_l), float(prior_m))


def doa_track_workspace_bytes(dims: Dimensions, config) -> int:
    d = dims.c()
    return int(native.lib().bf_doa_track_workspace_bytes(C.byref(d), C.byref(config)))


def doa_track(stream, packed_voltage, positions, wave_numbers, dims: Dimensions, config, window_directions,
              intensity, workspace) -> None:
    """The reference's adaptive tracker on the GPU (bf_doa_track): per window a
    coarse-to-fine (l, m) search, then the beam along the estimate.
    window_directions float [W][3]; intensity float [T][F] or None."""
    torch = _torch()
    validate_dimensions(dims)
    W = dims.n_time // int(config.block_len) if config.block_len else 0
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    pp = _dev(positions, "positions", torch.float32, 3 * dims.n_ant)
    k = _dev(wave_numbers, "wave_numbers", torch.float64, dims.n_freq)
    dd = _dev(window_directions, "window_directions", torch.float32, 3 * W)
    ii = None if intensity is None else _dev(intensity, "intensity", torch.float32, dims.n_time * dims.n_freq)
    ws = _dev(workspace, "workspace", torch.uint8, doa_track_workspace_bytes(dims, config))
    d = dims.c()
    check(native.lib().bf_doa_track(_stream_handle(stream), v, pp, k, C.byref(d), C.byref(config), dd, ii, ws))


# --------------------------------------------------------------------------
# weights (generate_weights, reference src/weights.cpp:11-60) on the device
# --------------------------------------------------------------------------

def generate_weights(stream, positions, frequencies, directions, weights, dims: Dimensions,
                     n_shards: int = 1) -> None:
    """Canonical complex64 weights [shard][B][F][A] from positions [A][3],
    frequencies [n_shards * F] and unit directions [B][3] (device arrays)."""
    torch = _torch()
    validate_dimensions(dims)
    pp = _dev(positions, "positions", torch.float32, 3 * dims.n_ant)
    ff = _dev(frequencies, "frequencies", torch.float32, n_shards * dims.n_freq)
    dd = _dev(directions, "directions", torch.float32, 3 * dims.n_beams)
    w = _dev(weights, "weights", torch.float32, 2 * n_shards * dims.n_beams * dims.n_freq * dims.n_ant)
    d = dims.c()
    check(native.lib().bf_generate_weights(_stream_handle(stream), pp, ff, dd, w, C.byref(d), int(n_shards)))


def apply_loss_mask(stream, packed_voltage, loss_mask, dims: Dimensions, integration_spectra: int,
                    valid_counts=None) -> None:
    """Zero every lost frame (loss_mask uint8 [T][F], 0 = lost) of the packed
    voltage [T][F][A] in place; valid_counts (uint32 [ceil(T/S)][F], or None)
    gets the valid frames per integration window and channel."""
    torch = _torch()
    validate_dimensions(dims)
    v = _dev(packed_voltage, "packed_voltage", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    m = _dev(loss_mask, "loss_mask", torch.uint8, dims.n_time * dims.n_freq)
    c = None
    if valid_counts is not None:
        W = -(-dims.n_time // max(int(integration_spectra), 1))
        c = _dev(valid_counts, "valid_counts", torch.uint32, W * dims.n_freq)
    d = dims.c()
    check(native.lib().bf_apply_loss_mask(_stream_handle(stream), v, m, C.byref(d), int(integration_spectra), c))


# --------------------------------------------------------------------------
# synthetic voltages
# --------------------------------------------------------------------------

def generator_scale(sigma: float) -> float:
    """float32 multiplier turning the generator's integer draw
    D = 2 * (sum of eight uniform 16-bit integers) - 8 * 65535, whose variance
    is 4 * 8 * (65536^2 - 1) / 12, into a value of standard deviation sigma."""
    std = math.sqrt(4.0 * 8.0 * (65536.0 ** 2 - 1.0) / 12.0)
    return float(np.float32(sigma / std))


def generate_voltage(stream, seed: int, sample_offset: int, sigma: float, mu, epoch_len: int,
                     out, dims: Dimensions) -> None:
    torch = _torch()
    o = _dev(out, "out", torch.uint8, dims.n_time * dims.n_freq * dims.n_ant)
    m = None
    if mu is not None:
        m = _dev(mu, "mu", torch.float32, 2 * dims.n_freq * dims.n_ant)
    d = dims.c()
    check(native.lib().bf_generate_voltage(_stream_handle(stream), int(seed), int(sample_offset),
                                           C.c_float(generator_scale(sigma)), m, int(epoch_len),
                                           o, C.byref(d)))


# --------------------------------------------------------------------------
# geometry (host; geometry.cpp:34-106, beam_tracker.cpp:44-76)
# --------------------------------------------------------------------------

def regular_array(rows: int, columns: int, spacing_m: float = 0.6) -> np.ndarray:
    pos = np.zeros((rows * columns, 3), np.float32)
    for r in range(rows):
        for c in range(columns):
            pos[r * columns + c] = (np.float32(c) * np.float32(spacing_m),
                                    np.float32(r) * np.float32(spacing_m), 0.0)
    return pos


def default_positions(n_ant: int, spacing_m: float = 0.6) -> np.ndarray:
    shapes = {32: (4, 8), 64: (8, 8), 128: (8, 16), 256: (16, 16)}
    if n_ant not in shapes:
        raise InvalidArgument(1, "default geometry is available only for 32, 64, 128, or 256 antennas")
    return regular_array(*shapes[n_ant], spacing_m)


def channelized_frequencies(n_freq: int = 336, start_hz: float = 300e6,
                            channel_width_hz: float = 300e3) -> np.ndarray:
    ch = np.arange(n_freq, dtype=np.float32)
    return (np.float32(start_hz) + ch * np.float32(channel_width_hz)).astype(np.float32)


def direction_from_lm(l: float, m: float) -> np.ndarray:
    l32, m32 = np.float32(l), np.float32(m)
    tr = np.float32(l32 * l32) + np.float32(m32 * m32)
    if not (np.isfinite(l32) and np.isfinite(m32)):
        raise InvalidArgument(1, "direction cosines l and m must be finite")
    if tr > np.float32(1.0):
        raise InvalidArgument(1, "direction cosines must satisfy l*l + m*m <= 1")
    return np.array([l32, m32, np.sqrt(np.float32(1.0) - tr, dtype=np.float32)], np.float32)


def tracker_window_count(n_time: int, integration_spectra: int) -> int:
    if integration_spectra == 0:
        raise InvalidArgument(1, "integration_spectra must be positive")
    return (n_time + integration_spectra - 1) // integration_spectra


def tracker_window_directions(l0: float, m0: float, rate_l: float, rate_m: float, n_time: int,
                              integration_spectra: int) -> np.ndarray:
    """One direction per window, at the window's first sample (beam_tracker.cpp:52-76)."""
    W = tracker_window_count(n_time, integration_spectra)
    out = np.zeros((W, 3), np.float32)
    for w in range(W):
        tf = np.float32(w * integration_spectra)
        l = np.float32(np.float32(l0) + np.float32(tf * np.float32(rate_l)))
        m = np.float32(np.float32(m0) + np.float32(tf * np.float32(rate_m)))
        out[w] = direction_from_lm(l, m)
    return out


def wave_numbers(frequencies_hz: np.ndarray) -> np.ndarray:
    return TWO_PI * frequencies_hz.astype(np.float64) / SPEED_OF_LIGHT


# --------------------------------------------------------------------------
# host one-shot wrappers (cuda_beamformer.hpp:98-123)
# --------------------------------------------------------------------------

def _to_dev(a: np.ndarray, stream):
    torch = _torch()
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.pin_memory().to("cuda", non_blocking=True)


def cuda_beamform_packed_intensity(packed: np.ndarray, weights: np.ndarray, dims: Dimensions,
                                   kernel=CudaBeamformerKernel.Direct) -> np.ndarray:
    torch = _torch()
    validate_dimensions(dims)
    v = _to_dev(packed.reshape(-1)[: dims.n_time * dims.n_freq * dims.n_ant], None)
    w = _to_dev(weights.astype(np.float32).reshape(-1), None)
    out = torch.empty(dims.n_time * dims.n_freq * dims.n_beams, dtype=torch.float32, device="cuda")
    launch_packed_beamformer(kernel, None, v, w, out, dims)
    return out.cpu().numpy()


def cuda_beamform_packed_integrated_intensity(packed: np.ndarray, weights: np.ndarray,
                                              dims: Dimensions, integration_spectra: int,
                                              kernel=CudaBeamformerKernel.Tiled) -> np.ndarray:
    torch = _torch()
    validate_dimensions(dims)
    nw = integrated_time_count(dims.n_time, integration_spectra)
    v = _to_dev(packed.reshape(-1)[: dims.n_time * dims.n_freq * dims.n_ant], None)
    w = _to_dev(weights.astype(np.float32).reshape(-1), None)
    out = torch.empty(nw * dims.n_freq * dims.n_beams, dtype=torch.float32, device="cuda")
    launch_packed_integrated_beamformer(kernel, None, v, w, out, dims, integration_spectra)
    return out.cpu().numpy()


def cuda_beamform_packed_quantized_integrated_intensity(
        packed: np.ndarray, weights: np.ndarray, dims: Dimensions, integration_spectra: int,
        kernel=CudaBeamformerKernel.Tiled) -> tuple[np.ndarray, np.ndarray]:
    torch = _torch()
    nw = integrated_time_count(dims.n_time, integration_spectra)
    qd = Dimensions(nw, dims.n_freq, dims.n_ant, dims.n_beams)
    v = _to_dev(packed.reshape(-1)[: dims.n_time * dims.n_freq * dims.n_ant], None)
    w = _to_dev(weights.astype(np.float32).reshape(-1), None)
    integ = torch.empty(nw * dims.n_freq * dims.n_beams, dtype=torch.float32, device="cuda")
    codes = torch.empty_like(integ, dtype=torch.int8)
    params = torch.empty(2 * quantization_parameter_count(qd), dtype=torch.float32, device="cuda")
    launch_packed_integrated_beamformer(kernel, None, v, w, integ, dims, integration_spectra)
    launch_quantize_integrated_intensity(None, integ, codes, params, qd)
    return codes.cpu().numpy(), params.cpu().numpy().reshape(-1, 2)
