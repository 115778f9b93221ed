"""ctypes binding of the C ABI in include/bf_b200.h.

The library is built in-tree (python -m beamform_project_b200.build).  There
is no fallback: if the shared object is missing or cannot be loaded, every
call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libbf_b200.so"
_lib = None

BF_OK = 0
BF_KERNEL_DIRECT, BF_KERNEL_TILED, BF_KERNEL_TENSOR = 0, 1, 2


class BeamformerError(RuntimeError):
    """Base class; `status` holds the bf_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class InvalidArgument(BeamformerError, ValueError):
    """std::invalid_argument in the reference."""


class LogicError(BeamformerError):
    """std::logic_error in the reference."""


class CudaError(BeamformerError):
    """std::runtime_error (CUDA failure) in the reference."""


class OverflowError_(BeamformerError, OverflowError):
    """std::overflow_error in the reference."""


class OutOfRange(BeamformerError, IndexError):
    """std::out_of_range in the reference."""


class DeviceTimeout(BeamformerError):
    """A bounded device wait ran out."""


class Unsupported(BeamformerError):
    """A valid request outside what the kernels support."""


class ResourceError(BeamformerError, MemoryError):
    """A served job whose device state can never fit the server's HBM budget."""


_ERRORS = {1: InvalidArgument, 2: LogicError, 3: CudaError, 4: OverflowError_, 5: OutOfRange,
           6: DeviceTimeout, 7: Unsupported, 8: ResourceError}


class Dims(C.Structure):
    _fields_ = [("n_time", C.c_uint64), ("n_freq", C.c_uint64), ("n_ant", C.c_uint64),
                ("n_beams", C.c_uint64)]


class ServeConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_jobs", C.c_uint32), ("window_spectra", C.c_uint32),
                ("pool_spectra", C.c_uint64), ("shard_channels", C.c_uint32), ("max_shards", C.c_uint32),
                ("pool_seed", C.c_uint64), ("pool_scale", C.c_float), ("window_budget_us", C.c_float),
                ("windows_per_step", C.c_uint32)]


class ServeJob(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_ant", C.c_uint32), ("n_shards", C.c_uint32), ("n_beams", C.c_uint32),
                ("n_spectra", C.c_uint64), ("integration_spectra", C.c_uint64), ("pool_offset", C.c_uint64),
                ("positions", C.c_void_p), ("frequencies", C.c_void_p), ("directions", C.c_void_p),
                ("trajectories", C.c_void_p), ("quantize", C.c_int32), ("pad", C.c_int32)]


class ServeStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("steps", "steps_timed", "job_windows", "jobs_submitted", "jobs_admitted",
                                          "jobs_done", "jobs_cancelled", "jobs_rejected", "live_jobs",
                                          "queued_jobs", "arena_bytes_in_use", "arena_bytes_peak",
                                          "graph_captures")] + \
               [(n, C.c_double) for n in ("beam_samples", "step_ms_total", "step_ms_p50", "step_ms_p99",
                                          "step_ms_max")] + [("kernel_launches", C.c_uint64),
                                                             ("predicted_ms_last", C.c_double)]


class GridConfig(C.Structure):
    _fields_ = [("form", C.c_int32), ("group_mult", C.c_int32), ("paired", C.c_int32), ("reserved", C.c_int32)]


class DoaTrackConfig(C.Structure):
    _fields_ = [("block_len", C.c_uint64), ("subarray", C.c_uint64), ("estimator", C.c_uint32),
                ("grid", C.c_uint32), ("levels", C.c_uint32), ("interp", C.c_uint32), ("fov_l", C.c_float),
                ("fov_m", C.c_float), ("forgetting", C.c_float), ("diag_load", C.c_float), ("prior_l", C.c_float),
                ("prior_m", C.c_float)]


class ServeJobInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("pad", C.c_uint32), ("submit_step", C.c_uint64), ("admit_step", C.c_uint64),
                ("last_step", C.c_uint64), ("windows_launched", C.c_uint64)]


_P = C.c_void_p
_U64 = C.c_uint64
_PP = C.POINTER(C.c_void_p)
_SIGS = {
    "bf_version": (C.c_char_p, []),
    "bf_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "bf_validate_dimensions": (C.c_int, [C.POINTER(Dims)]),
    "bf_device_info": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_uint64), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "bf_launch_packed_beamformer": (C.c_int, [C.c_int, _P, _P, _P, _P, C.POINTER(Dims)]),
    "bf_launch_packed_integrated_beamformer": (C.c_int, [C.c_int, _P, _P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_launch_quantize_integrated_intensity": (C.c_int, [_P, _P, _P, _P, C.POINTER(Dims)]),
    "bf_split_weight_bytes": (_U64, [C.POINTER(Dims), _U64]),
    "bf_prepare_split_weights": (C.c_int, [_P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_grid_tensor_integrated": (C.c_int, [_P, _P, _P, _P, _P, _P, C.POINTER(Dims), _U64, _U64]),
    "bf_cov_weight_bytes": (_U64, [C.POINTER(Dims), _U64]),
    "bf_prepare_cov_weights": (C.c_int, [_P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_grid_cov_integrated": (C.c_int, [_P, _P, _P, _P, _P, _P, C.POINTER(Dims), _U64, _U64]),
    "bf_grid_cov_estimate": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Dims), _U64, _U64]),
    "bf_auto_weight_bytes": (_U64, [C.POINTER(Dims), _U64]),
    "bf_prepare_auto_weights": (C.c_int, [_P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_grid_auto_workspace_bytes": (_U64, [C.POINTER(Dims), _U64, _U64]),
    "bf_grid_auto_integrated": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.POINTER(Dims), _U64, _U64]),
    "bf_kernel_versions": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "bf_autotune_grid": (C.c_int, [_P, C.POINTER(Dims), _U64, _U64, C.POINTER(GridConfig), C.POINTER(C.c_float),
                                   C.POINTER(C.c_uint8), C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "bf_grid_auto_integrated_with": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.POINTER(Dims), _U64, _U64,
                                               C.POINTER(GridConfig)]),
    "bf_tune_get": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _U64, C.POINTER(GridConfig), C.POINTER(C.c_int32)]),
    "bf_tune_set": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _U64, C.POINTER(GridConfig), C.c_float]),
    "bf_tune_clear": (C.c_int, []),
    "bf_tune_load": (C.c_int, [C.c_char_p]),
    "bf_tune_save": (C.c_int, [C.c_char_p]),
    "bf_tune_cache_path": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "bf_tune_pick": (C.c_int, [C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.c_double,
                               C.POINTER(C.c_uint32)]),
    "bf_grid_pipeline_chunk_spectra": (_U64, [C.POINTER(Dims), _U64, _U64, _U64]),
    "bf_grid_pipeline_create": (C.c_int, [C.POINTER(Dims), _U64, _U64, _U64, _PP]),
    "bf_grid_pipeline_create_checked": (C.c_int, [C.POINTER(Dims), _U64, _U64, _U64, _PP]),
    "bf_grid_pipeline_upload_weights": (C.c_int, [_P, _P]),
    "bf_grid_pipeline_run": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(C.c_float)]),
    "bf_grid_pipeline_destroy": (C.c_int, [_P]),
    "bf_tracker": (C.c_int, [_P, C.c_int, _P, _P, _P, _P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_grid_tensor_workspace_bytes": (_U64, [C.POINTER(Dims), _U64, _U64]),
    "bf_grid_tensor_quantized": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.POINTER(Dims), _U64, _U64]),
    "bf_take_device_error": (C.c_int, [C.POINTER(C.c_uint32)]),
    "bf_doa_covariance_i32": (C.c_int, [_P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_doa_workspace_bytes": (_U64, [C.POINTER(Dims), _U64, _U64]),
    "bf_doa_scan": (C.c_int, [_P, _P, _P, _P, C.POINTER(Dims), _U64, _U64, C.c_double, C.c_double,
                              C.c_double, C.c_double, _U64, C.c_double, _P, _P, _P, _P]),
    "bf_doa_scan_slice": (C.c_int, [_P, _P, _P, _P, C.POINTER(Dims), _U64, _U64, C.c_double, C.c_double,
                              C.c_double, C.c_double, _U64, C.c_double, _P, _P, _P, _P]),
    "bf_doa_covariance_i32_slice": (C.c_int, [_P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_doa_peak": (C.c_int, [_P, _P, _P, _U64, _U64, C.c_double, C.c_double, _P]),
    "bf_generate_voltage": (C.c_int, [_P, _U64, _U64, C.c_float, _P, _U64, _P, C.POINTER(Dims)]),
    "bf_doa_track_workspace_bytes": (_U64, [C.POINTER(Dims), C.POINTER(DoaTrackConfig)]),
    "bf_doa_track": (C.c_int, [_P, _P, _P, _P, C.POINTER(Dims), C.POINTER(DoaTrackConfig), _P, _P, _P]),
    "bf_generate_weights": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Dims), _U64]),
    "bf_apply_loss_mask": (C.c_int, [_P, _P, _P, C.POINTER(Dims), _U64, _P]),
    "bf_probe_bounded_wait": (C.c_int, [_P, _U64]),
    "bf_serve_job_bytes": (_U64, [C.POINTER(ServeConfig), C.POINTER(ServeJob)]),
    "bf_serve_create": (C.c_int, [C.POINTER(ServeConfig), _PP]),
    "bf_serve_create_host_only": (C.c_int, [C.POINTER(ServeConfig), _PP]),
    "bf_serve_destroy": (C.c_int, [_P]),
    "bf_serve_submit": (C.c_int, [_P, C.POINTER(ServeJob), C.POINTER(C.c_uint64)]),
    "bf_serve_step": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "bf_serve_poll": (C.c_int, [_P, _U64, C.POINTER(C.c_int32)]),
    "bf_serve_job_info_get": (C.c_int, [_P, _U64, C.POINTER(ServeJobInfo)]),
    "bf_serve_result": (C.c_int, [_P, _U64, _PP, _PP, _PP, C.POINTER(C.c_uint64)]),
    "bf_serve_cancel": (C.c_int, [_P, _U64]),
    "bf_serve_checkpoint": (C.c_int, [_P, _U64, _P, _U64, C.POINTER(C.c_uint64)]),
    "bf_serve_restore": (C.c_int, [_P, _P, _U64, C.POINTER(C.c_uint64)]),
    "bf_serve_release": (C.c_int, [_P, _U64]),
    "bf_serve_sync": (C.c_int, [_P]),
    "bf_serve_stats_get": (C.c_int, [_P, C.POINTER(ServeStats)]),
    "bf_serve_step_times": (C.c_int, [_P, C.POINTER(C.c_float), _U64, C.POINTER(C.c_uint64)]),
    "bf_serve_take_done": (C.c_int, [_P, C.POINTER(C.c_uint64), _U64, C.POINTER(C.c_uint64)]),
    "bf_serve_stream": (_P, [_P]),
    "bf_serve_pool": (C.c_int, [_P, _U64, _PP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
}


def lib() -> C.CDLL:
    """Load the product library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing: run python -m beamform_project_b200.build")
        handle = C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW | C.RTLD_GLOBAL)
        for name, (res, args) in _SIGS.items():
            if hasattr(handle, name):
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
        _lib = handle
    return _lib


def library_path() -> Path:
    return _LIB_PATH


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().bf_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != BF_OK:
        cls = _ERRORS.get(status, BeamformerError)
        raise cls(status, last_error() or f"bf_status {status}")


def take_device_error() -> int:
    """Read and clear the tensor-core kernels' device error word (0 = none)."""
    v = C.c_uint32(0)
    check(lib().bf_take_device_error(C.byref(v)))
    return int(v.value)


def dims(n_time: int, n_freq: int, n_ant: int, n_beams: int) -> Dims:
    return Dims(int(n_time), int(n_freq), int(n_ant), int(n_beams))
