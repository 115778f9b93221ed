"""The C ABI library loads, exports every declared symbol, and validates its
arguments on the host (no GPU needed: every check below returns before any
CUDA call)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from beamform_project_b200 import native
from beamform_project_b200.native import Dims

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols() -> list[str]:
    names = []
    for h in (ROOT / "include").glob("*.h"):
        names += re.findall(r"BF_API\s+[\w\s\*]+?\b(bf_\w+)\s*\(", h.read_text())
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    syms = declared_symbols()
    assert len(syms) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", str(native.library_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\b(bf_\w+)\b", out))
    for s in syms:
        assert s in exported, s
        assert hasattr(lib, s)
    assert b"sm_100a" in lib.bf_version()


def test_library_is_built_for_sm100a_only():
    """Every nvcc step of the product build targets sm_100a and nothing else
    (the loaded kernels' versions are checked on the GPU)."""
    from beamform_project_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    flags = build.NVCC_FLAGS
    gencodes = [flags[i + 1] for i, f in enumerate(flags) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"]
    assert not any(f.startswith("-arch") or f.startswith("--gpu-architecture") for f in flags)


@pytest.mark.gpu
def test_loaded_kernels_are_sm100(cuda):
    binary, ptx = C.c_int(0), C.c_int(0)
    native.check(native.lib().bf_kernel_versions(C.byref(binary), C.byref(ptx)))
    assert binary.value == 100, binary.value
    assert ptx.value == 100, ptx.value


def _d(t=8, f=336, a=32, b=4):
    return Dims(t, f, a, b)


@pytest.mark.parametrize("dims,msg", [
    (_d(t=0), "n_time must be positive"),
    (_d(f=672), "336 frequency channels"),
    (_d(a=48), "n_ant must be 32, 64, 128, or 256"),
    (_d(b=0), "n_beams must be between 1 and 128"),
    (_d(b=129), "n_beams must be between 1 and 128"),
])
def test_validate_dimensions_matches_reference(dims, msg):
    lib = native.lib()
    st = lib.bf_validate_dimensions(C.byref(dims))
    assert st == 1
    assert msg in native.last_error()
    with pytest.raises(native.InvalidArgument, match=msg):
        native.check(st)


def test_stage_calls_validate_before_launch():
    lib = native.lib()
    d = _d()
    fake = C.c_void_p(4096)  # never dereferenced: every call below fails validation first
    assert lib.bf_launch_packed_beamformer(9, None, fake, fake, fake, C.byref(d)) == 1
    assert "kernel selector" in native.last_error()
    assert lib.bf_launch_packed_beamformer(0, None, None, fake, fake, C.byref(d)) == 1
    assert "packed_voltage must not be null" in native.last_error()
    assert lib.bf_launch_packed_beamformer(0, None, C.c_void_p(4097), fake, fake, C.byref(d)) == 1
    assert "16-byte aligned" in native.last_error()
    assert lib.bf_launch_packed_integrated_beamformer(0, None, fake, fake, fake, C.byref(d), 0) == 1
    assert "integration_spectra must be positive" in native.last_error()
    assert lib.bf_launch_packed_beamformer(2, None, fake, fake, fake, C.byref(d)) == 7
    assert lib.bf_grid_tensor_integrated(None, fake, fake, fake, None, None, C.byref(d), 40, 1) == 7
    assert "multiple of 32" in native.last_error()
    assert lib.bf_grid_tensor_integrated(None, fake, fake, fake, fake, None, C.byref(d), 320, 1) == 1
    d1 = _d(b=1)
    assert lib.bf_tracker(None, 0, fake, fake, fake, fake, fake, None, C.byref(d), 16) == 1
    assert "n_beams == 1" in native.last_error()
    assert lib.bf_tracker(None, 0, fake, fake, fake, fake, None, None, C.byref(d1), 16) == 1
    assert lib.bf_tracker(None, 5, fake, fake, fake, fake, fake, None, C.byref(d1), 16) == 1
    assert lib.bf_tracker(None, 0, fake, fake, fake, fake, fake, None, C.byref(d1), 0) == 1


def test_grid_pipeline_checks_before_allocating():
    """bf_grid_pipeline_create validates the request before any CUDA call, and
    the chunk length follows lcm(128, integration_spectra)."""
    from beamform_project_b200 import api
    lib = native.lib()
    d = _d(t=32768, b=128)
    h = C.c_void_p()
    assert lib.bf_grid_pipeline_create(C.byref(d), 320, 2, 1000, C.byref(h)) == 1
    assert "multiple of lcm(128, integration_spectra) = 640" in native.last_error()
    assert lib.bf_grid_pipeline_create(C.byref(d), 40, 1, 0, C.byref(h)) == 7
    assert lib.bf_grid_pipeline_create(C.byref(d), 320, 0, 0, C.byref(h)) == 1
    assert lib.bf_grid_pipeline_create(C.byref(d), 320, 1, 0, None) == 1
    assert h.value is None
    assert api.grid_pipeline_chunk_spectra(api.Dimensions(32768, 336, 64, 128), 320, 2) == 1280
    assert api.grid_pipeline_chunk_spectra(api.Dimensions(32768, 336, 64, 128), 10, 1) == 2560
    assert api.grid_pipeline_chunk_spectra(api.Dimensions(700, 336, 32, 8), 320, 1, 6400) == 1280
    assert api.grid_pipeline_chunk_spectra(api.Dimensions(700, 336, 32, 8), 96, 1, 0) == 768
    assert api.grid_pipeline_chunk_spectra(api.Dimensions(700, 336, 32, 8), 320, 1, 100) == 0
    assert lib.bf_grid_pipeline_run(None, None, None, None, None, None) == 1
    assert lib.bf_grid_pipeline_destroy(None) == 0


def test_error_text_is_per_call():
    lib = native.lib()
    bad = _d(t=0)
    assert lib.bf_validate_dimensions(C.byref(bad)) == 1
    good = _d()
    assert lib.bf_validate_dimensions(C.byref(good)) == 0
    assert native.last_error() == ""


def test_python_api_checks_buffers_without_gpu():
    from beamform_project_b200 import api
    with pytest.raises(api.InvalidArgument):
        api.validate_dimensions(api.Dimensions(1, 100, 32, 4))
    assert api.integrated_time_count(32768, 320) == 103
    assert api.integrated_time_count(1024, 10) == 103
    assert api.quantization_layout(api.Dimensions(103, 336, 64, 128)) == (103, 21, 8)
    with pytest.raises(api.InvalidArgument):
        api.integrated_time_count(10, 0)


def test_host_buffer_checks_without_gpu():
    """The host-buffer pipeline's Python wrapper checks dtype, layout and size
    of host arrays before any call into the library."""
    import numpy as np
    from beamform_project_b200 import api
    a = np.zeros(64, np.uint8)
    assert api._host(a, "v", np.uint8, 64) == a.ctypes.data
    with pytest.raises(api.InvalidArgument, match="smaller than dimensions"):
        api._host(a, "v", np.uint8, 65)
    with pytest.raises(api.InvalidArgument, match="contiguous"):
        api._host(np.zeros(64, np.float32), "v", np.uint8, 1)
    with pytest.raises(api.InvalidArgument, match="contiguous"):
        api._host(np.zeros((8, 8), np.uint8)[:, ::2], "v", np.uint8, 1)


def test_doa_track_validates_before_any_cuda_call():
    from beamform_project_b200 import api
    d = api.Dimensions(1024, 336, 32, 1)
    fn = native.lib().bf_doa_track
    for cfg, msg in ((api.doa_track_config(100, subarray=8), "multiple of 128"),
                     (api.doa_track_config(256, subarray=8, grid=1), "grid must be"),
                     (api.doa_track_config(256), "at most 16"),
                     (api.doa_track_config(256, capon=True, subarray=20), "at most 16"),
                     (api.doa_track_config(256, subarray=8, forgetting=0.0), "forgetting")):
        st = fn(None, None, None, None, C.byref(d.c()), C.byref(cfg), None, None, None)
        assert st != 0 and msg in native.last_error(), (msg, native.last_error())
        assert api.doa_track_workspace_bytes(d, cfg) == 0
    ok = api.doa_track_config(256, subarray=8)
    assert api.doa_track_workspace_bytes(d, ok) > 1024 * 336 // 256 * 32 * 32 * 8


def test_doa_slice_entries_validate_before_launch():
    """The channel-slice DOA entries take an even count of 2 to 336 channels;
    the peak entry checks its sizes; nothing reaches the device."""
    lib = native.lib()
    fake = C.c_void_p(4096)
    for f in (3, 338, 0):
        d = Dims(256, f, 64, 1)
        assert lib.bf_doa_covariance_i32_slice(None, fake, fake, C.byref(d), 128) == 1
        assert "even count of 2 to 336" in native.last_error()
    d = Dims(256, 168, 64, 2)
    assert lib.bf_doa_covariance_i32_slice(None, fake, fake, C.byref(d), 128) == 1
    assert "n_beams == 1" in native.last_error()
    d = Dims(256, 168, 64, 1)
    assert lib.bf_doa_scan_slice(None, fake, fake, fake, C.byref(d), 100, 8, 0.9, 1e-3, -0.6, 0.004, 301, 0.0,
                                 fake, fake, fake, fake) == 1
    assert "block_len must divide n_time" in native.last_error()
    # the 336-channel entries keep the reference's dimension contract
    assert lib.bf_doa_covariance_i32(None, fake, fake, C.byref(d), 128) == 1
    assert "336 frequency channels" in native.last_error()
    assert lib.bf_doa_peak(None, fake, fake, 0, 301, -0.6, 0.004, fake) == 1
    assert lib.bf_doa_peak(None, fake, fake, 3, 0, -0.6, 0.004, fake) == 1
