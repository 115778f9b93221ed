"""ctypes access to the oracle (test infrastructure).

liboracle.so  - C restatement of the reference hot path (oracle/bf_oracle.c)
libbfref.so   - the reference CPU core compiled from its sources (oracle/_ref)
libbfref_perf_v3/v4.so - the same core built as the reference's performance
                library (-O3, -march x86-64-v3 / v4): timing only
libbfref_cuda.so - the reference's own CUDA kernels for sm_100a: timing only

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module.  It is the checker, never the thing measured as the product.
"""
from __future__ import annotations

import contextlib
import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
_ORACLE = ROOT / "oracle" / "liboracle.so"
_REF = ROOT / "oracle" / "_ref" / "libbfref.so"
_o = None
_r = None

P = C.c_void_p
U64 = C.c_uint64
F32 = C.c_float


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def oracle() -> C.CDLL:
    global _o
    if _o is None:
        if not _ORACLE.exists():
            import subprocess, sys
            subprocess.run([sys.executable, str(ROOT / "oracle" / "build.py")], check=True)
        o = C.CDLL(str(_ORACLE))
        o.orc_generate_weights.argtypes = [U64, U64, U64, P, P, P, P]
        o.orc_beamform_packed_intensity.argtypes = [P, P, U64, U64, U64, U64, P]
        o.orc_window_count.argtypes = [U64, U64]
        o.orc_window_count.restype = U64
        o.orc_integrate.argtypes = [P, U64, U64, U64, U64, P]
        o.orc_beamform_integrated.argtypes = [P, P, U64, U64, U64, U64, U64, P, U64, P]
        o.orc_beamform_integrated_f64.argtypes = [P, P, U64, U64, U64, U64, U64, P, U64, P]
        o.orc_quantize.argtypes = [P, U64, U64, U64, P, P]
        o.orc_direction_from_lm.argtypes = [F32, F32, P]
        o.orc_tracker_window_directions.argtypes = [F32, F32, F32, F32, U64, U64, P]
        o.orc_tracker_weights.argtypes = [U64, U64, U64, P, P, P, P]
        o.orc_tracker.argtypes = [P, P, U64, U64, U64, U64, P]
        o.orc_generate_voltage.argtypes = [U64, U64, U64, U64, U64, F32, P, U64, P]
        o.orc_covariance_block_i64.argtypes = [P, U64, U64, U64, P]
        D = C.c_double
        o.orc_doa_scan.argtypes = [P, U64, U64, U64, U64, U64, D, D, P, P, D, D, U64, D, P, P, P]
        o.orc_unpack.argtypes = [P, U64, P, P]
        o.orc_pack.argtypes = [C.c_int, C.c_int]
        _o = o
    return _o


def reference_available() -> bool:
    return _REF.exists()


def reference() -> C.CDLL:
    """The parity build of the reference CPU core (-ffp-contract=off)."""
    global _r
    if _r is None:
        _r = _bind_reference(C.CDLL(str(_REF)))
    return _r


_rp = None
_rp_level = None


def _host_cpu_flags() -> set[str]:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def reference_perf_level() -> str:
    """The best performance build of the reference core this host can run."""
    flags = _host_cpu_flags()
    v4 = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}
    v3 = {"avx2", "fma", "bmi1", "bmi2", "movbe"}
    base = ROOT / "oracle" / "_ref"
    if v4 <= flags and (base / "libbfref_perf_v4.so").exists():
        return "x86-64-v4"
    if v3 <= flags and (base / "libbfref_perf_v3.so").exists():
        return "x86-64-v3"
    return "x86-64-v2"


def reference_perf() -> C.CDLL:
    """The reference CPU core as its own performance library builds it (-O3,
    -march at the host's level): the timed CPU baseline.  Falls back to the
    parity build on a host below x86-64-v3."""
    global _rp, _rp_level
    if _rp is None:
        _rp_level = reference_perf_level()
        if _rp_level == "x86-64-v2":
            _rp = reference()
        else:
            _rp = _bind_reference(C.CDLL(str(ROOT / "oracle" / "_ref" / f"libbfref_perf_{_rp_level[-2:]}.so")))
    return _rp


def reference_perf_flags() -> str:
    reference_perf()
    if _rp_level == "x86-64-v2":
        return "g++ -O3 -march=x86-64-v2 -ffp-contract=off (parity build; host below x86-64-v3)"
    return f"g++ -O3 -march={_rp_level} -DBEAMFORMER_TRACKER_PERF -fopenmp (beamformer_core_perf flags)"


_rg = None


def reference_gpu_available() -> bool:
    return (ROOT / "oracle" / "_ref" / "libbfref_cuda.so").exists()


def reference_gpu() -> C.CDLL:
    """The reference's own CUDA kernels (src/cuda_beamformer.cu,
    src/cuda_quantize_int8.cu, src/cuda_beam_tracker_v5.cu) built for
    sm_100a: timed beside the B200 kernels, never used as a checker."""
    global _rg
    if _rg is None:
        g = C.CDLL(str(ROOT / "oracle" / "_ref" / "libbfref_cuda.so"))
        g.refgpu_last_error.restype = C.c_char_p
        g.refgpu_grid_integrated.argtypes = [C.c_int, P, P, P, P, U64, U64, U64, U64, U64]
        g.refgpu_quantize.argtypes = [P, P, P, P, U64, U64, U64, U64]
        g.refgpu_tracker_v5.argtypes = [P, P, U64, U64, U64, F32, F32, F32, F32, U64, U64, U64, P]
        _rg = g
    return _rg


def refgpu_check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"reference CUDA error {rc}: {reference_gpu().refgpu_last_error().decode()}")


def _bind_reference(r: C.CDLL) -> C.CDLL:
    r.ref_last_error.restype = C.c_char_p
    r.ref_cpu_beamform_packed_intensity.argtypes = [P, P, U64, U64, U64, U64, P]
    r.ref_cpu_integrate.argtypes = [P, U64, U64, U64, U64, U64, P]
    r.ref_cpu_quantize.argtypes = [P, U64, U64, U64, U64, P, P]
    r.ref_generate_weights.argtypes = [U64, U64, U64, P, P, P, P]
    r.ref_generate_tiled_weights.argtypes = [U64, U64, U64, P, P, P, P]
    r.ref_default_positions.argtypes = [U64, P]
    r.ref_channelized_frequencies.argtypes = [U64, P]
    r.ref_tracker_window_direction.argtypes = [F32, F32, F32, F32, U64, U64, P]
    r.ref_beam_tracker.argtypes = [C.c_int, P, U64, U64, U64, F32, F32, F32, F32, U64, P]
    r.ref_make_noise.argtypes = [U64, U64, U64, C.c_uint32, P]
    r.ref_make_one_hot.argtypes = [U64, U64, U64, U64, U64, U64, C.c_int, C.c_int, P]
    r.ref_make_point_source.argtypes = [U64, U64, U64, P, P, P, F32, P]
    r.ref_make_moving_point_source.argtypes = [U64, U64, U64, P, P, F32, F32, F32, F32, F32, P]
    r.ref_set_threads.argtypes = [C.c_int]
    r.ref_doa_directions.argtypes = [P, U64, U64, U64, P, P, C.c_int, U64, U64, F32, F32, U64, F32,
                                     F32, U64, F32, F32, P, P]
    r.ref_io_write.argtypes = [C.c_char_p, P, P, P, P, P, P, P] + [U64] * 9
    r.ref_io_read_check.argtypes = [C.c_char_p, P, P, P, P, P, P] + [U64] * 9
    return r


_timing = False


@contextlib.contextmanager
def perf_build():
    """Route the ref_* wrappers to the performance build of the reference core
    (the timed CPU baselines); parity checks use the default parity build."""
    global _timing
    prev = _timing
    _timing = True
    try:
        yield reference_perf()
    finally:
        _timing = prev


def _lib() -> C.CDLL:
    return reference_perf() if _timing else reference()


def _rcheck(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"reference error {rc}: {_lib().ref_last_error().decode()}")


# ---------------- oracle wrappers ----------------

def generate_weights(pos, freq, dirs) -> np.ndarray:
    A, F, B = len(pos), len(freq), len(dirs)
    out = np.zeros((B, F, A, 2), np.float32)
    oracle().orc_generate_weights(A, F, B, _ptr(np.ascontiguousarray(pos, np.float32)),
                                  _ptr(np.ascontiguousarray(freq, np.float32)),
                                  _ptr(np.ascontiguousarray(dirs, np.float32)), _ptr(out))
    return out


def beamform(v: np.ndarray, w: np.ndarray, T, F, A, B) -> np.ndarray:
    out = np.zeros((T, F, B), np.float32)
    oracle().orc_beamform_packed_intensity(_ptr(v), _ptr(w), T, F, A, B, _ptr(out))
    return out


def integrate(I: np.ndarray, T, F, B, S) -> np.ndarray:
    W = -(-T // S)
    out = np.zeros((W, F, B), np.float32)
    oracle().orc_integrate(_ptr(np.ascontiguousarray(I, np.float32)), T, F, B, S, _ptr(out))
    return out


def beamform_integrated(v, w, T, F, A, B, S, windows=None, f64=False) -> np.ndarray:
    W = -(-T // S)
    wl = None if windows is None else np.ascontiguousarray(windows, np.int64)
    out = np.zeros((W, F, B), np.float64 if f64 else np.float32)
    fn = oracle().orc_beamform_integrated_f64 if f64 else oracle().orc_beamform_integrated
    fn(_ptr(v), _ptr(w), T, F, A, B, S, _ptr(wl), 0 if wl is None else len(wl), _ptr(out))
    return out


def quantize(I: np.ndarray, W, F, B):
    ft, bt = -(-F // 16), -(-B // 16)
    codes = np.zeros((W, F, B), np.int8)
    params = np.zeros((W, ft, bt, 2), np.float32)
    oracle().orc_quantize(_ptr(np.ascontiguousarray(I, np.float32)), W, F, B, _ptr(codes), _ptr(params))
    return codes, params


def tracker_weights(dirs, pos, freq) -> np.ndarray:
    W, A, F = len(dirs), len(pos), len(freq)
    out = np.zeros((W, F, A, 2), np.float32)
    oracle().orc_tracker_weights(W, F, A, _ptr(np.ascontiguousarray(pos, np.float32)),
                                 _ptr(np.ascontiguousarray(freq, np.float32)),
                                 _ptr(np.ascontiguousarray(dirs, np.float32)), _ptr(out))
    return out


def tracker(v, window_weights, T, F, A, S) -> np.ndarray:
    out = np.zeros((T, F), np.float32)
    oracle().orc_tracker(_ptr(v), _ptr(np.ascontiguousarray(window_weights, np.float32)), T, F, A,
                         S, _ptr(out))
    return out


def generate_voltage(seed, offset, T, F, A, scale, mu=None, epoch_len=1) -> np.ndarray:
    out = np.zeros((T, F, A), np.uint8)
    m = None if mu is None else np.ascontiguousarray(mu, np.float32)
    oracle().orc_generate_voltage(seed, offset, T, F, A, scale, _ptr(m), epoch_len, _ptr(out))
    return out


def covariance_block(v, T, F, A) -> np.ndarray:
    R = np.zeros((F, A, A, 2), np.int64)
    oracle().orc_covariance_block_i64(_ptr(v), T, F, A, _ptr(R))
    return R


def covariance_blocks(v: np.ndarray, K: int) -> np.ndarray:
    """[B][F][A][A][2] int64 block sums of x x^H (blocks of K spectra)."""
    T, F, A = v.shape
    B = T // K
    out = np.zeros((B, F, A, A, 2), np.int64)
    for b in range(B):
        out[b] = covariance_block(np.ascontiguousarray(v[b * K:(b + 1) * K]), K, F, A)
    return out


def doa_scan(R: np.ndarray, K: int, subarray: int, lam: float, load: float, pos_sub: np.ndarray,
             kw: np.ndarray, l_first: float, l_step: float, n: int, m_fixed: float = 0.0):
    """FP64 smoothing / forgetting / Bartlett / Capon scan (orc_doa_scan)."""
    R = np.ascontiguousarray(R, np.int64)
    B, F, A = R.shape[0], R.shape[1], R.shape[2]
    bart = np.zeros((B, n), np.float64)
    cap = np.zeros((B, n), np.float64)
    lest = np.zeros((B, 2), np.float64)
    oracle().orc_doa_scan(_ptr(R), B, F, A, K, subarray, lam, load,
                          _ptr(np.ascontiguousarray(pos_sub, np.float32)),
                          _ptr(np.ascontiguousarray(kw, np.float64)), l_first, l_step, n, m_fixed,
                          _ptr(bart), _ptr(cap), _ptr(lest))
    return bart, cap, lest


def ref_doa_directions(v, pos, freq, K, capon=False, G=16, levels=2, fov_l=0.2, fov_m=0.2,
                       subarray=0, lam=1.0, load=1e-3, l0=0.0, m0=0.0, intensity=False):
    """CpuOptBeamTracker's per-window directions [W][3] (and, with
    intensity=True, its emitted [T][F] beam power as a second value)."""
    T, F, A = v.shape
    W = -(-T // K)
    out = np.zeros((W, 3), np.float32)
    inten = np.zeros((T, F), np.float32) if intensity else None
    _rcheck(_lib().ref_doa_directions(_ptr(np.ascontiguousarray(v)), T, F, A,
                                      _ptr(np.ascontiguousarray(pos, np.float32)),
                                      _ptr(np.ascontiguousarray(freq, np.float32)), int(capon), G,
                                      levels, fov_l, fov_m, subarray, lam, load, K, l0, m0, _ptr(out),
                                      _ptr(inten)))
    return (out, inten) if intensity else out


def unpack(v: np.ndarray):
    re = np.zeros(v.shape, np.int8)
    im = np.zeros(v.shape, np.int8)
    oracle().orc_unpack(_ptr(np.ascontiguousarray(v)), v.size, _ptr(re), _ptr(im))
    return re, im


# ---------------- reference wrappers ----------------

def ref_io_write(dirpath, arrays: dict, case: tuple) -> None:
    """Every on-disk format written by the reference's src/io.cpp (ref_shim.cpp)."""
    a = arrays
    _rcheck(_lib().ref_io_write(str(dirpath).encode(), _ptr(a["voltage"]), _ptr(a["weights"]), _ptr(a["tiled"]),
                                     _ptr(a["intensity"]), _ptr(a["codes"]), _ptr(a["params"]), _ptr(a["loss"]),
                                     *case))


def ref_io_read_check(dirpath, arrays: dict, case: tuple) -> None:
    """The reference's readers on dirpath; raises unless the contents equal arrays."""
    a = arrays
    _rcheck(_lib().ref_io_read_check(str(dirpath).encode(), _ptr(a["voltage"]), _ptr(a["weights"]),
                                          _ptr(a["tiled"]), _ptr(a["codes"]), _ptr(a["params"]), _ptr(a["loss"]),
                                          *case))


def ref_beamform(v, w, T, F, A, B) -> np.ndarray:
    out = np.zeros((T, F, B), np.float32)
    _rcheck(_lib().ref_cpu_beamform_packed_intensity(_ptr(v), _ptr(w), T, F, A, B, _ptr(out)))
    return out


def ref_integrate(I, T, F, A, B, S) -> np.ndarray:
    out = np.zeros((-(-T // S), F, B), np.float32)
    _rcheck(_lib().ref_cpu_integrate(_ptr(np.ascontiguousarray(I, np.float32)), T, F, A, B, S, _ptr(out)))
    return out


def ref_quantize(I, W, F, A, B):
    codes = np.zeros((W, F, B), np.int8)
    params = np.zeros((W, -(-F // 16), -(-B // 16), 2), np.float32)
    _rcheck(_lib().ref_cpu_quantize(_ptr(np.ascontiguousarray(I, np.float32)), W, F, A, B,
                                         _ptr(codes), _ptr(params)))
    return codes, params


def ref_generate_weights(pos, freq, dirs, tiled=False) -> np.ndarray:
    A, F, B = len(pos), len(freq), len(dirs)
    if tiled:
        out = np.zeros((F, -(-B // 32), A, 32, 2), np.float32)
        fn = _lib().ref_generate_tiled_weights
    else:
        out = np.zeros((B, F, A, 2), np.float32)
        fn = _lib().ref_generate_weights
    _rcheck(fn(A, F, B, _ptr(np.ascontiguousarray(pos, np.float32)),
               _ptr(np.ascontiguousarray(freq, np.float32)),
               _ptr(np.ascontiguousarray(dirs, np.float32)), _ptr(out)))
    return out


def ref_default_positions(A) -> np.ndarray:
    out = np.zeros((A, 3), np.float32)
    _rcheck(_lib().ref_default_positions(A, _ptr(out)))
    return out


def ref_channelized_frequencies(F) -> np.ndarray:
    out = np.zeros(F, np.float32)
    _rcheck(_lib().ref_channelized_frequencies(F, _ptr(out)))
    return out


def ref_tracker(v, T, F, A, l0, m0, rl, rm, S, variant=0) -> np.ndarray:
    out = np.zeros((T, F), np.float32)
    _rcheck(_lib().ref_beam_tracker(variant, _ptr(v), T, F, A, l0, m0, rl, rm, S, _ptr(out)))
    return out


def ref_tracker_window_direction(l0, m0, rl, rm, window, S) -> np.ndarray:
    out = np.zeros(3, np.float32)
    _rcheck(_lib().ref_tracker_window_direction(l0, m0, rl, rm, window, S, _ptr(out)))
    return out


def ref_make_noise(T, F, A, seed) -> np.ndarray:
    out = np.zeros((T, F, A), np.uint8)
    _rcheck(_lib().ref_make_noise(T, F, A, seed, _ptr(out)))
    return out


def ref_make_one_hot(T, F, A, t, f, a, re=3, im=-2) -> np.ndarray:
    out = np.zeros((T, F, A), np.uint8)
    _rcheck(_lib().ref_make_one_hot(T, F, A, t, f, a, re, im, _ptr(out)))
    return out


def ref_make_point_source(T, F, A, pos, freq, direction, amplitude=4.0) -> np.ndarray:
    out = np.zeros((T, F, A), np.uint8)
    _rcheck(_lib().ref_make_point_source(
        T, F, A, _ptr(np.ascontiguousarray(pos, np.float32)),
        _ptr(np.ascontiguousarray(freq, np.float32)),
        _ptr(np.ascontiguousarray(direction, np.float32)), amplitude, _ptr(out)))
    return out


def ref_make_moving_point_source(T, F, A, pos, freq, l0, m0, rl, rm, amplitude=4.0) -> np.ndarray:
    out = np.zeros((T, F, A), np.uint8)
    _rcheck(_lib().ref_make_moving_point_source(
        T, F, A, _ptr(np.ascontiguousarray(pos, np.float32)),
        _ptr(np.ascontiguousarray(freq, np.float32)), l0, m0, rl, rm, amplitude, _ptr(out)))
    return out
