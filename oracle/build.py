"""Build the oracle (test infrastructure only).

    python oracle/build.py

Products (git-ignored; a copy of the checkout used for GPU testing carries
the built files):
    oracle/liboracle.so        C restatement (bf_oracle.c), -ffp-contract=off
    oracle/_ref/libbfref.so    the reference CPU core, compiled directly from the
                               reference checkout's own source files plus
                               ref_shim.cpp; built only when the checkout is
                               present (a machine without it uses the
                               prebuilt file).
    oracle/_ref/beamformer_cpu the reference's CPU command-line beamformer and
    oracle/_ref/run_tracker_stream  tracker (CPU engines), from the same sources
                               plus its tools/beamformer_cpu.cpp and
                               tools/run_tracker_stream.cpp.

    oracle/_ref/libbfref_perf_v3.so, libbfref_perf_v4.so
                               the same CPU core built as the reference's own
                               performance library (beamformer_core_perf,
                               CMakeLists.txt:64-89: -O3, -march, and
                               BEAMFORMER_TRACKER_PERF) for timing only, at
                               x86-64-v3 (AVX2) and x86-64-v4 (AVX-512);
                               oracle/loader.py picks the best one the host
                               runs (-march=native would bind the binary to
                               the machine that built it).
    oracle/_ref/libbfref_cuda.so
                               the reference's own CUDA kernels (grid Direct
                               and Tiled, the int8 quantizer, tracker v5)
                               compiled by nvcc for sm_100a with
                               ref_cuda_shim.cu, for timing them on the same
                               GPU as the B200 kernels.

The reference sources are compiled with g++ / nvcc straight from where they
lie (no CMake, nothing copied).  The checkout is found through
BF_REFERENCE_ROOT, else as the directory `reference` beside the repository
checkout.  -ffp-contract=off keeps the float32 operation order of the source
(no FMA contraction), which is the order the CUDA kernels reproduce;
-march=x86-64-v2 keeps the parity build runnable on any x86-64 host.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("BF_REFERENCE_ROOT") or (HERE.parent.parent / "reference"))
REF_SOURCES = ["cpu_beamformer.cpp", "beam_tracker.cpp", "beam_tracker_opt.cpp",
               "beam_tracker_opt_v2.cpp", "cpu_opt_beam_tracker.cpp", "geometry.cpp",
               "io.cpp", "quantization.cpp", "synthetic_data.cpp", "temporal_integration.cpp",
               "weights.cpp"]
# the reference's CPU command-line programs (tools/), the comparators of the
# B200 command-line drop-ins (the tracker program built without CUDA runs its
# CPU engines)
REF_CLIS = ["beamformer_cpu.cpp", "run_tracker_stream.cpp"]


def _stale(out: Path, deps: list[Path]) -> bool:
    return not out.exists() or any(d.stat().st_mtime > out.stat().st_mtime for d in deps)


def build_oracle() -> Path:
    src = HERE / "bf_oracle.c"
    out = HERE / "liboracle.so"
    if _stale(out, [src]):
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
                        "-fno-fast-math", str(src), "-o", str(out), "-lm"], check=True)
    return out


def build_reference() -> Path | None:
    out = HERE / "_ref" / "libbfref.so"
    srcs = [REF / "src" / s for s in REF_SOURCES]
    if not all(s.exists() for s in srcs):
        return out if out.exists() else None
    shim = HERE / "ref_shim.cpp"
    if _stale(out, srcs + [shim]):
        out.parent.mkdir(exist_ok=True)
        subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
                        "-ffp-contract=off", "-march=x86-64-v2", "-I", str(REF / "include"),
                        *map(str, srcs), str(shim), "-o", str(out)], check=True)
    return out


PERF_LEVELS = ("x86-64-v3", "x86-64-v4")
REF_CUDA_SOURCES = ["cuda_beamformer.cu", "cuda_quantize_int8.cu", "cuda_beam_tracker_v5.cu"]


def build_reference_perf() -> list[Path]:
    """The reference's performance CPU core (timing only, never parity)."""
    outs = []
    srcs = [REF / "src" / s for s in REF_SOURCES]
    shim = HERE / "ref_shim.cpp"
    for level in PERF_LEVELS:
        out = HERE / "_ref" / f"libbfref_perf_{level[-2:]}.so"
        if not all(s.exists() for s in srcs):
            if out.exists():
                outs.append(out)
            continue
        if _stale(out, srcs + [shim]):
            out.parent.mkdir(exist_ok=True)
            subprocess.run(["g++", "-O3", f"-march={level}", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
                            "-DBEAMFORMER_TRACKER_PERF", "-I", str(REF / "include"),
                            *map(str, srcs), str(shim), "-o", str(out)], check=True)
        outs.append(out)
    return outs


def build_reference_cuda() -> Path | None:
    """The reference's CUDA kernels for sm_100a (timing beside the B200 kernels)."""
    out = HERE / "_ref" / "libbfref_cuda.so"
    srcs = [REF / "src" / s for s in REF_CUDA_SOURCES] + [REF / "src" / s for s in REF_SOURCES]
    if not all(s.exists() for s in srcs):
        return out if out.exists() else None
    shim = HERE / "ref_cuda_shim.cu"
    if _stale(out, srcs + [shim]):
        out.parent.mkdir(exist_ok=True)
        nvcc = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
        subprocess.run([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC,-fopenmp", "-shared", "-DBEAMFORMER_HAS_CUDA=1",
                        "-I", str(REF / "include"), "-I", str(REF / "src"),
                        *map(str, srcs), str(shim), "-o", str(out), "-lgomp"], check=True)
    return out


def build_reference_cli() -> list[Path]:
    outs = []
    for cli in REF_CLIS:
        out = HERE / "_ref" / Path(cli).stem
        srcs = [REF / "src" / s for s in REF_SOURCES] + [REF / "tools" / cli]
        if not all(s.exists() for s in srcs):
            if out.exists():
                outs.append(out)
            continue
        if _stale(out, srcs):
            out.parent.mkdir(exist_ok=True)
            subprocess.run(["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-march=x86-64-v2",
                            "-I", str(REF / "include"), *map(str, srcs), "-o", str(out)], check=True)
        outs.append(out)
    return outs


if __name__ == "__main__":
    print(build_oracle())
    print(build_reference())
    print(build_reference_cli())
    print(build_reference_perf())
    print(build_reference_cuda())
    sys.exit(0)
