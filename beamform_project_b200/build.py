"""Build the native libraries in-tree (no JIT cache, so the .so files travel).

    python -m beamform_project_b200.build          # product library (nvcc, sm_100a)

Products:
    beamform_project_b200/lib/libbf_b200.so   C ABI of include/bf_b200.h + kernels
    beamform_project_b200/lib/libbf_cxx.so    C++ API of include/beamformer/ over the C ABI
    beamform_project_b200/bin/beamformer_cuda command-line beamformer (the reference CLI's options)
    beamform_project_b200/bin/run_tracker_stream command-line tracker (the reference CLI's options)

The oracle (test infrastructure) is built by oracle/build.py.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"] + ARCH

CUDA_SOURCES = ["capi.cu", "grid_exact.cu", "quantize.cu", "generate.cu", "tracker.cu",
                "tracker_stream.cu", "grid_tc.cu", "no_alloc.cu", "doa_cov.cu", "doa_scan.cu",
                "serve_kernels.cu", "serve.cu", "selftest.cu", "loss_mask.cu", "pipeline.cu", "grid_cov.cu",
                "autotune.cu", "doa_track.cu"]
CXX_SOURCES = ["cxx_api.cpp", "io.cpp"]
CLI = PKG / "cli"
BIN = PKG / "bin"
CLI_PROGRAMS = ["beamformer_cuda", "run_tracker_stream"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or Path(cand).exists()):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str], log: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    log: list[str] = []
    headers = list(CSRC.glob("*.cuh")) + [INCLUDE / "bf_b200.h"]
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = obj_dir / (s.stem + ".o")
        if force or _stale(o, [s] + headers):
            _run([nvcc, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)], log)
        objs.append(o)
    so = LIB / "libbf_b200.so"
    if force or _stale(so, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(so), *map(str, objs), "-lcudart"], log)
    cxx_srcs = [CSRC / s for s in CXX_SOURCES if (CSRC / s).exists()]
    if cxx_srcs:
        cxx_so = LIB / "libbf_cxx.so"
        cxx_headers = list((INCLUDE / "beamformer").glob("*.hpp"))
        if force or _stale(cxx_so, cxx_srcs + cxx_headers + [so]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", str(INCLUDE),
                  "-I", "/usr/local/cuda/include", *map(str, cxx_srcs), "-o", str(cxx_so),
                  "-L", str(LIB), "-lbf_b200", "-Wl,-rpath,$ORIGIN",
                  "-L", "/usr/local/cuda/lib64", "-lcudart"], log)
        # command-line programs over the C++ API (beamform_project_b200/bin)
        BIN.mkdir(exist_ok=True)
        for prog in CLI_PROGRAMS:
            src = CLI / f"{prog}.cpp"
            out = BIN / prog
            if force or _stale(out, [src, cxx_so] + cxx_headers):
                _run(["g++", "-O2", "-std=c++17", "-I", str(INCLUDE), "-I", "/usr/local/cuda/include",
                      str(src), "-o", str(out), "-L", str(LIB), "-lbf_cxx", "-lbf_b200",
                      "-Wl,-rpath,$ORIGIN/../lib", "-L", "/usr/local/cuda/lib64", "-lcudart"], log)
        # C++ test programs (tests/cxx), built here so they ship with the libraries
        for name in ("test_cxx_api", "test_io"):
            test_src = ROOT / "tests" / "cxx" / f"{name}.cpp"
            test_bin = obj_dir / name
            if test_src.exists() and (force or _stale(test_bin, [test_src, cxx_so] + cxx_headers)):
                _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(INCLUDE),
                      "-I", "/usr/local/cuda/include", str(test_src), "-o", str(test_bin),
                      "-L", str(LIB), "-lbf_cxx", "-lbf_b200", f"-Wl,-rpath,{LIB}",
                      "-L", "/usr/local/cuda/lib64", "-lcudart"], log)
    (obj_dir / "build.log").write_text("\n".join(log))
    if verbose:
        print("\n".join(log))
    return so


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print("built", LIB / "libbf_b200.so")
