"""The C++ drop-in API (include/beamformer/) through its own test program
(tests/cxx/test_cxx_api.cpp, built by beamform_project_b200.build)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "beamform_project_b200" / "_build" / "test_cxx_api"


def test_cxx_headers_compile_without_cuda_device():
    """The headers are self-contained C++17 (CPU-only check)."""
    src = "\n".join(f'#include "beamformer/{h.name}"'
                    for h in sorted((ROOT / "include" / "beamformer").glob("*.hpp")))
    res = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(ROOT / "include"),
                          "-I", "/usr/local/cuda/include", "-x", "c++", "-"], input=src,
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


@pytest.mark.gpu
def test_cxx_api_program(cuda):
    assert BIN.exists(), "run python -m beamform_project_b200.build"
    res = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "ALL OK" in res.stdout
