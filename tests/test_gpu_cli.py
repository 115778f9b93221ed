"""The command-line drop-in (beamform_project_b200/bin/beamformer_cuda) on
files, against the reference's own CPU command-line beamformer
(oracle/_ref/beamformer_cpu, built from its tools/beamformer_cpu.cpp) and
the reference's integration and quantizer on the same inputs."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import random_voltage, rng

ROOT = Path(__file__).resolve().parent.parent
CLI = ROOT / "beamform_project_b200" / "bin" / "beamformer_cuda"
REF_CLI = ROOT / "oracle" / "_ref" / "beamformer_cpu"
F = 336
T, A, B = 640, 64, 37


def _files(tmp: Path):
    v = random_voltage(T, F, A, seed=21)
    ph = rng(22).random((B, F, A)) * 2 * np.pi
    w = np.stack([np.cos(ph), np.sin(ph)], -1).astype(np.float32)   # [B][F][A][re, im]
    tiles = -(-B // 32)
    tw = np.zeros((F, tiles, A, 32, 2), np.float32)                  # [F][tile][A][32][re, im]
    for b in range(B):
        tw[:, b // 32, :, b % 32, :] = w[b]
    paths = {"v": tmp / "voltage.bin", "w": tmp / "weights.bin", "tw": tmp / "tiled.bin"}
    v.tofile(paths["v"])
    w.tofile(paths["w"])
    tw.tofile(paths["tw"])
    return v, w, paths


def _run(prog: Path, *args) -> subprocess.CompletedProcess:
    assert prog.exists(), f"{prog} is not built"
    return subprocess.run([str(prog), *map(str, args)], capture_output=True, text=True, timeout=600)


def _common(paths, weights_key="w"):
    return ["--input", paths["v"], "--weights", paths[weights_key], "--n-time", T, "--n-ant", A, "--n-beams", B]


@pytest.mark.gpu
def test_float32_output_equals_reference_cli(cuda, ref, tmp_path):
    v, w, paths = _files(tmp_path)
    ref_out, out_d, out_t = tmp_path / "ref.f32", tmp_path / "direct.f32", tmp_path / "tiled.f32"
    r = _run(REF_CLI, *_common(paths), "--output", ref_out)
    assert r.returncode == 0, r.stderr
    r = _run(CLI, *_common(paths), "--output", out_d, "--kernel", "direct", "--metrics", tmp_path / "m.csv")
    assert r.returncode == 0, r.stderr
    assert "CUDA beamforming complete: kernel=direct" in r.stdout and "peak_integrated_beam=" in r.stdout
    r = _run(CLI, *_common(paths, "tw"), "--output", out_t, "--kernel", "tiled", "--metrics", tmp_path / "m.csv")
    assert r.returncode == 0, r.stderr
    expect = np.fromfile(ref_out, np.float32)
    assert expect.size == T * F * B
    assert np.array_equal(np.fromfile(out_d, np.float32), expect)
    assert np.array_equal(np.fromfile(out_t, np.float32), expect)
    rows = (tmp_path / "m.csv").read_text().splitlines()
    assert rows[0].startswith("backend,n_time,n_freq,n_ant,n_beams,load_ms") and len(rows) == 3
    assert rows[1].startswith(f"cuda,{T},{F},{A},{B},")


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,S", [("direct", 320), ("tiled", 10), ("tiled", 320)])
def test_int8_output_equals_reference_quantizer(cuda, ref, tmp_path, kernel, S):
    v, w, paths = _files(tmp_path)
    out, par, meta = tmp_path / "codes.i8", tmp_path / "params.f32", tmp_path / "meta.txt"
    r = _run(CLI, *_common(paths, "tw" if kernel == "tiled" else "w"), "--output", out, "--kernel", kernel,
             "--integration-spectra", S, "--output-format", "int8", "--quantization-params", par,
             "--quantization-metadata", meta, "--shard-id", 1)
    assert r.returncode == 0, r.stderr
    W = -(-T // S)
    I = ref.ref_beamform(v, w, T, F, A, B)
    integ = ref.ref_integrate(I, T, F, A, B, S)
    codes, params = ref.ref_quantize(integ, W, F, A, B)
    assert np.array_equal(np.fromfile(out, np.int8).reshape(W, F, B), codes)
    assert np.array_equal(np.fromfile(par, np.float32).reshape(params.shape), params)
    m = dict(line.split("=", 1) for line in meta.read_text().splitlines())
    assert m["format"] == "beamformer-quantized-int8-v1" and m["parameters_file"] == "params.f32"
    assert (m["n_time"], m["input_n_time"], m["integration_spectra"], m["shard_id"]) == (str(W), str(T), str(S), "1")


@pytest.mark.gpu
def test_tensor_kernel_within_split_precision_bar(cuda, orc, tmp_path):
    v, w, paths = _files(tmp_path)
    out = tmp_path / "tensor.f32"
    r = _run(CLI, *_common(paths), "--output", out, "--kernel", "tensor", "--integration-spectra", 320)
    assert r.returncode == 0, r.stderr
    assert "kernel=tensor" in r.stdout
    got = np.fromfile(out, np.float32).reshape(T // 320, F, B).astype(np.float64)
    exp = orc.beamform_integrated(v, w, T, F, A, B, 320, f64=True)
    assert np.all(np.abs(got - exp) <= 1e-3 + 1e-5 * np.abs(exp))


@pytest.mark.gpu
def test_covariance_kernel_within_bar(cuda, orc, tmp_path):
    v, w, paths = _files(tmp_path)
    out = tmp_path / "cov.f32"
    r = _run(CLI, *_common(paths), "--output", out, "--kernel", "covariance", "--integration-spectra", 320)
    assert r.returncode == 0, r.stderr
    assert "kernel=covariance" in r.stdout
    got = np.fromfile(out, np.float32).reshape(T // 320, F, B).astype(np.float64)
    exp = orc.beamform_integrated(v, w, T, F, A, B, 320, f64=True)
    assert np.all(np.abs(got - exp) <= 1e-3 + 1e-5 * np.abs(exp))


@pytest.mark.gpu
def test_errors_exit_one_with_message(cuda, tmp_path):
    _, _, paths = _files(tmp_path)
    r = _run(CLI, *_common(paths), "--output", tmp_path / "x", "--output-format", "int8")
    assert r.returncode == 1 and "int8 output requires --integration-spectra" in r.stderr
    r = _run(CLI, "--input", paths["v"], "--weights", paths["w"], "--output", tmp_path / "x", "--n-time", T + 1,
             "--n-ant", A, "--n-beams", B)
    assert r.returncode == 1 and "bytes; expected" in r.stderr
    r = _run(CLI, *_common(paths), "--output", tmp_path / "x", "--kernel", "warp")
    assert r.returncode == 1 and "kernel must be" in r.stderr


TRK = ROOT / "beamform_project_b200" / "bin" / "run_tracker_stream"
REF_TRK = ROOT / "oracle" / "_ref" / "run_tracker_stream"


@pytest.mark.gpu
@pytest.mark.parametrize("engine,spectra", [("cuda_fws", 320), ("cuda_v5", 10)])
def test_tracker_cli_within_reference_gpu_tolerance(cuda, ref, tmp_path, engine, spectra):
    """The tracker drop-in against the reference's CPU engine (cpu_v2), with
    the tolerance the reference's own GPU tracker tests use (|d| <= 1e-4 or
    |d| <= 1e-3 |ref|)."""
    Tt, At = 2048, 64
    pos = ref.ref_default_positions(At)
    freq = ref.ref_channelized_frequencies(F)
    v = ref.ref_make_moving_point_source(Tt, F, At, pos, freq, 0.05, -0.02, 2e-5, 1e-5, 3.0)
    src = tmp_path / "v.bin"
    v.tofile(src)
    args = ["--n-time", Tt, "--n-ant", At, "--spectra", spectra, "--source-l0", 0.05, "--source-m0", -0.02,
            "--source-dl", 2e-5, "--source-dm", 1e-5, "--input", src]
    r = _run(REF_TRK, "--engine", "cpu_v2", *args, "--output", tmp_path / "ref.f32")
    assert r.returncode == 0, r.stderr
    r = _run(TRK, "--engine", engine, *args, "--output", tmp_path / "b200.f32")
    assert r.returncode == 0, r.stderr
    assert f"Successfully ran {engine}" in r.stdout
    exp = np.fromfile(tmp_path / "ref.f32", np.float32)
    got = np.fromfile(tmp_path / "b200.f32", np.float32)
    assert got.size == exp.size == Tt * F
    d = np.abs(got - exp)
    assert np.all((d <= 1e-4) | (d <= 1e-3 * exp)), float((d / np.maximum(exp, 1e-30)).max())


@pytest.mark.gpu
def test_tracker_cli_errors(cuda, tmp_path):
    src = tmp_path / "v.bin"
    random_voltage(100, F, 32, seed=1).tofile(src)
    r = _run(TRK, "--engine", "cpu_v2", "--n-time", 100, "--n-ant", 32, "--input", src, "--output", tmp_path / "o")
    assert r.returncode == 1 and "Unknown engine or CUDA unavailable: cpu_v2" in r.stderr
    r = _run(TRK, "--n-time", 101, "--n-ant", 32, "--input", src, "--output", tmp_path / "o")
    assert r.returncode == 1 and "does not match expected" in r.stderr
    r = _run(TRK, "--n-time", 100)
    assert r.returncode == 1 and "--input and --output are required" in r.stderr
