"""On-disk formats (include/beamformer/io.hpp, beamform_project_b200/csrc/io.cpp)
against the reference's own src/io.cpp (compiled into oracle/_ref): the same
inputs give byte-identical files, each side reads the other's, and the error
behaviour (exception types, the file-size check) holds.  CPU only."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rng

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "beamform_project_b200" / "_build" / "test_io"
FILES = ["voltage.bin", "weights.bin", "tiled.bin", "intensity.bin", "codes.bin", "params.bin",
         "int8_meta.txt", "shard_payload.bin", "shard_meta.txt", "shard_loss.bin"]


def _case(T=23, A=32, B=37, S=10, shard_id=1, ts_start=123456789012345, ts_step=3, loss_id=42, seed=0):
    F = 336
    g = rng(seed)
    W = -(-T // S)
    arrays = {
        "voltage": g.integers(0, 256, size=T * F * A, dtype=np.uint8),
        "weights": g.standard_normal(B * F * A * 2).astype(np.float32),
        "tiled": g.standard_normal(F * (-(-B // 32)) * A * 32 * 2).astype(np.float32),
        "intensity": (g.random(T * F * B) * 1e4).astype(np.float32),
        "codes": g.integers(-128, 128, size=W * F * B, dtype=np.int8),
        "params": g.standard_normal(W * (-(-F // 16)) * (-(-B // 16)) * 2).astype(np.float32),
        "loss": (g.random(T * F) > 0.1).astype(np.uint8),
    }
    case = (T, F, A, B, S, shard_id, ts_start, ts_step, loss_id)
    return arrays, case


def _src(tmp: Path, arrays, case) -> Path:
    src = tmp / "src"
    src.mkdir()
    for k, v in arrays.items():
        v.tofile(src / f"{k}.raw")
    (src / "dims.txt").write_text(" ".join(map(str, case)) + "\n")
    return src


def _run(*args) -> str:
    assert BIN.exists(), "run python -m beamform_project_b200.build"
    res = subprocess.run([str(BIN), *map(str, args)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    return res.stdout


@pytest.mark.parametrize("params", [dict(), dict(T=320, A=64, B=128, S=320, shard_id=0, ts_start=0, ts_step=1,
                                                 loss_id=0, seed=1)])
def test_files_identical_to_reference_and_cross_readable(ref, tmp_path, params):
    arrays, case = _case(**params)
    src = _src(tmp_path, arrays, case)
    mine, theirs = tmp_path / "mine", tmp_path / "ref"
    mine.mkdir()
    theirs.mkdir()
    assert "WRITE OK" in _run("write", src, mine)
    ref.ref_io_write(theirs, arrays, case)
    for name in FILES:
        a, b = (mine / name).read_bytes(), (theirs / name).read_bytes()
        assert a == b, f"{name} differs ({len(a)} vs {len(b)} bytes)"
    # each side reads the other's files
    assert "READ OK" in _run("read", src, theirs)
    ref.ref_io_read_check(mine, arrays, case)


def test_metadata_text(tmp_path):
    arrays, case = _case()
    src = _src(tmp_path, arrays, case)
    out = tmp_path / "out"
    out.mkdir()
    _run("write", src, out)
    meta = dict(line.split("=", 1) for line in (out / "int8_meta.txt").read_text().splitlines())
    assert meta["format"] == "beamformer-quantized-int8-v1"
    assert meta["parameters_format"] == "little-endian-float32[offset,scale]"
    assert (meta["n_time"], meta["input_n_time"], meta["integration_spectra"]) == ("3", "23", "10")
    assert (meta["chunk_time"], meta["chunk_frequency"], meta["chunk_beam"], meta["invalid_code"]) == \
        ("1", "16", "16", "-128")
    assert meta["parameters_count"] == str(3 * 21 * 3)
    assert meta["timestamp_start"] == "123456789012345" and meta["absolute_frequency_start"] == "336"
    shard = dict(line.split("=", 1) for line in (out / "shard_meta.txt").read_text().splitlines())
    assert shard["format"] == "beamformer-packed-shard-v1"
    assert shard["payload_bytes"] == str(23 * 336 * 32) and shard["loss_mask_bytes"] == str(23 * 336)


def test_error_behaviour(tmp_path):
    assert "ERRORS OK" in _run("errors", tmp_path)


def _py_write(out: Path, arrays, case):
    from beamform_project_b200 import io as bio
    T, F, A, B, S, shard_id, ts_start, ts_step, loss_id = case
    d = bio.Dimensions(T, F, A, B)
    W = bio.integrated_time_count(T, S)
    wd = bio.Dimensions(W, F, A, B)
    bio.write_packed_voltage(out / "voltage.bin", arrays["voltage"], d)
    bio.write_weights(out / "weights.bin", arrays["weights"].reshape(-1, 2), d)
    bio.write_tiled_weights(out / "tiled.bin", arrays["tiled"].reshape(-1, 2), d)
    bio.write_intensities(out / "intensity.bin", arrays["intensity"], d)
    bio.write_quantized_intensities(out / "codes.bin", arrays["codes"], wd)
    bio.write_quantization_parameters(out / "params.bin", arrays["params"], wd)
    sd = bio.default_shard_descriptor(shard_id)
    sd.timestamp_start, sd.timestamp_step, sd.loss_mask_id = ts_start, ts_step, loss_id
    bio.write_quantized_output_metadata(out / "int8_meta.txt",
                                        bio.QuantizedOutputMetadata(wd, T, S, sd, "params.bin"))
    bio.write_packed_shard(out / "shard_payload.bin", out / "shard_meta.txt", out / "shard_loss.bin",
                           bio.PackedShard(sd, arrays["voltage"], arrays["loss"]), d)
    return d, wd, sd


def test_python_io_identical_to_reference_and_reads_it(ref, tmp_path):
    from beamform_project_b200 import io as bio
    arrays, case = _case(seed=3)
    mine, theirs = tmp_path / "py", tmp_path / "ref"
    mine.mkdir()
    theirs.mkdir()
    d, wd, sd = _py_write(mine, arrays, case)
    ref.ref_io_write(theirs, arrays, case)
    for name in FILES:
        assert (mine / name).read_bytes() == (theirs / name).read_bytes(), name
    ref.ref_io_read_check(mine, arrays, case)
    assert np.array_equal(bio.read_packed_voltage(theirs / "voltage.bin", d).reshape(-1), arrays["voltage"])
    w = bio.read_weights(theirs / "weights.bin", d)
    assert w.dtype == np.complex64 and np.array_equal(w.view(np.float32).reshape(-1), arrays["weights"])
    assert np.array_equal(bio.read_quantized_intensities(theirs / "codes.bin", wd).reshape(-1), arrays["codes"])
    assert np.array_equal(bio.read_quantization_parameters(theirs / "params.bin", wd).reshape(-1), arrays["params"])
    m = bio.read_quantized_output_metadata(theirs / "int8_meta.txt")
    assert (m.output_dims, m.input_n_time, m.integration_spectra, m.shard, m.parameters_file) == \
        (wd, case[0], case[4], sd, "params.bin")
    sh = bio.read_packed_shard(theirs / "shard_payload.bin", theirs / "shard_meta.txt", theirs / "shard_loss.bin", d)
    assert sh.descriptor == sd and np.array_equal(sh.loss_mask.reshape(-1), arrays["loss"])


def test_python_io_errors(tmp_path):
    from beamform_project_b200 import io as bio
    d = bio.Dimensions(4, 336, 32, 3)
    v = np.full(4 * 336 * 32, 0x11, np.uint8)
    bio.write_packed_voltage(tmp_path / "v.bin", v, d)
    with pytest.raises(ValueError):
        bio.write_packed_voltage(tmp_path / "short.bin", v[:10], d)
    with pytest.raises(ValueError):
        bio.write_packed_voltage(tmp_path / "bad.bin", v, bio.Dimensions(4, 100, 32, 3))
    with pytest.raises(RuntimeError, match="43008 bytes; expected 53760"):
        bio.read_packed_voltage(tmp_path / "v.bin", bio.Dimensions(5, 336, 32, 3))
    with pytest.raises(RuntimeError):
        bio.read_weights(tmp_path / "missing.bin", d)
    (tmp_path / "m.txt").write_text("format=beamformer-quantized-int8-v1\nno separator\n")
    with pytest.raises(RuntimeError, match="invalid quantized metadata line"):
        bio.read_quantized_output_metadata(tmp_path / "m.txt")
    mask = np.ones(4 * 336, np.uint8)
    mask[3] = 2
    with pytest.raises(ValueError, match="0 or 1"):
        bio.write_packed_shard(tmp_path / "p", tmp_path / "q", tmp_path / "r",
                               bio.PackedShard(bio.default_shard_descriptor(0), v, mask), d)
