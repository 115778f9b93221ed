"""On-disk formats for Python callers (numpy), the same files as
include/beamformer/io.hpp and the reference's src/io.cpp:60-344.

Binary files are raw little-endian arrays without a header, checked against
the dimensions on read:

    packed voltage    uint8 [T][F][A]          read_packed_voltage / write_packed_voltage
    weights           complex64 [B][F][A]      read_weights / write_weights
    tiled weights     complex64 [F][ceil(B/32)][A][32]
    intensities       float32 [T][F][B]        write_intensities
    quantized codes   int8 [W][F][B]           read_quantized_intensities / write_...
    parameters        float32 [W][ceil(F/16)][ceil(B/16)][offset, scale]
    loss mask         uint8 [T][F], 0 or 1

and two key=value text formats, "beamformer-packed-shard-v1" and
"beamformer-quantized-int8-v1", written with the reference's keys in its
order.  Dimension and size mismatches raise ValueError before anything is
written; unreadable, wrongly sized or malformed files raise RuntimeError
(std::invalid_argument and std::runtime_error in the C++ API).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

F_LOCAL = 336
SHARD_COUNT = 2
CHUNK_TIME, CHUNK_FREQ, CHUNK_BEAM = 1, 16, 16
INVALID_CODE = -128
SHARD_FORMAT = "beamformer-packed-shard-v1"
INT8_FORMAT = "beamformer-quantized-int8-v1"
PARAMS_FORMAT = "little-endian-float32[offset,scale]"


@dataclass(frozen=True)
class Dimensions:
    n_time: int
    n_freq: int = F_LOCAL
    n_ant: int = 64
    n_beams: int = 1

    def validate(self) -> None:
        """The reference's validate_dimensions rules (config.hpp)."""
        if self.n_time <= 0:
            raise ValueError("n_time must be positive")
        if self.n_freq != F_LOCAL:
            raise ValueError("the local-shard contract requires exactly 336 frequency channels")
        if self.n_ant not in (32, 64, 128, 256):
            raise ValueError("n_ant must be 32, 64, 128, or 256")
        if not 1 <= self.n_beams <= 128:
            raise ValueError("n_beams must be between 1 and 128")


@dataclass
class ShardDescriptor:
    shard_id: int = 0
    shard_count: int = SHARD_COUNT
    local_frequency_count: int = F_LOCAL
    absolute_frequency_start: int = 0
    timestamp_start: int = 0
    timestamp_step: int = 1
    loss_mask_id: int = 0
    loss_mask_independent: bool = True

    def validate(self) -> None:
        if self.shard_count != SHARD_COUNT:
            raise ValueError("shard_count must be exactly 2")
        if not 0 <= self.shard_id < self.shard_count:
            raise ValueError("shard_id is outside the two-shard band")
        if self.local_frequency_count != F_LOCAL:
            raise ValueError("local_frequency_count must be exactly 336")
        if not 0 <= self.absolute_frequency_start <= F_LOCAL * (SHARD_COUNT - 1):
            raise ValueError("absolute frequency start is outside the full band")
        if self.timestamp_step == 0:
            raise ValueError("timestamp_step must be positive")
        if not self.loss_mask_independent:
            raise ValueError("loss masks must be independent per shard")


def default_shard_descriptor(shard_id: int) -> ShardDescriptor:
    return ShardDescriptor(shard_id=shard_id, absolute_frequency_start=F_LOCAL * shard_id, loss_mask_id=shard_id)


@dataclass
class PackedShard:
    descriptor: ShardDescriptor
    payload: np.ndarray              # uint8 [T][F][A]
    loss_mask: np.ndarray            # uint8 [T][F]


@dataclass
class QuantizedOutputMetadata:
    output_dims: Dimensions
    input_n_time: int
    integration_spectra: int
    shard: ShardDescriptor = field(default_factory=ShardDescriptor)
    parameters_file: str = "parameters.bin"


def integrated_time_count(n_time: int, spectra: int) -> int:
    if spectra <= 0:
        raise ValueError("integration_spectra must be positive")
    if n_time <= 0:
        raise ValueError("n_time must be positive")
    return -(-n_time // spectra)


def quantization_parameter_count(d: Dimensions) -> int:
    d.validate()
    return (-(-d.n_time // CHUNK_TIME)) * (-(-d.n_freq // CHUNK_FREQ)) * (-(-d.n_beams // CHUNK_BEAM))


def tiled_weight_count(d: Dimensions) -> int:
    return d.n_freq * (-(-d.n_beams // 32)) * d.n_ant * 32


# ---------------- raw arrays ----------------

def _load(path, dtype, count: int) -> np.ndarray:
    path = Path(path)
    try:
        size = path.stat().st_size
    except OSError as e:
        raise RuntimeError(f"cannot inspect input file: {path}") from e
    want = count * np.dtype(dtype).itemsize
    if size != want:
        raise RuntimeError(f"{path} has {size} bytes; expected {want}")
    return np.fromfile(path, dtype=dtype, count=count)


def _store(path, data: np.ndarray, dtype, count: int, what: str) -> None:
    a = np.ascontiguousarray(data, dtype=dtype).reshape(-1)
    if a.size != count:
        raise ValueError(f"{what} does not match dimensions")
    with open(path, "wb") as fh:
        a.tofile(fh)


def read_packed_voltage(path, d: Dimensions) -> np.ndarray:
    d.validate()
    return _load(path, np.uint8, d.n_time * d.n_freq * d.n_ant).reshape(d.n_time, d.n_freq, d.n_ant)


def write_packed_voltage(path, voltage: np.ndarray, d: Dimensions) -> None:
    d.validate()
    _store(path, voltage, np.uint8, d.n_time * d.n_freq * d.n_ant, "packed voltage size")


def read_weights(path, d: Dimensions) -> np.ndarray:
    d.validate()
    return _load(path, np.complex64, d.n_beams * d.n_freq * d.n_ant).reshape(d.n_beams, d.n_freq, d.n_ant)


def write_weights(path, weights: np.ndarray, d: Dimensions) -> None:
    d.validate()
    _store(path, _complex(weights), np.complex64, d.n_beams * d.n_freq * d.n_ant, "weight count")


def read_tiled_weights(path, d: Dimensions) -> np.ndarray:
    d.validate()
    return _load(path, np.complex64, tiled_weight_count(d)).reshape(d.n_freq, -(-d.n_beams // 32), d.n_ant, 32)


def write_tiled_weights(path, weights: np.ndarray, d: Dimensions) -> None:
    d.validate()
    _store(path, _complex(weights), np.complex64, tiled_weight_count(d), "tiled weight count")


def write_intensities(path, intensities: np.ndarray, d: Dimensions) -> None:
    d.validate()
    _store(path, intensities, np.float32, d.n_time * d.n_freq * d.n_beams, "intensity count")


def read_quantized_intensities(path, d: Dimensions) -> np.ndarray:
    d.validate()
    return _load(path, np.int8, d.n_time * d.n_freq * d.n_beams).reshape(d.n_time, d.n_freq, d.n_beams)


def write_quantized_intensities(path, codes: np.ndarray, d: Dimensions) -> None:
    d.validate()
    _store(path, codes, np.int8, d.n_time * d.n_freq * d.n_beams, "quantized intensity count")


def read_quantization_parameters(path, integrated: Dimensions) -> np.ndarray:
    """float32 [count][2] of (offset, scale)."""
    return _load(path, np.float32, 2 * quantization_parameter_count(integrated)).reshape(-1, 2)


def write_quantization_parameters(path, params: np.ndarray, integrated: Dimensions) -> None:
    _store(path, params, np.float32, 2 * quantization_parameter_count(integrated), "quantization parameter count")


def _complex(a: np.ndarray) -> np.ndarray:
    """complex64 array, or float32 [..., 2] (re, im) pairs viewed as complex64."""
    a = np.asarray(a)
    if np.iscomplexobj(a):
        return a.astype(np.complex64)
    a = np.ascontiguousarray(a, np.float32)
    if a.shape[-1:] != (2,):
        raise ValueError("weights must be complex64 or float32 [..., 2]")
    return a.view(np.complex64)[..., 0]


# ---------------- key=value metadata ----------------

def _store_fields(path, fields: list[tuple[str, object]]) -> None:
    with open(path, "w", newline="\n") as fh:
        for k, v in fields:
            fh.write(f"{k}={v}\n")


def _load_fields(path, what: str) -> dict[str, str]:
    """key=value lines (the last value of a repeated key wins); a line
    without '=' or with an empty key is an error."""
    try:
        text = Path(path).read_text()
    except OSError as e:
        raise RuntimeError(f"cannot open {what} file: {path}") from e
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    out: dict[str, str] = {}
    for line in lines:
        eq = line.find("=")
        if eq <= 0:
            raise RuntimeError(f"invalid {what} line in: {path}")
        out[line[:eq]] = line[eq + 1:]
    return out


def _need(fields: dict[str, str], key: str, what: str, path) -> str:
    if key not in fields:
        raise RuntimeError(f"missing {what} field {key} in: {path}")
    return fields[key]


def _shard_fields(d: ShardDescriptor) -> list[tuple[str, object]]:
    return [("shard_id", d.shard_id), ("shard_count", d.shard_count),
            ("local_frequency_count", d.local_frequency_count),
            ("absolute_frequency_start", d.absolute_frequency_start), ("timestamp_start", d.timestamp_start),
            ("timestamp_step", d.timestamp_step), ("loss_mask_id", d.loss_mask_id),
            ("loss_mask_independent", 1 if d.loss_mask_independent else 0)]


def _read_shard(get, flag) -> ShardDescriptor:
    return ShardDescriptor(int(get("shard_id")), int(get("shard_count")), int(get("local_frequency_count")),
                           int(get("absolute_frequency_start")), int(get("timestamp_start")),
                           int(get("timestamp_step")), int(get("loss_mask_id")), flag("loss_mask_independent"))


def _validate_metadata(m: QuantizedOutputMetadata) -> None:
    m.output_dims.validate()
    if m.integration_spectra <= 0:
        raise ValueError("integration_spectra must be positive")
    m.shard.validate()
    if m.input_n_time <= 0:
        raise ValueError("quantized metadata input_n_time must be positive")
    if integrated_time_count(m.input_n_time, m.integration_spectra) != m.output_dims.n_time:
        raise ValueError("quantized metadata time dimensions are inconsistent")
    if not m.parameters_file:
        raise ValueError("quantized metadata parameters_file must not be empty")


def write_quantized_output_metadata(path, m: QuantizedOutputMetadata) -> None:
    _validate_metadata(m)
    d = m.output_dims
    _store_fields(path, [("format", INT8_FORMAT), ("n_time", d.n_time), ("n_freq", d.n_freq), ("n_ant", d.n_ant),
                         ("n_beams", d.n_beams), ("input_n_time", m.input_n_time),
                         ("integration_spectra", m.integration_spectra), ("chunk_time", CHUNK_TIME),
                         ("chunk_frequency", CHUNK_FREQ), ("chunk_beam", CHUNK_BEAM), ("invalid_code", INVALID_CODE),
                         ("parameters_format", PARAMS_FORMAT), ("parameters_file", m.parameters_file),
                         ("parameters_count", quantization_parameter_count(d))] + _shard_fields(m.shard))


def read_quantized_output_metadata(path) -> QuantizedOutputMetadata:
    what = "quantized metadata"
    f = _load_fields(path, what)
    get = lambda k: _need(f, k, what, path)  # noqa: E731

    def flag(k):
        v = get(k)
        if v not in ("0", "1"):
            raise RuntimeError(f"invalid {what} flag {k}")
        return v == "1"

    if (get("format") != INT8_FORMAT or get("parameters_format") != PARAMS_FORMAT
            or int(get("chunk_time")) != CHUNK_TIME or int(get("chunk_frequency")) != CHUNK_FREQ
            or int(get("chunk_beam")) != CHUNK_BEAM or int(get("invalid_code")) != INVALID_CODE):
        raise RuntimeError(f"unsupported quantized metadata format: {path}")
    m = QuantizedOutputMetadata(Dimensions(int(get("n_time")), int(get("n_freq")), int(get("n_ant")),
                                           int(get("n_beams"))),
                                int(get("input_n_time")), int(get("integration_spectra")), _read_shard(get, flag),
                                get("parameters_file"))
    if int(get("parameters_count")) != quantization_parameter_count(m.output_dims):
        raise RuntimeError(f"quantization parameter count is inconsistent: {path}")
    _validate_metadata(m)
    return m


def _validate_shard(s: PackedShard, d: Dimensions) -> None:
    d.validate()
    s.descriptor.validate()
    if np.asarray(s.payload).size != d.n_time * d.n_freq * d.n_ant:
        raise ValueError("shard payload size does not match dimensions")
    mask = np.asarray(s.loss_mask)
    if mask.size != d.n_time * d.n_freq:
        raise ValueError("loss mask size does not match dimensions")
    if mask.size and int(mask.max()) > 1:
        raise ValueError("loss mask entries must be 0 or 1")


def write_packed_shard(payload_path, metadata_path, loss_mask_path, shard: PackedShard, d: Dimensions) -> None:
    _validate_shard(shard, d)
    write_packed_voltage(payload_path, shard.payload, d)
    _store(loss_mask_path, shard.loss_mask, np.uint8, d.n_time * d.n_freq, "loss mask size")
    _store_fields(metadata_path, [("format", SHARD_FORMAT), ("n_time", d.n_time), ("n_freq", d.n_freq),
                                  ("n_ant", d.n_ant), ("n_beams", d.n_beams)] + _shard_fields(shard.descriptor) +
                  [("payload_bytes", d.n_time * d.n_freq * d.n_ant), ("loss_mask_bytes", d.n_time * d.n_freq)])


def read_packed_shard(payload_path, metadata_path, loss_mask_path, d: Dimensions) -> PackedShard:
    d.validate()
    what = "shard metadata"
    f = _load_fields(metadata_path, what)
    get = lambda k: _need(f, k, what, metadata_path)  # noqa: E731

    def flag(k):
        v = get(k)
        if v not in ("0", "1"):
            raise RuntimeError(f"invalid {what} flag {k}")
        return v == "1"

    if (get("format") != SHARD_FORMAT or int(get("n_time")) != d.n_time or int(get("n_freq")) != d.n_freq
            or int(get("n_ant")) != d.n_ant or int(get("n_beams")) != d.n_beams
            or int(get("payload_bytes")) != d.n_time * d.n_freq * d.n_ant
            or int(get("loss_mask_bytes")) != d.n_time * d.n_freq):
        raise RuntimeError(f"shard metadata does not match dimensions: {metadata_path}")
    shard = PackedShard(_read_shard(get, flag), read_packed_voltage(payload_path, d),
                        _load(loss_mask_path, np.uint8, d.n_time * d.n_freq).reshape(d.n_time, d.n_freq))
    _validate_shard(shard, d)
    return shard


__all__ = [n for n in dir() if not n.startswith("_") and n not in ("annotations", "np", "Path", "dataclass", "field")]
