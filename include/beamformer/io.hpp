// io.hpp -- the on-disk formats of the voltage beamformer (same declarations
// as the reference's include/beamformer/io.hpp:10-51, files byte-identical to
// those of its src/io.cpp).
//
// Binary files are raw little-endian arrays with no header; a reader checks
// the file size against the dimensions first:
//   packed voltage      u8 [T][F][A] (low nibble re, high nibble im)
//   weights             complex64 [B][F][A]
//   tiled weights       complex64 [F][ceil(B/32)][A][32]
//   intensities         float32 [T][F][B]
//   quantized codes     int8 [W][F][B]
//   parameters          float32 [W][ceil(F/16)][ceil(B/16)][offset, scale]
//   loss mask           u8 [T][F], 0 or 1
// Two text formats of key=value lines: "beamformer-packed-shard-v1" (the
// metadata of a packed shard) and "beamformer-quantized-int8-v1" (the
// metadata of an int8 product).
// Errors: std::invalid_argument for dimension or size mismatches before
// writing, std::runtime_error for files that cannot be opened, have the wrong
// size, or hold malformed or inconsistent metadata.
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/quantization.hpp"

#include <filesystem>
#include <vector>

namespace beamformer {

PackedVoltage read_packed_voltage(const std::filesystem::path& path, const Dimensions& dims);
void write_packed_voltage(const std::filesystem::path& path, const PackedVoltage& voltage,
                          const Dimensions& dims);

void write_packed_shard(const std::filesystem::path& payload_path, const std::filesystem::path& metadata_path,
                        const std::filesystem::path& loss_mask_path, const PackedShard& shard,
                        const Dimensions& dims);
PackedShard read_packed_shard(const std::filesystem::path& payload_path, const std::filesystem::path& metadata_path,
                              const std::filesystem::path& loss_mask_path, const Dimensions& dims);

Weights read_weights(const std::filesystem::path& path, const Dimensions& dims);
void write_weights(const std::filesystem::path& path, const Weights& weights, const Dimensions& dims);
TiledWeights read_tiled_weights(const std::filesystem::path& path, const Dimensions& dims);
void write_tiled_weights(const std::filesystem::path& path, const TiledWeights& weights, const Dimensions& dims);

void write_intensities(const std::filesystem::path& path, const Intensities& intensities, const Dimensions& dims);

QuantizedIntensities read_quantized_intensities(const std::filesystem::path& path, const Dimensions& dims);
void write_quantized_intensities(const std::filesystem::path& path, const QuantizedIntensities& intensities,
                                 const Dimensions& dims);
std::vector<Int8QuantizationParameters> read_quantization_parameters(const std::filesystem::path& path,
                                                                     const Dimensions& integrated_dims);
void write_quantization_parameters(const std::filesystem::path& path,
                                   const std::vector<Int8QuantizationParameters>& parameters,
                                   const Dimensions& integrated_dims);
void write_quantized_output_metadata(const std::filesystem::path& path, const QuantizedOutputMetadata& metadata);
QuantizedOutputMetadata read_quantized_output_metadata(const std::filesystem::path& path);

}  // namespace beamformer
