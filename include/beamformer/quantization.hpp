// quantization.hpp -- int8 chunk quantization contract (same declarations as
// the reference's include/beamformer/quantization.hpp:16-78 and the layout of
// src/quantization.cpp:34-59: one (offset, scale) pair per 1 x 16 x 16
// (window x frequency x beam) chunk, codes in [-127, 127], -128 = non-finite).
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/temporal_integration.hpp"

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace beamformer {

inline constexpr std::size_t quantization_chunk_time = 1;
inline constexpr std::size_t quantization_chunk_frequency = 16;
inline constexpr std::size_t quantization_chunk_beam = 16;
inline constexpr std::int8_t quantized_invalid_code = -128;
inline constexpr std::int8_t quantized_min_code = -127;
inline constexpr std::int8_t quantized_max_code = 127;

struct Int8QuantizationParameters {
    float offset = 0.0F;
    float scale = 0.0F;
};
static_assert(sizeof(Int8QuantizationParameters) == 2 * sizeof(float));

struct QuantizationLayout {
    std::size_t time_tiles = 0;
    std::size_t frequency_tiles = 0;
    std::size_t beam_tiles = 0;
};

inline QuantizationLayout quantization_layout(const Dimensions& integrated_dims) {
    validate_dimensions(integrated_dims);
    auto up = [](std::size_t v, std::size_t d) { return v / d + (v % d == 0 ? 0U : 1U); };
    return {up(integrated_dims.n_time, quantization_chunk_time),
            up(integrated_dims.n_freq, quantization_chunk_frequency),
            up(integrated_dims.n_beams, quantization_chunk_beam)};
}

inline std::size_t quantization_parameter_count(const Dimensions& integrated_dims) {
    const auto l = quantization_layout(integrated_dims);
    return l.time_tiles * l.frequency_tiles * l.beam_tiles;
}

inline std::size_t quantization_parameter_index(std::size_t time_tile, std::size_t frequency_tile,
                                                std::size_t beam_tile, const Dimensions& integrated_dims) {
    const auto l = quantization_layout(integrated_dims);
    if (time_tile >= l.time_tiles || frequency_tile >= l.frequency_tiles || beam_tile >= l.beam_tiles) {
        throw std::out_of_range("quantization parameter tile is outside dimensions");
    }
    return (time_tile * l.frequency_tiles + frequency_tile) * l.beam_tiles + beam_tile;
}

struct QuantizedIntegratedOutput {
    QuantizedIntensities codes;
    std::vector<Int8QuantizationParameters> parameters;
};

// What a reader of an int8 product needs besides the codes and parameters
// (reference quantization.hpp:75-83, validation src/quantization.cpp:235-249).
struct QuantizedOutputMetadata {
    Dimensions output_dims;
    std::size_t input_n_time = 0;
    TemporalIntegrationConfig temporal_integration{0};
    ShardDescriptor shard;
    std::string parameters_file;
};

inline void validate_quantized_output_metadata(const QuantizedOutputMetadata& metadata) {
    validate_dimensions(metadata.output_dims);
    validate_temporal_config(metadata.temporal_integration);
    validate_shard_descriptor(metadata.shard);
    if (metadata.input_n_time == 0) {
        throw std::invalid_argument("quantized metadata input_n_time must be positive");
    }
    if (integrated_time_count(metadata.input_n_time, metadata.temporal_integration) != metadata.output_dims.n_time) {
        throw std::invalid_argument("quantized metadata time dimensions are inconsistent");
    }
    if (metadata.parameters_file.empty()) {
        throw std::invalid_argument("quantized metadata parameters_file must not be empty");
    }
}

}  // namespace beamformer
