// formats.hpp -- complex type, packed int4 contract, buffer aliases, index
// formulas and byte counts.  Same declarations as the reference's
// include/beamformer/{complex,int4,formats,indexing}.hpp (complex.hpp:7-13,
// int4.hpp:14-39, formats.hpp:12-90, indexing.hpp:13-66): the packed
// [T][F][E] voltage layout, the [B][F][A] and tiled [F][Btile][A][32] weight
// layouts and the [T][F][B] intensity layout are the drop-in contract.
#pragma once

#include "beamformer/config.hpp"

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <type_traits>
#include <vector>

namespace beamformer {

struct ComplexFloat {
    float real;
    float imag;
};
static_assert(sizeof(ComplexFloat) == 2 * sizeof(float));
static_assert(std::is_trivially_copyable_v<ComplexFloat>);

struct ComplexInt4 {
    std::int8_t real;
    std::int8_t imag;
};

// Signed two's-complement nibble (int4.hpp:19-24).
constexpr std::int8_t decode_signed_nibble(const std::uint8_t nibble) {
    const auto bits = static_cast<std::uint8_t>(nibble & 0x0F);
    return bits < 8 ? static_cast<std::int8_t>(bits) : static_cast<std::int8_t>(static_cast<int>(bits) - 16);
}

// Low nibble = real, high nibble = imaginary (int4.hpp:26-30).
constexpr ComplexInt4 unpack_complex_int4(const std::uint8_t packed) {
    return {decode_signed_nibble(packed), decode_signed_nibble(static_cast<std::uint8_t>(packed >> 4))};
}

inline std::uint8_t pack_complex_int4(const std::int8_t real, const std::int8_t imag) {
    if (real < -8 || real > 7 || imag < -8 || imag > 7) {
        throw std::out_of_range("int4 components must be in [-8, 7]");
    }
    return static_cast<std::uint8_t>((static_cast<std::uint8_t>(real) & 0x0F) |
                                     ((static_cast<std::uint8_t>(imag) & 0x0F) << 4));
}

using PackedVoltage = std::vector<std::uint8_t>;
using ComplexVoltage = std::vector<ComplexFloat>;
using Weights = std::vector<ComplexFloat>;
using TiledWeights = std::vector<ComplexFloat>;
using Intensities = std::vector<float>;
using QuantizedIntensities = std::vector<std::int8_t>;
using LossMask = std::vector<std::uint8_t>;

constexpr std::size_t voltage_sample_count(const Dimensions& dims) { return dims.n_time * dims.n_freq * dims.n_ant; }
constexpr std::size_t packed_voltage_bytes(const Dimensions& dims) { return voltage_sample_count(dims); }
// one validity byte (0 = lost, 1 = valid) per [time][local frequency] frame
constexpr std::size_t loss_mask_count(const Dimensions& dims) { return dims.n_time * dims.n_freq; }

// One frequency shard as it arrives: the packed payload, its descriptor and
// its loss mask (reference formats.hpp:22-34).
struct PackedShard {
    ShardDescriptor descriptor;
    PackedVoltage payload;
    LossMask loss_mask;
};
using PackedShardSet = std::array<PackedShard, frequency_shard_count>;

// reference src/synthetic_data.cpp:139-171
inline void validate_packed_shard(const PackedShard& shard, const Dimensions& dims) {
    validate_dimensions(dims);
    validate_shard_descriptor(shard.descriptor);
    if (shard.payload.size() != packed_voltage_bytes(dims)) {
        throw std::invalid_argument("shard payload size does not match dimensions");
    }
    if (shard.loss_mask.size() != loss_mask_count(dims)) {
        throw std::invalid_argument("loss mask size does not match dimensions");
    }
    for (const std::uint8_t v : shard.loss_mask) {
        if (v > 1U) throw std::invalid_argument("loss mask entries must be 0 or 1");
    }
}

inline void validate_packed_shards(const PackedShardSet& shards, const Dimensions& dims) {
    validate_dimensions(dims);
    for (std::size_t i = 0; i < frequency_shard_count; ++i) {
        validate_packed_shard(shards[i], dims);
        if (shards[i].descriptor.shard_id != i) {
            throw std::invalid_argument("shard IDs must identify their array slot");
        }
    }
    if (shards[0].descriptor.absolute_frequency_start == shards[1].descriptor.absolute_frequency_start) {
        throw std::invalid_argument("the two shards must have distinct frequency origins");
    }
    if (shards[0].descriptor.loss_mask_id == shards[1].descriptor.loss_mask_id) {
        throw std::invalid_argument("the two shards must have independent loss masks");
    }
}
constexpr std::size_t weight_bytes(const Dimensions& dims) {
    return dims.n_beams * dims.n_freq * dims.n_ant * 2 * sizeof(float);
}
constexpr std::size_t tiled_weight_beam_tile = 32;
constexpr std::size_t tiled_weight_beam_tiles(const Dimensions& dims) {
    return (dims.n_beams + tiled_weight_beam_tile - 1) / tiled_weight_beam_tile;
}
constexpr std::size_t tiled_weight_count(const Dimensions& dims) {
    return dims.n_freq * tiled_weight_beam_tiles(dims) * dims.n_ant * tiled_weight_beam_tile;
}
constexpr std::size_t tiled_weight_bytes(const Dimensions& dims) { return tiled_weight_count(dims) * 2 * sizeof(float); }
constexpr std::size_t intensity_bytes(const Dimensions& dims) {
    return dims.n_time * dims.n_freq * dims.n_beams * sizeof(float);
}
constexpr std::size_t quantized_intensity_bytes(const Dimensions& dims) {
    return dims.n_time * dims.n_freq * dims.n_beams * sizeof(std::int8_t);
}

constexpr std::size_t voltage_index(std::size_t t, std::size_t f, std::size_t e, const Dimensions& d) {
    return (t * d.n_freq + f) * d.n_ant + e;
}
constexpr std::size_t weight_index(std::size_t b, std::size_t f, std::size_t a, const Dimensions& d) {
    return (b * d.n_freq + f) * d.n_ant + a;
}
constexpr std::size_t tiled_weight_index(std::size_t f, std::size_t tile, std::size_t a, std::size_t lb,
                                         const Dimensions& d) {
    return ((f * tiled_weight_beam_tiles(d) + tile) * d.n_ant + a) * tiled_weight_beam_tile + lb;
}
constexpr std::size_t intensity_index(std::size_t t, std::size_t f, std::size_t b, const Dimensions& d) {
    return (t * d.n_freq + f) * d.n_beams + b;
}

}  // namespace beamformer
