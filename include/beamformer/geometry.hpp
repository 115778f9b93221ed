// geometry.hpp -- the geometry pieces the tracker path needs.  Same
// declarations as the reference's include/beamformer/geometry.hpp:12-36
// (Vec2/Vec3, regular_array, default_positions, channelized_frequencies,
// direction_from_lm) with the reference's rules (src/geometry.cpp:34-106).
// Beam-grid construction and file loaders stay with the reference's CPU
// library (not on the hot path).
#pragma once

#include "beamformer/config.hpp"

#include <array>
#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <vector>

namespace beamformer {

using Vec3 = std::array<float, 3>;
using Vec2 = std::array<float, 2>;

inline std::vector<Vec3> regular_array(const std::size_t rows, const std::size_t columns,
                                       const float spacing_m = default_spacing_m) {
    if (rows == 0 || columns == 0) throw std::invalid_argument("array rows and columns must be positive");
    if (spacing_m <= 0.0F) throw std::invalid_argument("antenna spacing must be positive");
    std::vector<Vec3> p;
    p.reserve(rows * columns);
    for (std::size_t r = 0; r < rows; ++r)
        for (std::size_t c = 0; c < columns; ++c)
            p.push_back({static_cast<float>(c) * spacing_m, static_cast<float>(r) * spacing_m, 0.0F});
    return p;
}

inline std::vector<Vec3> default_positions(const std::size_t n_ant, const float spacing_m = default_spacing_m) {
    switch (n_ant) {
        case 32: return regular_array(4, 8, spacing_m);
        case 64: return regular_array(8, 8, spacing_m);
        case 128: return regular_array(8, 16, spacing_m);
        case 256: return regular_array(16, 16, spacing_m);
        default: break;
    }
    throw std::invalid_argument("default geometry is available only for 32, 64, 128, or 256 antennas");
}

inline std::vector<float> channelized_frequencies(const std::size_t n_freq = default_frequency_channels,
                                                  const float start_hz = default_frequency_start_hz,
                                                  const float channel_width_hz = default_channel_width_hz) {
    if (n_freq == 0) throw std::invalid_argument("frequency count must be positive");
    if (!std::isfinite(start_hz) || start_hz <= 0.0F || !std::isfinite(channel_width_hz) ||
        channel_width_hz <= 0.0F) {
        throw std::invalid_argument("frequency start and channel width must be positive");
    }
    std::vector<float> f(n_freq);
    for (std::size_t c = 0; c < n_freq; ++c) f[c] = start_hz + static_cast<float>(c) * channel_width_hz;
    return f;
}

inline Vec3 direction_from_lm(const float l, const float m) {
    if (!std::isfinite(l) || !std::isfinite(m)) throw std::invalid_argument("direction cosines l and m must be finite");
    const float t = l * l + m * m;
    if (t > 1.0F) throw std::invalid_argument("direction cosines must satisfy l*l + m*m <= 1");
    return {l, m, std::sqrt(1.0F - t)};
}

}  // namespace beamformer
