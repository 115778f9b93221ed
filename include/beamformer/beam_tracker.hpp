// beam_tracker.hpp -- tracker configuration and trajectory.  Same
// declarations as the reference's include/beamformer/beam_tracker.hpp:31-74
// and the rules of src/beam_tracker.cpp:29-76: one steering direction per
// integration window, evaluated at the window's first sample on a linear
// (l, m) trajectory; n_beams must be 1.
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/geometry.hpp"
#include "beamformer/temporal_integration.hpp"

#include <cmath>
#include <cstddef>
#include <stdexcept>

namespace beamformer {

struct TrackerTrajectoryConfig {
    Vec3 direction_start = direction_from_lm(0.0F, 0.0F);
    Vec2 direction_rate_per_sample = {0.0F, 0.0F};
};

struct TrackerConfig {
    TrackerTrajectoryConfig trajectory;
    std::size_t integration_spectra = integration_direct.integration_spectra;
};

inline constexpr std::size_t tracker_beam_count = 1;

inline std::size_t tracker_window_count(const std::size_t n_time, const std::size_t integration_spectra) {
    if (integration_spectra == 0) throw std::invalid_argument("integration_spectra must be positive");
    return (n_time + integration_spectra - 1) / integration_spectra;
}

inline Vec3 tracker_direction(const TrackerTrajectoryConfig& trajectory, const std::size_t t) {
    const float l = trajectory.direction_start[0] + static_cast<float>(t) * trajectory.direction_rate_per_sample[0];
    const float m = trajectory.direction_start[1] + static_cast<float>(t) * trajectory.direction_rate_per_sample[1];
    return direction_from_lm(l, m);
}

inline Vec3 tracker_window_direction(const TrackerTrajectoryConfig& trajectory, const std::size_t window,
                                     const std::size_t integration_spectra) {
    if (integration_spectra == 0) throw std::invalid_argument("integration_spectra must be positive");
    return tracker_direction(trajectory, window * integration_spectra);
}

// Argument checks of the reference's validate_tracker_config
// (src/beam_tracker.cpp:29-54).
inline void validate_tracker_config(const Dimensions& dims, const TrackerConfig& tracker) {
    validate_dimensions(dims);
    if (dims.n_beams != tracker_beam_count) {
        throw std::invalid_argument("tracker requires exactly n_beams == 1 (use tracker_beam_count)");
    }
    if (tracker.integration_spectra == 0) throw std::invalid_argument("tracker integration_spectra must be positive");
    const auto& s = tracker.trajectory.direction_start;
    const double n2 = static_cast<double>(s[0]) * s[0] + static_cast<double>(s[1]) * s[1] +
                      static_cast<double>(s[2]) * s[2];
    if (!std::isfinite(n2) || std::abs(n2 - 1.0) > 1.0e-3) {
        throw std::invalid_argument("tracker direction_start must be a finite unit vector");
    }
    for (const float c : tracker.trajectory.direction_rate_per_sample) {
        if (!std::isfinite(c)) throw std::invalid_argument("tracker direction_rate_per_sample must be finite");
    }
}

}  // namespace beamformer
