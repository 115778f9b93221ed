// temporal_integration.hpp -- integration windows (same declarations as the
// reference's include/beamformer/temporal_integration.hpp:11-43 and the
// window count of src/temporal_integration.cpp:16-45: W = ceil(T / S), the
// last window may be partial).
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"

#include <cstddef>
#include <cstdint>
#include <stdexcept>

namespace beamformer {

inline constexpr std::uint64_t spectrum_period_us_numerator = 10;
inline constexpr std::uint64_t spectrum_period_us_denominator = 3;

struct TemporalIntegrationConfig {
    std::size_t integration_spectra;
};

inline constexpr TemporalIntegrationConfig integration_after_upchan{10};
inline constexpr TemporalIntegrationConfig integration_direct{320};
inline constexpr TemporalIntegrationConfig integration_with_upchan = integration_after_upchan;
inline constexpr TemporalIntegrationConfig integration_without_upchan = integration_direct;
inline constexpr std::size_t default_integration_spectra = integration_without_upchan.integration_spectra;

using IntegratedIntensities = Intensities;

inline void validate_temporal_config(const TemporalIntegrationConfig& config) {
    if (config.integration_spectra == 0) throw std::invalid_argument("integration_spectra must be positive");
}

inline std::size_t integrated_time_count(const std::size_t n_time,
                                         const std::size_t integration_spectra = default_integration_spectra) {
    if (integration_spectra == 0) throw std::invalid_argument("integration_spectra must be positive");
    if (n_time == 0) throw std::invalid_argument("n_time must be positive");
    return n_time / integration_spectra + (n_time % integration_spectra == 0 ? 0U : 1U);
}

inline std::size_t integrated_time_count(const std::size_t n_time, const TemporalIntegrationConfig& config) {
    validate_temporal_config(config);
    return integrated_time_count(n_time, config.integration_spectra);
}

inline std::size_t integrated_intensity_count(const Dimensions& dims, const TemporalIntegrationConfig& config) {
    validate_dimensions(dims);
    return integrated_time_count(dims.n_time, config) * dims.n_freq * dims.n_beams;
}

inline std::size_t integrated_intensity_count(const Dimensions& dims,
                                              const std::size_t integration_spectra = default_integration_spectra) {
    return integrated_intensity_count(dims, TemporalIntegrationConfig{integration_spectra});
}

}  // namespace beamformer
