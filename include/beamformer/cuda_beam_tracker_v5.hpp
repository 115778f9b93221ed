// cuda_beam_tracker_v5.hpp -- GPU tracker entry points.  Same declarations
// as the reference's include/beamformer/cuda_beam_tracker_v5.hpp:45-125
// (V5ExecutionConfig, host-vector and device-resident calls, the batched
// stream), backed by the B200 streaming tracker kernel: default geometry and
// channel plan as in the reference (src/cuda_beam_tracker_v5.cu:278-312),
// per-spectrum [T][F][1] float32 output.  V5ExecutionConfig's tuning fields
// are accepted and ignored (the B200 kernel has one launch shape); its
// enable_cuda_graph flag captures BatchedTrackerStreamV5's kernel launch.
//
// Extension: cuda_beam_tracker_device_resident_ex takes caller positions,
// wave numbers and window directions and can also (or only) write the
// per-window integrated power [W][F].
#pragma once

#include "beamformer/beam_tracker.hpp"
#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

namespace beamformer {

struct V5ExecutionConfig {
    std::size_t time_chunk_size = 80;
    std::size_t time_unroll = 8;
    bool enable_cuda_graph = false;
};

Intensities cuda_beam_tracker_v5(const PackedVoltage& packed, const Dimensions& dims, const TrackerConfig& tracker,
                                 const V5ExecutionConfig& config = V5ExecutionConfig{});

void cuda_beam_tracker_v5_into(const PackedVoltage& packed, const Dimensions& dims, const TrackerConfig& tracker,
                               Intensities& intensity, const V5ExecutionConfig& config = V5ExecutionConfig{});

// Device-resident: d_packed [T][F][A] and d_intensity [T][F] on the device,
// launched on `stream` (cudaStream_t, may be null).  Copies the window
// directions and wave numbers into a small buffer it owns per thread.
void cuda_beam_tracker_v5_device_resident(const std::uint8_t* d_packed, float* d_intensity, const Dimensions& dims,
                                          const TrackerConfig& tracker,
                                          const V5ExecutionConfig& config = V5ExecutionConfig{},
                                          void* stream = nullptr);

// Fully caller-supplied geometry on the device (positions [A][3] float,
// wave numbers [F] double, window directions [W][3] float); either output may
// be null.  Allocates nothing.
void cuda_beam_tracker_device_resident_ex(const std::uint8_t* d_packed, const float* d_positions,
                                          const double* d_wave_numbers, const float* d_window_directions,
                                          float* d_intensity, float* d_integrated, const Dimensions& dims,
                                          std::size_t integration_spectra, void* stream = nullptr);

class BatchedTrackerStreamV5 {
  public:
    BatchedTrackerStreamV5(const Dimensions& single_window_dims, const TrackerConfig& tracker,
                           std::size_t batch_size, const V5ExecutionConfig& config = V5ExecutionConfig{});
    ~BatchedTrackerStreamV5();
    BatchedTrackerStreamV5(const BatchedTrackerStreamV5&) = delete;
    BatchedTrackerStreamV5& operator=(const BatchedTrackerStreamV5&) = delete;

    void process_batch(std::size_t first_window_index, const std::uint8_t* host_packed, float* host_intensity);
    void process_batch_kernel_only(std::size_t first_window_index);
    float last_kernel_time_ms() const;
    std::uint8_t* device_packed_buffer();
    float* device_intensity_buffer();
    void* device_stream();
    std::size_t batch_size() const;
    std::size_t window_bytes() const;
    std::size_t batch_voltage_bytes() const;
    std::size_t batch_output_floats() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace beamformer
