// cuda_beamformer.hpp -- host pipelines over the B200 kernels.  Same
// declarations as the reference's include/beamformer/cuda_beamformer.hpp:
// 14-123: CudaBeamformerWorkspace (buffers, stream and events reused across
// calls, weights resident, voltage uploaded per call), the one-shot
// wrappers and cuda_device_info.  Errors are the reference's exception
// types; timings are CUDA-event milliseconds per phase.
//
// Added selector value: CudaBeamformerKernel::TensorSplit runs the tcgen05
// split-precision kernel (per-spectrum or integrated output; integration
// length below 32 or a multiple of 32; any antenna count).  upload_weights
// then takes canonical [B][F][A] weights and prepares the fp16 hi + lo
// operand on the device.
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/cuda_frame.hpp"
#include "beamformer/cuda_stage_api.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/quantization.hpp"
#include "beamformer/temporal_integration.hpp"

#include <cstddef>
#include <memory>
#include <optional>
#include <string>

struct bf_grid_pipeline;  // include/bf_b200.h

namespace beamformer {

enum class CudaBeamformerOutput {
    Float32,
    QuantizedInt8,
};

struct CudaBeamformerTimings {
    double setup_ms = 0.0;
    double host_to_device_ms = 0.0;
    double kernel_ms = 0.0;
    double temporal_integration_ms = 0.0;  // fused: always zero
    double quantization_ms = 0.0;
    double device_to_device_ms = 0.0;
    double device_to_host_ms = 0.0;
};

struct CudaDeviceInfo {
    std::string name;
    int compute_major = 0;
    int compute_minor = 0;
    std::size_t global_memory_bytes = 0;
    int driver_version = 0;
    int runtime_version = 0;
};

CudaDeviceInfo cuda_device_info();

class CudaBeamformerWorkspace {
  public:
    explicit CudaBeamformerWorkspace(const Dimensions& capacity,
                                     CudaBeamformerKernel kernel = CudaBeamformerKernel::Direct,
                                     std::optional<TemporalIntegrationConfig> temporal_integration = std::nullopt,
                                     CudaBeamformerOutput output = CudaBeamformerOutput::Float32);
    ~CudaBeamformerWorkspace();

    CudaBeamformerWorkspace(const CudaBeamformerWorkspace&) = delete;
    CudaBeamformerWorkspace& operator=(const CudaBeamformerWorkspace&) = delete;

    double setup_ms() const;
    CudaBeamformerKernel kernel() const;
    double upload_packed_voltage(const PackedVoltage& packed, const Dimensions& dims);
    double upload_weights(const Weights& weights, const Dimensions& dims);
    double run_kernel(const Dimensions& dims);
    double download_intensity(Intensities& intensity, const Dimensions& dims);
    CudaBeamformerTimings run_pipeline(const PackedVoltage& packed, Intensities& intensity, const Dimensions& dims);
    CudaBeamformerTimings run_integrated_pipeline(const PackedVoltage& packed, IntegratedIntensities& intensity,
                                                  const Dimensions& dims);
    CudaBeamformerTimings run_quantized_integrated_pipeline(const PackedVoltage& packed,
                                                            QuantizedIntegratedOutput& intensity,
                                                            const Dimensions& dims);
    CudaBeamformerTimings run_device_frame(const CudaFrameView& voltage, const CudaFrameView& weights,
                                           CudaFrameView& output, CudaFrameView* quantization_parameters = nullptr);

    bool has_temporal_integration() const;
    bool has_int8_quantization() const;
    std::size_t packed_voltage_capacity_bytes() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// Added: the TensorSplit grid fed from host memory (bf_grid_pipeline_* of
// bf_b200.h).  Weights stay resident; each run() streams a block of n_shards
// shards ([shard][T][F][A] bytes) in time chunks whose host-to-device copy,
// kernels and device-to-host copy overlap on three streams, with products
// bit-identical to one TensorSplit launch over the block.  Outputs are
// resized to [shard][W][F][B] (codes) and [shard][W][F/16][B/16]
// (parameters); run() returns the device milliseconds of the block.
class CudaChunkedGridPipeline {
  public:
    CudaChunkedGridPipeline(const Dimensions& dims, const TemporalIntegrationConfig& temporal_integration,
                            std::size_t n_shards = 1, std::size_t chunk_spectra = 0);
    ~CudaChunkedGridPipeline();

    CudaChunkedGridPipeline(const CudaChunkedGridPipeline&) = delete;
    CudaChunkedGridPipeline& operator=(const CudaChunkedGridPipeline&) = delete;

    std::size_t chunk_spectra() const;
    void upload_weights(const Weights& weights);  // [shard][B][F][A]
    double run(const PackedVoltage& packed, IntegratedIntensities* integrated, QuantizedIntegratedOutput* quantized);

  private:
    bf_grid_pipeline* pipeline_ = nullptr;
    Dimensions dims_;
    std::size_t spectra_ = 0, n_shards_ = 0, chunk_ = 0;
};

Intensities cuda_beamform_packed_intensity(const PackedVoltage& packed, const Weights& weights,
                                           const Dimensions& dims, CudaBeamformerTimings* timings = nullptr,
                                           CudaBeamformerKernel kernel = CudaBeamformerKernel::Direct);

IntegratedIntensities cuda_beamform_packed_integrated_intensity(
    const PackedVoltage& packed, const Weights& weights, const Dimensions& dims,
    const TemporalIntegrationConfig& temporal_integration, CudaBeamformerTimings* timings = nullptr,
    CudaBeamformerKernel kernel = CudaBeamformerKernel::Tiled);

QuantizedIntegratedOutput cuda_beamform_packed_quantized_integrated_intensity(
    const PackedVoltage& packed, const Weights& weights, const Dimensions& dims,
    const TemporalIntegrationConfig& temporal_integration, CudaBeamformerTimings* timings = nullptr,
    CudaBeamformerKernel kernel = CudaBeamformerKernel::Tiled);

}  // namespace beamformer
