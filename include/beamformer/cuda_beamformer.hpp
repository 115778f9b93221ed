// cuda_beamformer.hpp -- host pipelines over the B200 kernels.  Same
// declarations as the reference's include/beamformer/cuda_beamformer.hpp:
// 14-123: CudaBeamformerWorkspace (buffers, stream and events reused across
// calls, weights resident, voltage uploaded per call), the one-shot
// wrappers and cuda_device_info.  Errors are the reference's exception
// types; timings are CUDA-event milliseconds per phase.
//
// Added selector value: CudaBeamformerKernel::TensorSplit runs the tcgen05
// split-precision kernel (per-spectrum or integrated output; integration
// length below 32 or a multiple of 32; 32 or 64 antennas).  upload_weights
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
