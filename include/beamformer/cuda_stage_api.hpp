// cuda_stage_api.hpp -- device-stage API (same declarations as the
// reference's include/beamformer/cuda_stage_api.hpp:14-42).  Each call runs
// one stage on caller-owned device buffers and the caller's stream; none
// allocates memory or synchronises.  Errors are the reference's exception
// types: std::invalid_argument (dimensions, kernel and integration rules),
// std::runtime_error (CUDA), std::overflow_error (grid too large).
//
// Kernel selector: Direct (canonical [B][F][A] weights) and Tiled (tiled
// [F][ceil(B/32)][A][32] weights) reproduce the reference float32 operation
// order bit for bit.  TensorSplit is the tcgen05 split-precision kernel; it
// reads weights prepared by prepare_split_weights; through this stage API it
// writes integrated output (the workspace also gives per-spectrum output).
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/quantization.hpp"
#include "beamformer/temporal_integration.hpp"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace beamformer {

enum class CudaBeamformerKernel {
    Direct,
    Tiled,
    TensorSplit,
    // Opt-in covariance form (integrated output only, 64 antennas, integration a
    // multiple of 64 spectra up to 16384): each window's power from its exact
    // INT32 covariance.  Its relative error grows for beams far below the
    // strongest source's power; TensorSplit has no such dependence.
    TensorCovariance,
    // Checked tensor path (integrated output only, any n_ant): the
    // covariance form where it applies, with every unit whose error estimate
    // exceeds the calibrated limit recomputed by TensorSplit, so every value
    // stays within 1e-5 relative of FP64; TensorSplit elsewhere.  Its stage
    // call is launch_checked_integrated_beamformer (it needs a workspace).
    TensorChecked,
};

void launch_packed_beamformer(CudaBeamformerKernel kernel, cudaStream_t stream,
                              const std::uint8_t* packed_voltage, const ComplexFloat* weights,
                              float* intensity, const Dimensions& dims);

// Direct accepts 320 spectra only and Tiled 10 or 320, as in the reference
// (src/cuda_beamformer.cu:418-433); TensorSplit accepts any length below 32
// and any multiple of 32.
void launch_packed_integrated_beamformer(CudaBeamformerKernel kernel, cudaStream_t stream,
                                         const std::uint8_t* packed_voltage, const ComplexFloat* weights,
                                         float* integrated_intensity, const Dimensions& dims,
                                         const TemporalIntegrationConfig& temporal_integration);

void launch_quantize_integrated_intensity(cudaStream_t stream, const float* integrated_intensity,
                                          std::int8_t* quantized_intensity,
                                          Int8QuantizationParameters* parameters,
                                          const Dimensions& integrated_dims);

// Loss-mask consumption (the reference defines the mask, formats.hpp:22-30,
// but no consumer): every byte of a lost frame (loss_mask[t][f] == 0) of the
// packed voltage becomes 0, in place; valid_counts (uint32
// [ceil(T / integration_spectra)][F], may be null) gets the valid frames per
// integration window and channel.  Device pointers, caller's stream.
void launch_apply_loss_mask(cudaStream_t stream, std::uint8_t* packed_voltage, const std::uint8_t* loss_mask,
                            const Dimensions& dims, std::size_t integration_spectra, std::uint32_t* valid_counts);

// Bytes of the TensorSplit weight operand for `dims` (one shard).
std::size_t split_weight_bytes(const Dimensions& dims);

// Canonical device weights -> TensorSplit operand (device, split_weight_bytes).
void prepare_split_weights(cudaStream_t stream, const ComplexFloat* weights, void* split_weights,
                           const Dimensions& dims);

// Bytes of the TensorCovariance weight operand for `dims` (one shard), and the
// conversion from canonical device weights.
std::size_t cov_weight_bytes(const Dimensions& dims);
void prepare_cov_weights(cudaStream_t stream, const ComplexFloat* weights, void* cov_weights,
                         const Dimensions& dims);

// TensorChecked: operand bytes and preparation from canonical device weights,
// workspace bytes (device, may be 0), and the stage call (bf_grid_auto_* of
// the C ABI).  After the call the workspace's first 32-bit word holds how many
// split-kernel units were recomputed.
std::size_t checked_weight_bytes(const Dimensions& dims);
void prepare_checked_weights(cudaStream_t stream, const ComplexFloat* weights, void* checked_weights,
                             const Dimensions& dims);
std::size_t checked_workspace_bytes(const Dimensions& dims, const TemporalIntegrationConfig& temporal_integration);
void launch_checked_integrated_beamformer(cudaStream_t stream, const std::uint8_t* packed_voltage,
                                          const void* checked_weights, float* integrated_intensity, void* workspace,
                                          const Dimensions& dims,
                                          const TemporalIntegrationConfig& temporal_integration);

}  // namespace beamformer
