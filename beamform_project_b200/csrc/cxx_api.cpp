// cxx_api.cpp -- the reference's C++ interface (include/beamformer/) over the
// C ABI (include/bf_b200.h).
//
// Every call goes through the C ABI; a non-OK status is rethrown as the
// exception type the reference uses for that failure (std::invalid_argument,
// std::logic_error, std::runtime_error, std::overflow_error,
// std::out_of_range), with the reference's message text where it has one.
// Workspace structure follows the reference's CudaBeamformerWorkspace
// (src/cuda_beamformer.cu:545-1079): device buffers sized for a capacity,
// weights resident, voltage uploaded per call, CUDA-event timings per phase.
#include "beamformer/cuda_beam_tracker_v5.hpp"
#include "beamformer/cuda_beamformer.hpp"
#include "beamformer/served.hpp"
#include "bf_b200.h"

#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace beamformer {
namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kSpeedOfLight = 299'792'458.0;

std::string last_error_text() {
    char buf[1024];
    bf_last_error(buf, sizeof(buf));
    return std::string(buf);
}

void check(bf_status st) {
    if (st == BF_OK) return;
    const std::string msg = last_error_text();
    switch (st) {
        case BF_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
        case BF_ERR_LOGIC: throw std::logic_error(msg);
        case BF_ERR_OVERFLOW: throw std::overflow_error(msg);
        case BF_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
        case BF_ERR_UNSUPPORTED: throw std::invalid_argument(msg);
        case BF_ERR_RESOURCE: throw std::length_error(msg);
        default: throw std::runtime_error(msg);
    }
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

bf_dims to_c(const Dimensions& d) { return bf_dims{d.n_time, d.n_freq, d.n_ant, d.n_beams}; }

int to_c(CudaBeamformerKernel k) {
    switch (k) {
        case CudaBeamformerKernel::Direct: return BF_KERNEL_DIRECT;
        case CudaBeamformerKernel::Tiled: return BF_KERNEL_TILED;
        case CudaBeamformerKernel::TensorSplit: return BF_KERNEL_TENSOR;
        case CudaBeamformerKernel::TensorCovariance: break;  // its own entry points
        case CudaBeamformerKernel::TensorChecked: break;
    }
    throw std::invalid_argument("unknown CUDA beamformer kernel selector");
}

// The reference's integration-length rule (src/cuda_beamformer.cu:418-433).
void validate_cuda_temporal_integration(CudaBeamformerKernel kernel, const TemporalIntegrationConfig& t) {
    validate_temporal_config(t);
    const std::size_t s = t.integration_spectra;
    if (kernel == CudaBeamformerKernel::TensorCovariance) {
        if (s < 64 || s % 64 != 0 || s > 16384) {
            throw std::invalid_argument(
                "the TensorCovariance kernel needs integration spectra a multiple of 64, at most 16384");
        }
        return;
    }
    if (kernel == CudaBeamformerKernel::TensorSplit || kernel == CudaBeamformerKernel::TensorChecked) {
        if (s > 32 && s % 32 != 0) {
            throw std::invalid_argument(
                "the tensor-core kernels need integration spectra below 32 or a multiple of 32");
        }
        return;
    }
    if (s != integration_after_upchan.integration_spectra && s != integration_direct.integration_spectra) {
        throw std::invalid_argument("CUDA temporal integration supports only 10 or 320 spectra");
    }
    if (kernel == CudaBeamformerKernel::Direct && s != integration_direct.integration_spectra) {
        throw std::invalid_argument("the Direct CUDA kernel supports only 320-spectrum temporal integration");
    }
}

template <class T>
struct DeviceBuffer {
    T* ptr = nullptr;
    std::size_t count = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t n) : count(n) {
        if (n) check_cuda(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)), "cudaMalloc");
    }
    ~DeviceBuffer() {
        if (ptr) cudaFree(ptr);
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), count(o.count) { o.ptr = nullptr; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        std::swap(ptr, o.ptr);
        std::swap(count, o.count);
        return *this;
    }
};

struct Event {
    cudaEvent_t e = nullptr;
    Event() { check_cuda(cudaEventCreate(&e), "cudaEventCreate"); }
    ~Event() {
        if (e) cudaEventDestroy(e);
    }
    Event(const Event&) = delete;
    Event& operator=(const Event&) = delete;
};

float elapsed(const Event& a, const Event& b) {
    float ms = 0.f;
    check_cuda(cudaEventElapsedTime(&ms, a.e, b.e), "cudaEventElapsedTime");
    return ms;
}

std::size_t weight_storage_count(const Dimensions& dims, CudaBeamformerKernel kernel) {
    return kernel == CudaBeamformerKernel::Tiled ? tiled_weight_count(dims) : dims.n_beams * dims.n_freq * dims.n_ant;
}

}  // namespace

// --------------------------------------------------------------------------
// stage API
// --------------------------------------------------------------------------

void launch_packed_beamformer(CudaBeamformerKernel kernel, cudaStream_t stream, const std::uint8_t* packed_voltage,
                              const ComplexFloat* weights, float* intensity, const Dimensions& dims) {
    validate_dimensions(dims);
    if (kernel == CudaBeamformerKernel::TensorSplit || kernel == CudaBeamformerKernel::TensorCovariance ||
        kernel == CudaBeamformerKernel::TensorChecked) {
        throw std::invalid_argument("the tensor-core kernels produce integrated output only");
    }
    const bf_dims d = to_c(dims);
    check(bf_launch_packed_beamformer(to_c(kernel), stream, packed_voltage,
                                      reinterpret_cast<const float*>(weights), intensity, &d));
}

void launch_packed_integrated_beamformer(CudaBeamformerKernel kernel, cudaStream_t stream,
                                         const std::uint8_t* packed_voltage, const ComplexFloat* weights,
                                         float* integrated_intensity, const Dimensions& dims,
                                         const TemporalIntegrationConfig& temporal_integration) {
    validate_dimensions(dims);
    validate_cuda_temporal_integration(kernel, temporal_integration);
    const bf_dims d = to_c(dims);
    if (kernel == CudaBeamformerKernel::TensorChecked) {
        throw std::invalid_argument(
            "the TensorChecked kernel needs a workspace: use launch_checked_integrated_beamformer");
    }
    if (kernel == CudaBeamformerKernel::TensorCovariance) {
        // `weights` is the operand prepared by prepare_cov_weights
        check(bf_grid_cov_integrated(stream, packed_voltage, weights, integrated_intensity, nullptr, nullptr, &d,
                                     temporal_integration.integration_spectra, 1));
        return;
    }
    if (kernel == CudaBeamformerKernel::TensorSplit) {
        // `weights` is the operand prepared by prepare_split_weights
        check(bf_grid_tensor_integrated(stream, packed_voltage, weights, integrated_intensity, nullptr, nullptr, &d,
                                        temporal_integration.integration_spectra, 1));
        return;
    }
    check(bf_launch_packed_integrated_beamformer(to_c(kernel), stream, packed_voltage,
                                                 reinterpret_cast<const float*>(weights), integrated_intensity, &d,
                                                 temporal_integration.integration_spectra));
}

void launch_quantize_integrated_intensity(cudaStream_t stream, const float* integrated_intensity,
                                          std::int8_t* quantized_intensity, Int8QuantizationParameters* parameters,
                                          const Dimensions& integrated_dims) {
    const std::size_t chunks = quantization_parameter_count(integrated_dims);
    if (chunks > std::numeric_limits<unsigned int>::max()) {
        throw std::overflow_error("CUDA quantization grid exceeds the supported size");
    }
    const bf_dims d = to_c(integrated_dims);
    check(bf_launch_quantize_integrated_intensity(stream, integrated_intensity, quantized_intensity,
                                                  reinterpret_cast<float*>(parameters), &d));
}

void launch_apply_loss_mask(cudaStream_t stream, std::uint8_t* packed_voltage, const std::uint8_t* loss_mask,
                            const Dimensions& dims, std::size_t integration_spectra, std::uint32_t* valid_counts) {
    const bf_dims d = to_c(dims);
    check(bf_apply_loss_mask(stream, packed_voltage, loss_mask, &d, integration_spectra, valid_counts));
}

std::size_t split_weight_bytes(const Dimensions& dims) {
    const bf_dims d = to_c(dims);
    return static_cast<std::size_t>(bf_split_weight_bytes(&d, 1));
}

void prepare_split_weights(cudaStream_t stream, const ComplexFloat* weights, void* split_weights,
                           const Dimensions& dims) {
    const bf_dims d = to_c(dims);
    check(bf_prepare_split_weights(stream, reinterpret_cast<const float*>(weights), split_weights, &d, 1));
}

std::size_t cov_weight_bytes(const Dimensions& dims) {
    const bf_dims d = to_c(dims);
    return static_cast<std::size_t>(bf_cov_weight_bytes(&d, 1));
}

void prepare_cov_weights(cudaStream_t stream, const ComplexFloat* weights, void* cov_weights,
                         const Dimensions& dims) {
    const bf_dims d = to_c(dims);
    check(bf_prepare_cov_weights(stream, reinterpret_cast<const float*>(weights), cov_weights, &d, 1));
}

std::size_t checked_weight_bytes(const Dimensions& dims) {
    const bf_dims d = to_c(dims);
    return static_cast<std::size_t>(bf_auto_weight_bytes(&d, 1));
}

void prepare_checked_weights(cudaStream_t stream, const ComplexFloat* weights, void* checked_weights,
                             const Dimensions& dims) {
    const bf_dims d = to_c(dims);
    check(bf_prepare_auto_weights(stream, reinterpret_cast<const float*>(weights), checked_weights, &d, 1));
}

std::size_t checked_workspace_bytes(const Dimensions& dims, const TemporalIntegrationConfig& temporal_integration) {
    const bf_dims d = to_c(dims);
    return static_cast<std::size_t>(bf_grid_auto_workspace_bytes(&d, temporal_integration.integration_spectra, 1));
}

void launch_checked_integrated_beamformer(cudaStream_t stream, const std::uint8_t* packed_voltage,
                                          const void* checked_weights, float* integrated_intensity, void* workspace,
                                          const Dimensions& dims,
                                          const TemporalIntegrationConfig& temporal_integration) {
    validate_dimensions(dims);
    validate_cuda_temporal_integration(CudaBeamformerKernel::TensorChecked, temporal_integration);
    const bf_dims d = to_c(dims);
    check(bf_grid_auto_integrated(stream, packed_voltage, checked_weights, integrated_intensity, nullptr, nullptr,
                                  workspace, &d, temporal_integration.integration_spectra, 1));
}

CudaDeviceInfo cuda_device_info() {
    CudaDeviceInfo info;
    char name[256];
    uint64_t mem = 0;
    check(bf_device_info(name, sizeof(name), &info.compute_major, &info.compute_minor, &mem, &info.driver_version,
                         &info.runtime_version));
    info.name = name;
    info.global_memory_bytes = static_cast<std::size_t>(mem);
    return info;
}

// --------------------------------------------------------------------------
// workspace
// --------------------------------------------------------------------------

struct CudaBeamformerWorkspace::Impl {
    Dimensions capacity;
    CudaBeamformerKernel kernel;
    std::optional<TemporalIntegrationConfig> temporal;
    CudaBeamformerOutput output;
    DeviceBuffer<std::uint8_t> voltage;
    DeviceBuffer<ComplexFloat> weights;     // canonical or tiled
    DeviceBuffer<std::uint8_t> split;       // TensorSplit / TensorCovariance / TensorChecked operand
    DeviceBuffer<std::uint8_t> scratch;     // TensorChecked fallback list
    DeviceBuffer<float> intensity;          // per-spectrum output
    DeviceBuffer<float> integrated;
    DeviceBuffer<std::int8_t> codes;
    DeviceBuffer<Int8QuantizationParameters> params;
    cudaStream_t stream = nullptr;
    Event start, transfer_end, kernel_end, quant_end, d2d_end, result_end;
    double setup_ms = 0.0;
    std::size_t loaded_voltage = 0;
    std::size_t loaded_weights = 0;

    Impl(const Dimensions& cap, CudaBeamformerKernel k, std::optional<TemporalIntegrationConfig> t,
         CudaBeamformerOutput o)
        : capacity(cap), kernel(k), temporal(t), output(o), voltage(voltage_sample_count(cap)) {
        check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (tensor()) {
            weights = DeviceBuffer<ComplexFloat>(cap.n_beams * cap.n_freq * cap.n_ant);
            split = DeviceBuffer<std::uint8_t>(kernel == CudaBeamformerKernel::TensorSplit ? split_weight_bytes(cap)
                                               : kernel == CudaBeamformerKernel::TensorChecked
                                                   ? checked_weight_bytes(cap)
                                                   : cov_weight_bytes(cap));
            if (kernel == CudaBeamformerKernel::TensorChecked && t) {
                scratch = DeviceBuffer<std::uint8_t>(checked_workspace_bytes(cap, *t));
            }
        } else {
            weights = DeviceBuffer<ComplexFloat>(weight_storage_count(cap, kernel));
        }
        if (!temporal) intensity = DeviceBuffer<float>(cap.n_time * cap.n_freq * cap.n_beams);
        if (temporal) {
            integrated = DeviceBuffer<float>(integrated_intensity_count(cap, *temporal));
            if (output == CudaBeamformerOutput::QuantizedInt8) {
                const Dimensions qd{integrated_time_count(cap.n_time, *temporal), cap.n_freq, cap.n_ant,
                                    cap.n_beams};
                codes = DeviceBuffer<std::int8_t>(integrated_intensity_count(cap, *temporal));
                params = DeviceBuffer<Int8QuantizationParameters>(quantization_parameter_count(qd));
            }
        }
    }
    ~Impl() {
        if (stream) cudaStreamDestroy(stream);
    }

    bool tensor() const {
        return kernel == CudaBeamformerKernel::TensorSplit || kernel == CudaBeamformerKernel::TensorCovariance ||
               kernel == CudaBeamformerKernel::TensorChecked;
    }
    void validate_request(const Dimensions& dims) const {
        validate_dimensions(dims);
        if (dims.n_freq != capacity.n_freq || dims.n_ant != capacity.n_ant || dims.n_time > capacity.n_time ||
            dims.n_beams > capacity.n_beams) {
            throw std::invalid_argument("dimensions exceed CUDA workspace capacity");
        }
    }
    std::size_t required_weights(const Dimensions& dims) const {
        return tensor() ? dims.n_beams * dims.n_freq * dims.n_ant : weight_storage_count(dims, kernel);
    }
    void require_weights(const Dimensions& dims) const {
        if (loaded_weights != required_weights(dims)) {
            throw std::logic_error("weights have not been uploaded for these dimensions");
        }
    }
    void require_temporal() const {
        if (!temporal) throw std::logic_error("CUDA workspace was not constructed with temporal integration");
    }
    void require_quantization() const {
        require_temporal();
        if (output != CudaBeamformerOutput::QuantizedInt8) {
            throw std::logic_error("CUDA workspace was not constructed with int8 quantization");
        }
    }
    // Launch the configured beamformer into the configured output buffer.
    void launch(const Dimensions& dims, const std::uint8_t* v, const void* w, float* out) {
        const bf_dims d = to_c(dims);
        if (kernel == CudaBeamformerKernel::TensorChecked) {
            // the workspace is sized for the capacity; a shorter request needs no more
            if (checked_workspace_bytes(dims, *temporal) > scratch.count) {
                throw std::invalid_argument("dimensions exceed CUDA workspace capacity");
            }
            check(bf_grid_auto_integrated(stream, v, w, out, nullptr, nullptr, scratch.ptr, &d,
                                          temporal->integration_spectra, 1));
        } else if (kernel == CudaBeamformerKernel::TensorCovariance) {
            check(bf_grid_cov_integrated(stream, v, w, out, nullptr, nullptr, &d, temporal->integration_spectra, 1));
        } else if (kernel == CudaBeamformerKernel::TensorSplit) {
            // per-spectrum output is integration over one spectrum ([T][F][B] == [W][F][B])
            check(bf_grid_tensor_integrated(stream, v, w, out, nullptr, nullptr, &d,
                                            temporal ? temporal->integration_spectra : 1, 1));
        } else if (temporal) {
            check(bf_launch_packed_integrated_beamformer(to_c(kernel), stream, v, static_cast<const float*>(w), out,
                                                         &d, temporal->integration_spectra));
        } else {
            check(bf_launch_packed_beamformer(to_c(kernel), stream, v, static_cast<const float*>(w), out, &d));
        }
    }
    const void* weight_operand() const {
        return tensor() ? static_cast<const void*>(split.ptr) : static_cast<const void*>(weights.ptr);
    }
    // canonical weights on the device -> the tensor kernels' operand
    void prepare_operand(const void* canonical, const Dimensions& dims) {
        const bf_dims d = to_c(dims);
        if (kernel == CudaBeamformerKernel::TensorSplit) {
            check(bf_prepare_split_weights(stream, static_cast<const float*>(canonical), split.ptr, &d, 1));
        } else if (kernel == CudaBeamformerKernel::TensorCovariance) {
            check(bf_prepare_cov_weights(stream, static_cast<const float*>(canonical), split.ptr, &d, 1));
        } else if (kernel == CudaBeamformerKernel::TensorChecked) {
            check(bf_prepare_auto_weights(stream, static_cast<const float*>(canonical), split.ptr, &d, 1));
        }
    }
};

CudaBeamformerWorkspace::CudaBeamformerWorkspace(const Dimensions& capacity, CudaBeamformerKernel kernel,
                                                 std::optional<TemporalIntegrationConfig> temporal_integration,
                                                 CudaBeamformerOutput output) {
    validate_dimensions(capacity);
    if (temporal_integration) validate_cuda_temporal_integration(kernel, *temporal_integration);
    if (output == CudaBeamformerOutput::QuantizedInt8 && !temporal_integration) {
        throw std::invalid_argument("int8 quantization requires a temporal-integration configuration");
    }
    if (kernel == CudaBeamformerKernel::TensorChecked) {
        if (!temporal_integration) {
            throw std::invalid_argument("the TensorChecked kernel produces integrated output only");
        }
    }
    if (kernel == CudaBeamformerKernel::TensorCovariance) {
        if (capacity.n_ant != 64) throw std::invalid_argument("the TensorCovariance kernel supports n_ant 64");
        if (!temporal_integration) {
            throw std::invalid_argument("the TensorCovariance kernel produces integrated output only");
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    impl_ = std::make_unique<Impl>(capacity, kernel, temporal_integration, output);
    impl_->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

CudaBeamformerWorkspace::~CudaBeamformerWorkspace() = default;

double CudaBeamformerWorkspace::setup_ms() const { return impl_->setup_ms; }
CudaBeamformerKernel CudaBeamformerWorkspace::kernel() const { return impl_->kernel; }
bool CudaBeamformerWorkspace::has_temporal_integration() const { return impl_->temporal.has_value(); }
bool CudaBeamformerWorkspace::has_int8_quantization() const {
    return impl_->output == CudaBeamformerOutput::QuantizedInt8;
}
std::size_t CudaBeamformerWorkspace::packed_voltage_capacity_bytes() const {
    return voltage_sample_count(impl_->capacity);
}

double CudaBeamformerWorkspace::upload_packed_voltage(const PackedVoltage& packed, const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    const std::size_t n = voltage_sample_count(dims);
    if (packed.size() < n) throw std::invalid_argument("packed voltage is smaller than dimensions");
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(m.voltage.ptr, packed.data(), n, cudaMemcpyHostToDevice, m.stream), "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.transfer_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.transfer_end.e), "cudaEventSynchronize");
    m.loaded_voltage = n;
    return elapsed(m.start, m.transfer_end);
}

double CudaBeamformerWorkspace::upload_weights(const Weights& weights, const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    const std::size_t n = m.required_weights(dims);
    if (weights.size() != n) throw std::invalid_argument("weight count does not match selected kernel layout");
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(m.weights.ptr, weights.data(), n * sizeof(ComplexFloat), cudaMemcpyHostToDevice,
                               m.stream),
               "cudaMemcpyAsync weights");
    m.prepare_operand(m.weights.ptr, dims);
    check_cuda(cudaEventRecord(m.transfer_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.transfer_end.e), "cudaEventSynchronize");
    m.loaded_weights = n;
    return elapsed(m.start, m.transfer_end);
}

double CudaBeamformerWorkspace::run_kernel(const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    if (m.loaded_voltage < voltage_sample_count(dims)) {
        throw std::logic_error("packed voltage has not been uploaded for these dimensions");
    }
    m.require_weights(dims);
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    m.launch(Dimensions{dims}, m.voltage.ptr, m.weight_operand(), m.temporal ? m.integrated.ptr : m.intensity.ptr);
    check_cuda(cudaEventRecord(m.kernel_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.kernel_end.e), "cudaEventSynchronize");
    return elapsed(m.start, m.kernel_end);
}

double CudaBeamformerWorkspace::download_intensity(Intensities& intensity, const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    const std::size_t n = dims.n_time * dims.n_freq * dims.n_beams;
    if (intensity.size() < n) throw std::invalid_argument("intensity output is smaller than dimensions");
    if (!m.intensity.ptr) throw std::logic_error("this workspace has no per-spectrum intensity buffer");
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(intensity.data(), m.intensity.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, m.stream),
               "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.result_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.result_end.e), "cudaEventSynchronize");
    return elapsed(m.start, m.result_end);
}

CudaBeamformerTimings CudaBeamformerWorkspace::run_pipeline(const PackedVoltage& packed, Intensities& intensity,
                                                            const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    if (m.temporal) {
        throw std::logic_error("run_pipeline needs a per-spectrum (non-integrating) workspace");
    }
    const std::size_t nv = voltage_sample_count(dims), no = dims.n_time * dims.n_freq * dims.n_beams;
    if (packed.size() < nv) throw std::invalid_argument("packed voltage is smaller than dimensions");
    if (intensity.size() < no) throw std::invalid_argument("intensity output is smaller than dimensions");
    m.require_weights(dims);
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(m.voltage.ptr, packed.data(), nv, cudaMemcpyHostToDevice, m.stream), "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.transfer_end.e, m.stream), "cudaEventRecord");
    m.launch(dims, m.voltage.ptr, m.weight_operand(), m.intensity.ptr);
    check_cuda(cudaEventRecord(m.kernel_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(intensity.data(), m.intensity.ptr, no * sizeof(float), cudaMemcpyDeviceToHost,
                               m.stream),
               "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.result_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.result_end.e), "cudaEventSynchronize");
    m.loaded_voltage = nv;
    CudaBeamformerTimings t;
    t.host_to_device_ms = elapsed(m.start, m.transfer_end);
    t.kernel_ms = elapsed(m.transfer_end, m.kernel_end);
    t.device_to_host_ms = elapsed(m.kernel_end, m.result_end);
    return t;
}

CudaBeamformerTimings CudaBeamformerWorkspace::run_integrated_pipeline(const PackedVoltage& packed,
                                                                       IntegratedIntensities& intensity,
                                                                       const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    m.require_temporal();
    const std::size_t nv = voltage_sample_count(dims), no = integrated_intensity_count(dims, *m.temporal);
    if (packed.size() < nv) throw std::invalid_argument("packed voltage is smaller than dimensions");
    if (intensity.size() < no) throw std::invalid_argument("integrated intensity output is smaller than dimensions");
    m.require_weights(dims);
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(m.voltage.ptr, packed.data(), nv, cudaMemcpyHostToDevice, m.stream), "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.transfer_end.e, m.stream), "cudaEventRecord");
    m.launch(dims, m.voltage.ptr, m.weight_operand(), m.integrated.ptr);
    check_cuda(cudaEventRecord(m.kernel_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(intensity.data(), m.integrated.ptr, no * sizeof(float), cudaMemcpyDeviceToHost,
                               m.stream),
               "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.result_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.result_end.e), "cudaEventSynchronize");
    m.loaded_voltage = nv;
    CudaBeamformerTimings t;
    t.host_to_device_ms = elapsed(m.start, m.transfer_end);
    t.kernel_ms = elapsed(m.transfer_end, m.kernel_end);
    t.device_to_host_ms = elapsed(m.kernel_end, m.result_end);
    return t;
}

CudaBeamformerTimings CudaBeamformerWorkspace::run_quantized_integrated_pipeline(const PackedVoltage& packed,
                                                                                 QuantizedIntegratedOutput& out,
                                                                                 const Dimensions& dims) {
    auto& m = *impl_;
    m.validate_request(dims);
    m.require_quantization();
    const std::size_t nv = voltage_sample_count(dims), no = integrated_intensity_count(dims, *m.temporal);
    const Dimensions qd{integrated_time_count(dims.n_time, *m.temporal), dims.n_freq, dims.n_ant, dims.n_beams};
    const std::size_t np = quantization_parameter_count(qd);
    if (packed.size() < nv) throw std::invalid_argument("packed voltage is smaller than dimensions");
    if (out.codes.size() < no || out.parameters.size() < np) {
        throw std::invalid_argument("quantized output is smaller than dimensions");
    }
    m.require_weights(dims);
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(m.voltage.ptr, packed.data(), nv, cudaMemcpyHostToDevice, m.stream), "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.transfer_end.e, m.stream), "cudaEventRecord");
    m.launch(dims, m.voltage.ptr, m.weight_operand(), m.integrated.ptr);
    check_cuda(cudaEventRecord(m.kernel_end.e, m.stream), "cudaEventRecord");
    launch_quantize_integrated_intensity(m.stream, m.integrated.ptr, m.codes.ptr, m.params.ptr, qd);
    check_cuda(cudaEventRecord(m.quant_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(out.codes.data(), m.codes.ptr, no, cudaMemcpyDeviceToHost, m.stream), "cudaMemcpyAsync");
    check_cuda(cudaMemcpyAsync(out.parameters.data(), m.params.ptr, np * sizeof(Int8QuantizationParameters),
                               cudaMemcpyDeviceToHost, m.stream),
               "cudaMemcpyAsync");
    check_cuda(cudaEventRecord(m.result_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.result_end.e), "cudaEventSynchronize");
    m.loaded_voltage = nv;
    CudaBeamformerTimings t;
    t.host_to_device_ms = elapsed(m.start, m.transfer_end);
    t.kernel_ms = elapsed(m.transfer_end, m.kernel_end);
    t.quantization_ms = elapsed(m.kernel_end, m.quant_end);
    t.device_to_host_ms = elapsed(m.quant_end, m.result_end);
    return t;
}

CudaChunkedGridPipeline::CudaChunkedGridPipeline(const Dimensions& dims,
                                                 const TemporalIntegrationConfig& temporal_integration,
                                                 std::size_t n_shards, std::size_t chunk_spectra)
    : dims_(dims), spectra_(temporal_integration.integration_spectra), n_shards_(n_shards) {
    validate_dimensions(dims);
    const bf_dims d = to_c(dims);
    check(bf_grid_pipeline_create(&d, spectra_, n_shards_, chunk_spectra, &pipeline_));
    chunk_ = bf_grid_pipeline_chunk_spectra(&d, spectra_, n_shards_, chunk_spectra);
}

CudaChunkedGridPipeline::~CudaChunkedGridPipeline() { bf_grid_pipeline_destroy(pipeline_); }

std::size_t CudaChunkedGridPipeline::chunk_spectra() const { return chunk_; }

void CudaChunkedGridPipeline::upload_weights(const Weights& weights) {
    if (weights.size() != n_shards_ * dims_.n_beams * dims_.n_freq * dims_.n_ant) {
        throw std::invalid_argument("weight count does not match selected kernel layout");
    }
    check(bf_grid_pipeline_upload_weights(pipeline_, reinterpret_cast<const float*>(weights.data())));
}

double CudaChunkedGridPipeline::run(const PackedVoltage& packed, IntegratedIntensities* integrated,
                                   QuantizedIntegratedOutput* quantized) {
    if (packed.size() < n_shards_ * voltage_sample_count(dims_)) {
        throw std::invalid_argument("packed voltage is smaller than dimensions");
    }
    const Dimensions qd{integrated_time_count(dims_.n_time, TemporalIntegrationConfig{spectra_}), dims_.n_freq,
                        dims_.n_ant, dims_.n_beams};
    const std::size_t n_out = n_shards_ * qd.n_time * qd.n_freq * qd.n_beams;
    if (integrated != nullptr) integrated->resize(n_out);
    if (quantized != nullptr) {
        quantized->codes.resize(n_out);
        quantized->parameters.resize(n_shards_ * quantization_parameter_count(qd));
    }
    float ms = 0.0F;
    check(bf_grid_pipeline_run(pipeline_, packed.data(), integrated ? integrated->data() : nullptr,
                               quantized ? quantized->codes.data() : nullptr,
                               quantized ? reinterpret_cast<float*>(quantized->parameters.data()) : nullptr, &ms));
    return ms;
}

namespace {
bool same_shard(const ShardDescriptor& a, const ShardDescriptor& b) {
    return a.shard_id == b.shard_id && a.shard_count == b.shard_count &&
           a.local_frequency_count == b.local_frequency_count &&
           a.absolute_frequency_start == b.absolute_frequency_start && a.timestamp_start == b.timestamp_start &&
           a.timestamp_step == b.timestamp_step && a.loss_mask_id == b.loss_mask_id &&
           a.loss_mask_independent == b.loss_mask_independent;
}

void check_frame_shape(const CudaFrameView& f, CudaDataType type, std::size_t rank, const FrameShape& shape,
                       const char* label) {
    validate_contiguous_cuda_buffer_view(f.buffer);
    if (f.buffer.type != type || f.buffer.rank != rank || f.buffer.shape != shape) {
        throw std::invalid_argument(std::string(label) + " shape or dtype does not match");
    }
}
}  // namespace

// Offline device frame (reference src/cuda_beamformer.cu:930-1079): checks
// frame ids, shard metadata, shapes and dtypes, then runs the configured
// stages straight into the caller's output buffer (no device-to-device copy).
CudaBeamformerTimings CudaBeamformerWorkspace::run_device_frame(const CudaFrameView& voltage,
                                                                const CudaFrameView& weights, CudaFrameView& output,
                                                                CudaFrameView* quantization_parameters) {
    auto& m = *impl_;
    validate_cuda_frame_view(voltage);
    validate_cuda_frame_view(weights);
    validate_cuda_frame_view(output);
    if (voltage.metadata.frame_id != output.metadata.frame_id) {
        throw std::invalid_argument("output frame_id does not match input");
    }
    if (!same_shard(voltage.metadata.shard, output.metadata.shard)) {
        throw std::invalid_argument("output shard metadata does not match input");
    }
    if (voltage.buffer.type != CudaDataType::PackedInt4x2 || voltage.buffer.rank != 3) {
        throw std::invalid_argument("offline device frame voltage must be packed int4x2 with rank 3");
    }
    if (output.buffer.rank != 3) throw std::invalid_argument("offline device frame dimensions do not match");
    const Dimensions dims{voltage.buffer.shape[0], voltage.buffer.shape[1], voltage.buffer.shape[2],
                          output.buffer.shape[2]};
    m.validate_request(dims);
    if (output.buffer.shape[1] != dims.n_freq) throw std::invalid_argument("offline device frame dimensions do not match");
    const bool tiled = m.kernel == CudaBeamformerKernel::Tiled;
    const FrameShape wshape = tiled ? FrameShape{dims.n_freq, tiled_weight_beam_tiles(dims), dims.n_ant,
                                                 tiled_weight_beam_tile}
                                    : FrameShape{dims.n_beams, dims.n_freq, dims.n_ant, 0};
    check_frame_shape(weights, CudaDataType::ComplexFloat32, tiled ? 4 : 3, wshape, "offline device frame weights");
    if (!same_shard(voltage.metadata.shard, weights.metadata.shard)) {
        throw std::invalid_argument("offline device frame weights shard does not match input");
    }
    Dimensions od = dims;
    if (m.temporal) od.n_time = integrated_time_count(dims.n_time, *m.temporal);
    const bool quant = m.output == CudaBeamformerOutput::QuantizedInt8;
    check_frame_shape(output, quant ? CudaDataType::SignedInt8 : CudaDataType::Float32, 3,
                      {od.n_time, od.n_freq, od.n_beams, 0}, "offline device frame output");
    if (quant) {
        if (!m.temporal || quantization_parameters == nullptr) {
            throw std::invalid_argument("offline int8 output requires temporal integration parameters");
        }
        validate_cuda_frame_view(*quantization_parameters);
        if (quantization_parameters->metadata.frame_id != voltage.metadata.frame_id) {
            throw std::invalid_argument("quantization parameters frame_id does not match input");
        }
        if (!same_shard(voltage.metadata.shard, quantization_parameters->metadata.shard)) {
            throw std::invalid_argument("quantization parameters shard metadata does not match input");
        }
        const auto l = quantization_layout(od);
        check_frame_shape(*quantization_parameters, CudaDataType::Float32, 4,
                          {l.time_tiles, l.frequency_tiles, l.beam_tiles, 2}, "offline quantization parameters");
    } else if (quantization_parameters != nullptr) {
        throw std::invalid_argument("float32 offline output must not provide quantization parameters");
    }

    const auto* v = static_cast<const std::uint8_t*>(voltage.buffer.device_data);
    const void* w = weights.buffer.device_data;
    CudaBeamformerTimings t;
    check_cuda(cudaEventRecord(m.start.e, m.stream), "cudaEventRecord");
    if (m.tensor()) {
        m.prepare_operand(w, dims);
        w = m.split.ptr;
    }
    check_cuda(cudaEventRecord(m.transfer_end.e, m.stream), "cudaEventRecord");
    float* out = quant ? m.integrated.ptr : static_cast<float*>(output.buffer.device_data);
    m.launch(dims, v, w, out);
    check_cuda(cudaEventRecord(m.kernel_end.e, m.stream), "cudaEventRecord");
    if (quant) {
        launch_quantize_integrated_intensity(m.stream, m.integrated.ptr, static_cast<std::int8_t*>(output.buffer.device_data),
                                             static_cast<Int8QuantizationParameters*>(quantization_parameters->buffer.device_data),
                                             od);
    }
    check_cuda(cudaEventRecord(m.quant_end.e, m.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(m.quant_end.e), "cudaEventSynchronize");
    t.kernel_ms = elapsed(m.transfer_end, m.kernel_end);
    t.quantization_ms = elapsed(m.kernel_end, m.quant_end);
    return t;
}

// --------------------------------------------------------------------------
// one-shot wrappers (reference src/cuda_beamformer.cu:1081-1173)
// --------------------------------------------------------------------------

Intensities cuda_beamform_packed_intensity(const PackedVoltage& packed, const Weights& weights, const Dimensions& dims,
                                           CudaBeamformerTimings* timings, CudaBeamformerKernel kernel) {
    validate_dimensions(dims);
    if (packed.size() != voltage_sample_count(dims)) {
        throw std::invalid_argument("packed voltage size does not match dimensions");
    }
    CudaBeamformerWorkspace ws(dims, kernel);
    Intensities out(dims.n_time * dims.n_freq * dims.n_beams);
    ws.upload_weights(weights, dims);
    auto t = ws.run_pipeline(packed, out, dims);
    t.setup_ms = ws.setup_ms();
    if (timings) *timings = t;
    return out;
}

IntegratedIntensities cuda_beamform_packed_integrated_intensity(const PackedVoltage& packed, const Weights& weights,
                                                                const Dimensions& dims,
                                                                const TemporalIntegrationConfig& temporal_integration,
                                                                CudaBeamformerTimings* timings,
                                                                CudaBeamformerKernel kernel) {
    validate_dimensions(dims);
    validate_cuda_temporal_integration(kernel, temporal_integration);
    if (packed.size() != voltage_sample_count(dims)) {
        throw std::invalid_argument("packed voltage size does not match dimensions");
    }
    CudaBeamformerWorkspace ws(dims, kernel, temporal_integration);
    IntegratedIntensities out(integrated_intensity_count(dims, temporal_integration));
    ws.upload_weights(weights, dims);
    auto t = ws.run_integrated_pipeline(packed, out, dims);
    t.setup_ms = ws.setup_ms();
    if (timings) *timings = t;
    return out;
}

QuantizedIntegratedOutput cuda_beamform_packed_quantized_integrated_intensity(
    const PackedVoltage& packed, const Weights& weights, const Dimensions& dims,
    const TemporalIntegrationConfig& temporal_integration, CudaBeamformerTimings* timings,
    CudaBeamformerKernel kernel) {
    validate_dimensions(dims);
    validate_cuda_temporal_integration(kernel, temporal_integration);
    if (packed.size() != voltage_sample_count(dims)) {
        throw std::invalid_argument("packed voltage size does not match dimensions");
    }
    CudaBeamformerWorkspace ws(dims, kernel, temporal_integration, CudaBeamformerOutput::QuantizedInt8);
    const Dimensions qd{integrated_time_count(dims.n_time, temporal_integration), dims.n_freq, dims.n_ant,
                        dims.n_beams};
    QuantizedIntegratedOutput out;
    out.codes.resize(integrated_intensity_count(dims, temporal_integration));
    out.parameters.resize(quantization_parameter_count(qd));
    ws.upload_weights(weights, dims);
    auto t = ws.run_quantized_integrated_pipeline(packed, out, dims);
    t.setup_ms = ws.setup_ms();
    if (timings) *timings = t;
    return out;
}

// --------------------------------------------------------------------------
// tracker (reference src/cuda_beam_tracker_v5.cu:278-605)
// --------------------------------------------------------------------------
namespace {

// Window directions and wave numbers of the default geometry / channel plan,
// like the reference's host pre-scan (src/cuda_beam_tracker_v5.cu:278-312).
void tracker_pre_scan(const Dimensions& dims, const TrackerConfig& tracker, std::size_t first_window,
                      std::vector<float>& dirs, std::vector<double>& k, std::vector<float>& pos) {
    validate_tracker_config(dims, tracker);
    const std::size_t W = tracker_window_count(dims.n_time, tracker.integration_spectra);
    dirs.resize(3 * W);
    for (std::size_t w = 0; w < W; ++w) {
        const Vec3 d = tracker_window_direction(tracker.trajectory, first_window + w, tracker.integration_spectra);
        dirs[3 * w] = d[0];
        dirs[3 * w + 1] = d[1];
        dirs[3 * w + 2] = d[2];
    }
    const auto f = channelized_frequencies(dims.n_freq);
    k.resize(dims.n_freq);
    for (std::size_t c = 0; c < dims.n_freq; ++c) k[c] = kTwoPi * static_cast<double>(f[c]) / kSpeedOfLight;
    const auto p = default_positions(dims.n_ant);
    pos.resize(3 * dims.n_ant);
    for (std::size_t a = 0; a < dims.n_ant; ++a)
        for (int c = 0; c < 3; ++c) pos[3 * a + c] = p[a][c];
}

struct TrackerGeometry {
    DeviceBuffer<float> dirs, pos;
    DeviceBuffer<double> k;
    void upload(const std::vector<float>& hd, const std::vector<double>& hk, const std::vector<float>& hp,
                cudaStream_t s) {
        if (dirs.count < hd.size()) dirs = DeviceBuffer<float>(hd.size());
        if (k.count < hk.size()) k = DeviceBuffer<double>(hk.size());
        if (pos.count < hp.size()) pos = DeviceBuffer<float>(hp.size());
        check_cuda(cudaMemcpyAsync(dirs.ptr, hd.data(), hd.size() * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        check_cuda(cudaMemcpyAsync(k.ptr, hk.data(), hk.size() * 8, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        check_cuda(cudaMemcpyAsync(pos.ptr, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    }
};

}  // namespace

void cuda_beam_tracker_device_resident_ex(const std::uint8_t* d_packed, const float* d_positions,
                                          const double* d_wave_numbers, const float* d_window_directions,
                                          float* d_intensity, float* d_integrated, const Dimensions& dims,
                                          std::size_t integration_spectra, void* stream) {
    const bf_dims d = to_c(dims);
    check(bf_tracker(stream, 1, d_packed, d_positions, d_wave_numbers, d_window_directions, d_intensity, d_integrated,
                     &d, integration_spectra));
}

void cuda_beam_tracker_v5_device_resident(const std::uint8_t* d_packed, float* d_intensity, const Dimensions& dims,
                                          const TrackerConfig& tracker, const V5ExecutionConfig&, void* stream) {
    std::vector<float> dirs, pos;
    std::vector<double> k;
    tracker_pre_scan(dims, tracker, 0, dirs, k, pos);
    auto s = static_cast<cudaStream_t>(stream);
    // small per-call geometry buffers, stream-ordered like the reference's
    // cudaMallocAsync / cudaFreeAsync pair (src/cuda_beam_tracker_v5.cu:383-420)
    float* dd = nullptr;
    float* dp = nullptr;
    double* dk = nullptr;
    check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&dd), dirs.size() * 4, s), "cudaMallocAsync");
    check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&dp), pos.size() * 4, s), "cudaMallocAsync");
    check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&dk), k.size() * 8, s), "cudaMallocAsync");
    check_cuda(cudaMemcpyAsync(dd, dirs.data(), dirs.size() * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    check_cuda(cudaMemcpyAsync(dp, pos.data(), pos.size() * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    check_cuda(cudaMemcpyAsync(dk, k.data(), k.size() * 8, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    const bf_dims d = to_c(dims);
    const bf_status st = bf_tracker(s, 1, d_packed, dp, dk, dd, d_intensity, nullptr, &d, tracker.integration_spectra);
    cudaFreeAsync(dd, s);
    cudaFreeAsync(dp, s);
    cudaFreeAsync(dk, s);
    check(st);
    // pageable host vectors must outlive the copies
    check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
}

void cuda_beam_tracker_v5_into(const PackedVoltage& packed, const Dimensions& dims, const TrackerConfig& tracker,
                               Intensities& intensity, const V5ExecutionConfig&) {
    std::vector<float> dirs, pos;
    std::vector<double> k;
    tracker_pre_scan(dims, tracker, 0, dirs, k, pos);
    if (packed.size() != voltage_sample_count(dims)) {
        throw std::invalid_argument("voltage buffer size does not match dimensions");
    }
    const std::size_t out_n = dims.n_time * dims.n_freq * dims.n_beams;
    if (intensity.size() != out_n) intensity.resize(out_n);
    cudaStream_t s = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    try {
        DeviceBuffer<std::uint8_t> dv(packed.size());
        DeviceBuffer<float> di(out_n);
        TrackerGeometry g;
        g.upload(dirs, k, pos, s);
        check_cuda(cudaMemcpyAsync(dv.ptr, packed.data(), packed.size(), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        const bf_dims d = to_c(dims);
        check(bf_tracker(s, 1, dv.ptr, g.pos.ptr, g.k.ptr, g.dirs.ptr, di.ptr, nullptr, &d, tracker.integration_spectra));
        check_cuda(cudaMemcpyAsync(intensity.data(), di.ptr, out_n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    } catch (...) {
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
}

Intensities cuda_beam_tracker_v5(const PackedVoltage& packed, const Dimensions& dims, const TrackerConfig& tracker,
                                 const V5ExecutionConfig& config) {
    Intensities out(dims.n_time * dims.n_freq * dims.n_beams);
    cuda_beam_tracker_v5_into(packed, dims, tracker, out, config);
    return out;
}

struct BatchedTrackerStreamV5::Impl {
    Dimensions win_dims, batch_dims;
    TrackerConfig tracker;
    std::size_t batch = 0;
    V5ExecutionConfig config;
    cudaStream_t stream = nullptr;
    Event start, stop;
    float last_ms = 0.f;
    DeviceBuffer<std::uint8_t> v;
    DeviceBuffer<float> out;
    TrackerGeometry geom;
    std::vector<float> dirs, pos;
    std::vector<double> k;
    std::size_t geometry_first_window = std::numeric_limits<std::size_t>::max();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;

    Impl(const Dimensions& w, const TrackerConfig& t, std::size_t b, const V5ExecutionConfig& c)
        : win_dims(w), tracker(t), batch(b), config(c) {
        if (b == 0) throw std::invalid_argument("batch_size must be positive");
        batch_dims = w;
        batch_dims.n_time = w.n_time * b;
        validate_tracker_config(batch_dims, tracker);
        check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        v = DeviceBuffer<std::uint8_t>(voltage_sample_count(batch_dims));
        out = DeviceBuffer<float>(batch_dims.n_time * batch_dims.n_freq);
        set_first_window(0);
    }
    ~Impl() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
    // The batch's windows start at absolute window first_window_index *
    // (window spectra / integration spectra); their directions are
    // refreshed when it changes (the reference uses window 0 for every batch).
    void set_first_window(std::size_t first) {
        if (first == geometry_first_window) return;
        const std::size_t windows_per_frame = win_dims.n_time / tracker.integration_spectra;
        tracker_pre_scan(batch_dims, tracker, first * windows_per_frame, dirs, k, pos);
        geom.upload(dirs, k, pos, stream);
        check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        geometry_first_window = first;
    }
    void launch() {
        const bf_dims d = to_c(batch_dims);
        check(bf_tracker(stream, 1, v.ptr, geom.pos.ptr, geom.k.ptr, geom.dirs.ptr, out.ptr, nullptr, &d,
                         tracker.integration_spectra));
    }
    void kernel_only(std::size_t first) {
        set_first_window(first);
        if (config.enable_cuda_graph) {
            if (!graph_exec) {
                check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "BeginCapture");
                launch();
                check_cuda(cudaStreamEndCapture(stream, &graph), "EndCapture");
                check_cuda(cudaGraphInstantiate(&graph_exec, graph, nullptr, nullptr, 0), "GraphInstantiate");
            }
            check_cuda(cudaEventRecord(start.e, stream), "cudaEventRecord");
            check_cuda(cudaGraphLaunch(graph_exec, stream), "cudaGraphLaunch");
        } else {
            check_cuda(cudaEventRecord(start.e, stream), "cudaEventRecord");
            launch();
        }
        check_cuda(cudaEventRecord(stop.e, stream), "cudaEventRecord");
        check_cuda(cudaEventSynchronize(stop.e), "cudaEventSynchronize");
        last_ms = elapsed(start, stop);
    }
};

BatchedTrackerStreamV5::BatchedTrackerStreamV5(const Dimensions& single_window_dims, const TrackerConfig& tracker,
                                               std::size_t batch_size, const V5ExecutionConfig& config)
    : impl_(std::make_unique<Impl>(single_window_dims, tracker, batch_size, config)) {}
BatchedTrackerStreamV5::~BatchedTrackerStreamV5() = default;

void BatchedTrackerStreamV5::process_batch(std::size_t first_window_index, const std::uint8_t* host_packed,
                                           float* host_intensity) {
    auto& m = *impl_;
    check_cuda(cudaMemcpyAsync(m.v.ptr, host_packed, voltage_sample_count(m.batch_dims), cudaMemcpyHostToDevice,
                               m.stream),
               "cudaMemcpyAsync");
    m.kernel_only(first_window_index);
    check_cuda(cudaMemcpyAsync(host_intensity, m.out.ptr, m.batch_dims.n_time * m.batch_dims.n_freq * 4,
                               cudaMemcpyDeviceToHost, m.stream),
               "cudaMemcpyAsync");
    check_cuda(cudaStreamSynchronize(m.stream), "cudaStreamSynchronize");
}
void BatchedTrackerStreamV5::process_batch_kernel_only(std::size_t first_window_index) {
    impl_->kernel_only(first_window_index);
}
float BatchedTrackerStreamV5::last_kernel_time_ms() const { return impl_->last_ms; }
std::uint8_t* BatchedTrackerStreamV5::device_packed_buffer() { return impl_->v.ptr; }
float* BatchedTrackerStreamV5::device_intensity_buffer() { return impl_->out.ptr; }
void* BatchedTrackerStreamV5::device_stream() { return impl_->stream; }
std::size_t BatchedTrackerStreamV5::batch_size() const { return impl_->batch; }
std::size_t BatchedTrackerStreamV5::window_bytes() const { return voltage_sample_count(impl_->win_dims); }
std::size_t BatchedTrackerStreamV5::batch_voltage_bytes() const { return voltage_sample_count(impl_->batch_dims); }
std::size_t BatchedTrackerStreamV5::batch_output_floats() const {
    return impl_->batch_dims.n_time * impl_->batch_dims.n_freq;
}

// ---------------------------------------------------------------------------
// ServedBeamformer (bf_serve_*)
// ---------------------------------------------------------------------------

namespace {

float generator_scale(float sigma) {
    // the generator's draw 2 * (sum of eight uniform 16-bit integers) - 8 * 65535
    // has variance 4 * 8 * (65536^2 - 1) / 12
    const double sd = std::sqrt(4.0 * 8.0 * (65536.0 * 65536.0 - 1.0) / 12.0);
    return static_cast<float>(static_cast<double>(sigma) / sd);
}

}  // namespace

ServedBeamformer::ServedBeamformer(const ServedConfig& c) {
    bf_serve_config cfg{};
    cfg.hbm_budget_bytes = c.hbm_budget_bytes;
    cfg.max_jobs = c.max_jobs;
    cfg.window_spectra = c.window_spectra;
    cfg.pool_spectra = c.pool_spectra;
    cfg.shard_channels = c.shard_channels;
    cfg.max_shards = c.max_shards;
    cfg.pool_seed = c.pool_seed;
    cfg.pool_scale = generator_scale(c.pool_sigma);
    cfg.window_budget_us = c.window_budget_us;
    cfg.windows_per_step = c.windows_per_step;
    check(bf_serve_create(&cfg, &server_));
}

ServedBeamformer::~ServedBeamformer() {
    if (server_ != nullptr) bf_serve_destroy(server_);
}

std::uint64_t ServedBeamformer::submit(const ServedJob& job) {
    if (job.positions.size() != job.n_ant) throw std::invalid_argument("position count must match n_ant");
    bf_serve_job j{};
    j.kind = job.kind == ServedJobKind::Grid ? BF_SERVE_GRID : BF_SERVE_TRACKER;
    j.n_ant = static_cast<uint32_t>(job.n_ant);
    j.n_shards = static_cast<uint32_t>(job.n_shards);
    j.n_beams = static_cast<uint32_t>(job.n_beams);
    j.n_spectra = job.n_spectra;
    j.integration_spectra = job.integration_spectra;
    j.pool_offset = job.pool_offset;
    j.positions = job.positions.empty() ? nullptr : job.positions.front().data();
    j.frequencies = job.frequencies_hz.empty() ? nullptr : job.frequencies_hz.data();
    if (job.kind == ServedJobKind::Grid) {
        if (job.directions.size() != job.n_beams) throw std::invalid_argument("beam direction count must match n_beams");
        j.directions = job.directions.front().data();
    } else {
        if (job.trajectories.size() != job.n_beams) throw std::invalid_argument("trajectory count must match n_beams");
        j.trajectories = job.trajectories.front().data();
    }
    j.quantize = job.quantize ? 1 : 0;
    std::uint64_t id = 0;
    check(bf_serve_submit(server_, &j, &id));
    return id;
}

std::size_t ServedBeamformer::step() {
    uint32_t n = 0;
    check(bf_serve_step(server_, &n));
    return n;
}

ServedJobState ServedBeamformer::state(std::uint64_t job_id) {
    int32_t st = BF_JOB_UNKNOWN;
    check(bf_serve_poll(server_, job_id, &st));
    return static_cast<ServedJobState>(st);
}

std::vector<std::uint64_t> ServedBeamformer::take_done() {
    std::vector<std::uint64_t> ids(256);
    std::vector<std::uint64_t> out;
    while (true) {
        uint64_t n = 0;
        check(bf_serve_take_done(server_, ids.data(), ids.size(), &n));
        out.insert(out.end(), ids.begin(), ids.begin() + static_cast<std::ptrdiff_t>(n));
        if (n < ids.size()) return out;
    }
}

ServedResult ServedBeamformer::result(std::uint64_t job_id) {
    float* integ = nullptr;
    int8_t* codes = nullptr;
    float* params = nullptr;
    uint64_t w = 0;
    check(bf_serve_result(server_, job_id, &integ, &codes, &params, &w));
    return ServedResult{integ, codes, params, static_cast<std::size_t>(w)};
}

void ServedBeamformer::cancel(std::uint64_t job_id) { check(bf_serve_cancel(server_, job_id)); }
void ServedBeamformer::release(std::uint64_t job_id) { check(bf_serve_release(server_, job_id)); }

std::vector<std::uint8_t> ServedBeamformer::checkpoint(std::uint64_t job_id) {
    std::uint64_t n = 0;
    check(bf_serve_checkpoint(server_, job_id, nullptr, 0, &n));
    std::vector<std::uint8_t> image(n);
    check(bf_serve_checkpoint(server_, job_id, image.data(), n, &n));
    image.resize(n);
    return image;
}

std::uint64_t ServedBeamformer::restore(const std::vector<std::uint8_t>& image) {
    std::uint64_t id = 0;
    check(bf_serve_restore(server_, image.data(), image.size(), &id));
    return id;
}
void ServedBeamformer::synchronize() { check(bf_serve_sync(server_)); }

ServedStats ServedBeamformer::stats() {
    bf_serve_stats st{};
    check(bf_serve_stats_get(server_, &st));
    ServedStats out;
    out.steps = st.steps;
    out.job_windows = st.job_windows;
    out.jobs_done = st.jobs_done;
    out.live_jobs = st.live_jobs;
    out.queued_jobs = st.queued_jobs;
    out.arena_bytes_peak = st.arena_bytes_peak;
    out.graph_captures = st.graph_captures;
    out.beam_samples = st.beam_samples;
    out.window_ms_p50 = st.step_ms_p50;
    out.window_ms_p99 = st.step_ms_p99;
    return out;
}

std::vector<float> ServedBeamformer::window_times_ms() {
    uint64_t n = 0;
    check(bf_serve_step_times(server_, nullptr, 0, &n));
    std::vector<float> out(n);
    if (n > 0) check(bf_serve_step_times(server_, out.data(), n, &n));
    return out;
}

void* ServedBeamformer::stream() { return bf_serve_stream(server_); }

ServedBeamformer::Pool ServedBeamformer::pool(std::uint64_t n_ant) {
    Pool p;
    check(bf_serve_pool(server_, n_ant, &p.data, &p.spectra, &p.channels));
    return p;
}

}  // namespace beamformer
