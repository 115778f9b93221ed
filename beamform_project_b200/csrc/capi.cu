// capi.cu -- the extern "C" boundary (include/bf_b200.h).
//
// Validation and error texts follow the reference so a C++ layer can rethrow
// the same exception types with the same messages:
//   validate_dimensions        include/beamformer/config.hpp:81-94
//   integration checks         src/temporal_integration.cpp:10-26
//   tracker checks             src/beam_tracker.cpp:29-54
// Everything here is host code: argument checks, then one kernel launch on
// the caller's stream.  No allocation, no synchronisation, no exceptions.
#include "bf_internal.cuh"
#include "serve.cuh"

#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>

namespace bf {
namespace {
thread_local std::string g_last_error;
}

bf_status set_error(bf_status code, const std::string& message) {
    g_last_error = message;
    return code;
}

bf_status clear_error() {
    g_last_error.clear();
    return BF_OK;
}

bf_status validate_dims(const bf_dims* dims) {
    if (dims == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "dims must not be null");
    if (dims->n_time == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_time must be positive");
    if (dims->n_freq != 336) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         "the local-shard contract requires exactly 336 frequency channels");
    }
    const uint64_t a = dims->n_ant;
    if (a != 32 && a != 64 && a != 128 && a != 256) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "n_ant must be 32, 64, 128, or 256");
    }
    if (dims->n_beams == 0 || dims->n_beams > 128) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "n_beams must be between 1 and 128");
    }
    return BF_OK;
}

}  // namespace bf

using namespace bf;

namespace {

bool aligned(const void* p, uintptr_t bytes) {
    return (reinterpret_cast<uintptr_t>(p) % bytes) == 0;
}

bf_status check_ptr(const void* p, uintptr_t align, const char* name) {
    if (p == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, std::string(name) + " must not be null");
    if (!aligned(p, align)) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         std::string(name) + " must be " + std::to_string(align) + "-byte aligned");
    }
    return BF_OK;
}

#define BF_TRY(expr)                  \
    do {                              \
        const bf_status _s = (expr);  \
        if (_s != BF_OK) return _s;   \
    } while (0)

}  // namespace

extern "C" {

BF_API const char* bf_version(void) { return "beamform_b200 0.1.0 (sm_100a)"; }

BF_API size_t bf_last_error(char* buf, size_t n) {
    const std::string& e = g_last_error;
    if (buf != nullptr && n > 0) {
        const size_t c = e.size() < n - 1 ? e.size() : n - 1;
        std::memcpy(buf, e.data(), c);
        buf[c] = '\0';
    }
    return e.size();
}

BF_API bf_status bf_validate_dimensions(const bf_dims* dims) {
    clear_error();
    return validate_dims(dims);
}

BF_API bf_status bf_device_info(char* name_buf, size_t name_len, int* compute_major,
                                int* compute_minor, uint64_t* global_memory_bytes,
                                int* driver_version, int* runtime_version) {
    clear_error();
    int device = 0;
    BF_TRY(cuda_status(cudaGetDevice(&device), "cudaGetDevice"));
    cudaDeviceProp prop{};
    BF_TRY(cuda_status(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties"));
    if (name_buf != nullptr && name_len > 0) std::snprintf(name_buf, name_len, "%s", prop.name);
    if (compute_major) *compute_major = prop.major;
    if (compute_minor) *compute_minor = prop.minor;
    if (global_memory_bytes) *global_memory_bytes = prop.totalGlobalMem;
    if (driver_version) BF_TRY(cuda_status(cudaDriverGetVersion(driver_version), "cudaDriverGetVersion"));
    if (runtime_version) BF_TRY(cuda_status(cudaRuntimeGetVersion(runtime_version), "cudaRuntimeGetVersion"));
    return BF_OK;
}

BF_API bf_status bf_launch_packed_beamformer(int kernel, void* stream,
                                             const uint8_t* packed_voltage,
                                             const float* weights, float* intensity,
                                             const bf_dims* dims) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (kernel != BF_KERNEL_DIRECT && kernel != BF_KERNEL_TILED) {
        if (kernel == BF_KERNEL_TENSOR) {
            return set_error(BF_ERR_UNSUPPORTED,
                             "the tensor-core kernel produces integrated output only");
        }
        return set_error(BF_ERR_INVALID_ARGUMENT, "unknown CUDA beamformer kernel selector");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(weights, 8, "weights"));
    BF_TRY(check_ptr(intensity, 4, "intensity"));
    return launch_grid_exact(kernel, static_cast<cudaStream_t>(stream), packed_voltage, weights,
                             intensity, *dims, 1, false);
}

BF_API bf_status bf_launch_packed_integrated_beamformer(
    int kernel, void* stream, const uint8_t* packed_voltage, const float* weights,
    float* integrated_intensity, const bf_dims* dims, uint64_t integration_spectra) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    if (kernel != BF_KERNEL_DIRECT && kernel != BF_KERNEL_TILED) {
        if (kernel == BF_KERNEL_TENSOR) {
            return set_error(BF_ERR_UNSUPPORTED,
                             "use bf_grid_tensor_integrated with prepared split weights");
        }
        return set_error(BF_ERR_INVALID_ARGUMENT, "unknown CUDA beamformer kernel selector");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(weights, 8, "weights"));
    BF_TRY(check_ptr(integrated_intensity, 4, "integrated_intensity"));
    return launch_grid_exact(kernel, static_cast<cudaStream_t>(stream), packed_voltage, weights,
                             integrated_intensity, *dims, integration_spectra, true);
}

BF_API bf_status bf_launch_quantize_integrated_intensity(void* stream,
                                                         const float* integrated_intensity,
                                                         int8_t* codes, float* params,
                                                         const bf_dims* integrated_dims) {
    clear_error();
    BF_TRY(validate_dims(integrated_dims));
    BF_TRY(check_ptr(integrated_intensity, 4, "integrated_intensity"));
    BF_TRY(check_ptr(codes, 1, "codes"));
    BF_TRY(check_ptr(params, 8, "params"));
    return launch_quantize(static_cast<cudaStream_t>(stream), integrated_intensity, codes, params,
                           *integrated_dims);
}

BF_API uint64_t bf_split_weight_bytes(const bf_dims* dims, uint64_t n_shards) {
    if (dims == nullptr) return 0;
    return split_weight_bytes(*dims, n_shards);
}

BF_API bf_status bf_prepare_split_weights(void* stream, const float* weights, void* split_weights,
                                          const bf_dims* dims, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    BF_TRY(check_ptr(weights, 8, "weights"));
    BF_TRY(check_ptr(split_weights, 16, "split_weights"));
    return launch_prepare_split(static_cast<cudaStream_t>(stream), weights, split_weights, *dims,
                                n_shards);
}

BF_API bf_status bf_grid_tensor_integrated(void* stream, const uint8_t* packed_voltage,
                                           const void* split_weights, float* integrated,
                                           int8_t* codes, float* params, const bf_dims* dims,
                                           uint64_t integration_spectra, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    if (integration_spectra > 32 && integration_spectra % 32 != 0) {
        return set_error(BF_ERR_UNSUPPORTED,
                         "the tensor-core kernel needs integration_spectra below 32 or a multiple of 32");
    }
    if ((codes == nullptr) != (params == nullptr)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "codes and params must both be given or both be null");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(split_weights, 16, "split_weights"));
    BF_TRY(check_ptr(integrated, 16, "integrated"));
    if (codes != nullptr) BF_TRY(check_ptr(params, 8, "params"));
    return launch_grid_tensor(static_cast<cudaStream_t>(stream), packed_voltage, split_weights,
                              integrated, codes, params, *dims, integration_spectra, n_shards, nullptr);
}

BF_API uint64_t bf_grid_tensor_workspace_bytes(const bf_dims* dims, uint64_t integration_spectra,
                                               uint64_t n_shards) {
    if (dims == nullptr || integration_spectra == 0) return 0;
    return grid_tensor_counter_count(*dims, integration_spectra, n_shards) * sizeof(unsigned);
}

BF_API bf_status bf_grid_tensor_quantized(void* stream, const uint8_t* packed_voltage,
                                          const void* split_weights, float* integrated, int8_t* codes,
                                          float* params, void* workspace, const bf_dims* dims,
                                          uint64_t integration_spectra, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    if (integration_spectra > 32 && integration_spectra % 32 != 0) {
        return set_error(BF_ERR_UNSUPPORTED,
                         "the tensor-core kernel needs integration_spectra below 32 or a multiple of 32");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(split_weights, 16, "split_weights"));
    BF_TRY(check_ptr(integrated, 16, "integrated"));
    BF_TRY(check_ptr(codes, 1, "codes"));
    BF_TRY(check_ptr(params, 8, "params"));
    BF_TRY(check_ptr(workspace, 4, "workspace"));
    return launch_grid_tensor(static_cast<cudaStream_t>(stream), packed_voltage, split_weights,
                              integrated, codes, params, *dims, integration_spectra, n_shards,
                              static_cast<unsigned*>(workspace));
}

BF_API uint64_t bf_cov_weight_bytes(const bf_dims* dims, uint64_t n_shards) {
    if (dims == nullptr) return 0;
    return cov_weight_bytes(*dims, n_shards);
}

BF_API bf_status bf_prepare_cov_weights(void* stream, const float* weights, void* cov_weights,
                                        const bf_dims* dims, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (dims->n_ant != 64) return set_error(BF_ERR_UNSUPPORTED, "the covariance-form grid supports n_ant 64");
    BF_TRY(check_ptr(weights, 8, "weights"));
    BF_TRY(check_ptr(cov_weights, 16, "cov_weights"));
    return launch_prepare_cov(static_cast<cudaStream_t>(stream), weights, cov_weights, *dims, n_shards);
}

BF_API bf_status bf_grid_cov_integrated(void* stream, const uint8_t* packed_voltage, const void* cov_weights,
                                        float* integrated, int8_t* codes, float* params, const bf_dims* dims,
                                        uint64_t integration_spectra, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    BF_TRY(check_grid_cov(*dims, integration_spectra, n_shards));
    if ((codes == nullptr) != (params == nullptr)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "codes and params must both be given or both be null");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(cov_weights, 16, "cov_weights"));
    BF_TRY(check_ptr(integrated, 16, "integrated"));
    if (codes != nullptr) BF_TRY(check_ptr(params, 8, "params"));
    return launch_grid_cov(static_cast<cudaStream_t>(stream), packed_voltage, cov_weights, integrated, codes,
                           params, *dims, integration_spectra, n_shards);
}

BF_API bf_status bf_grid_cov_estimate(void* stream, const uint8_t* packed_voltage, const void* cov_weights,
                                      float* integrated, float* estimate, const bf_dims* dims,
                                      uint64_t integration_spectra, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    BF_TRY(check_grid_cov(*dims, integration_spectra, n_shards));
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(cov_weights, 16, "cov_weights"));
    BF_TRY(check_ptr(integrated, 16, "integrated"));
    BF_TRY(check_ptr(estimate, 4, "estimate"));
    return launch_grid_cov_estimate(static_cast<cudaStream_t>(stream), packed_voltage, cov_weights, integrated,
                                    estimate, *dims, integration_spectra, n_shards);
}

BF_API uint64_t bf_auto_weight_bytes(const bf_dims* dims, uint64_t n_shards) {
    if (dims == nullptr || validate_dims(dims) != BF_OK) return 0;
    return auto_weight_bytes(*dims, n_shards);
}

BF_API bf_status bf_prepare_auto_weights(void* stream, const float* weights, void* auto_weights,
                                         const bf_dims* dims, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    BF_TRY(check_ptr(weights, 8, "weights"));
    BF_TRY(check_ptr(auto_weights, 16, "auto_weights"));
    return launch_prepare_auto(static_cast<cudaStream_t>(stream), weights, auto_weights, *dims, n_shards);
}

BF_API uint64_t bf_grid_auto_workspace_bytes(const bf_dims* dims, uint64_t integration_spectra, uint64_t n_shards) {
    if (dims == nullptr || validate_dims(dims) != BF_OK || integration_spectra == 0 || n_shards == 0) return 0;
    return auto_workspace_bytes(*dims, integration_spectra, n_shards);
}

BF_API bf_status bf_grid_auto_integrated(void* stream, const uint8_t* packed_voltage, const void* auto_weights,
                                         float* integrated, int8_t* codes, float* params, void* workspace,
                                         const bf_dims* dims, uint64_t integration_spectra, uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    if (integration_spectra > 32 && integration_spectra % 32 != 0) {
        return set_error(BF_ERR_UNSUPPORTED,
                         "the tensor-core kernels need integration_spectra below 32 or a multiple of 32");
    }
    if ((codes == nullptr) != (params == nullptr)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "codes and params must both be given or both be null");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(auto_weights, 16, "auto_weights"));
    BF_TRY(check_ptr(integrated, 16, "integrated"));
    if (codes != nullptr) BF_TRY(check_ptr(params, 8, "params"));
    if (auto_uses_cov(*dims, integration_spectra, n_shards)) BF_TRY(check_ptr(workspace, 256, "workspace"));
    return launch_grid_auto(static_cast<cudaStream_t>(stream), packed_voltage, auto_weights, integrated, codes, params,
                            workspace, *dims, integration_spectra, n_shards);
}

BF_API bf_status bf_tracker(void* stream, int mode, const uint8_t* packed_voltage,
                            const float* positions, const double* wave_numbers,
                            const float* window_directions, float* intensity,
                            float* integrated, const bf_dims* dims,
                            uint64_t integration_spectra) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (dims->n_beams != 1) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         "tracker requires exactly n_beams == 1 (use tracker_beam_count)");
    }
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "tracker integration_spectra must be positive");
    }
    if (mode != 0 && mode != 1) return set_error(BF_ERR_INVALID_ARGUMENT, "unknown tracker mode");
    if (intensity == nullptr && integrated == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "intensity and integrated are both null");
    }
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(positions, 4, "positions"));
    BF_TRY(check_ptr(wave_numbers, 8, "wave_numbers"));
    BF_TRY(check_ptr(window_directions, 4, "window_directions"));
    if (intensity != nullptr) BF_TRY(check_ptr(intensity, 4, "intensity"));
    if (integrated != nullptr) BF_TRY(check_ptr(integrated, 4, "integrated"));
    return launch_tracker(static_cast<cudaStream_t>(stream), mode, packed_voltage, positions,
                          wave_numbers, window_directions, intensity, integrated, *dims,
                          integration_spectra);
}

// The DOA entries take the reference's 336-channel shard; the _slice entries
// take a contiguous slice of it (an even count of 2 to 336 channels), the
// share of one GPU when the channels of a job are split across GPUs.
static bf_status validate_doa_dims(const bf_dims* dims, bool slice) {
    if (!slice) {
        BF_TRY(validate_dims(dims));
    } else {
        if (dims == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "dims must not be null");
        if (dims->n_time == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_time must be positive");
        if (dims->n_freq < 2 || dims->n_freq > 336 || dims->n_freq % 2 != 0) {
            return set_error(BF_ERR_INVALID_ARGUMENT, "a channel slice holds an even count of 2 to 336 channels");
        }
        const uint64_t a = dims->n_ant;
        if (a != 32 && a != 64 && a != 128 && a != 256) {
            return set_error(BF_ERR_INVALID_ARGUMENT, "n_ant must be 32, 64, 128, or 256");
        }
    }
    if (dims->n_beams != 1) return set_error(BF_ERR_INVALID_ARGUMENT, "the DOA path takes n_beams == 1");
    return BF_OK;
}

static bf_status doa_covariance_impl(void* stream, const uint8_t* packed_voltage, int32_t* covariance,
                                     const bf_dims* dims, uint64_t block_len, bool slice) {
    clear_error();
    BF_TRY(validate_doa_dims(dims, slice));
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(covariance, 8, "covariance"));
    return launch_doa_covariance(static_cast<cudaStream_t>(stream), packed_voltage, covariance, *dims,
                                 block_len);
}

BF_API bf_status bf_doa_covariance_i32(void* stream, const uint8_t* packed_voltage,
                                       int32_t* covariance, const bf_dims* dims, uint64_t block_len) {
    return doa_covariance_impl(stream, packed_voltage, covariance, dims, block_len, false);
}

BF_API bf_status bf_doa_covariance_i32_slice(void* stream, const uint8_t* packed_voltage,
                                             int32_t* covariance, const bf_dims* dims, uint64_t block_len) {
    return doa_covariance_impl(stream, packed_voltage, covariance, dims, block_len, true);
}

BF_API uint64_t bf_doa_workspace_bytes(const bf_dims* dims, uint64_t block_len, uint64_t subarray) {
    if (dims == nullptr || block_len == 0) return 0;
    const uint64_t M = (subarray > 0 && subarray < dims->n_ant) ? subarray : dims->n_ant;
    return doa_workspace_bytes(dims->n_time / block_len, dims->n_freq, M);
}

static bf_status doa_scan_impl(void* stream, const int32_t* covariance, const float* positions,
                               const double* wave_numbers, const bf_dims* dims, uint64_t block_len,
                               uint64_t subarray, double forgetting, double diag_load, double l_first,
                               double l_step, uint64_t n_points, double m_fixed, double* bartlett,
                               double* capon, double* l_est, void* workspace, bool slice) {
    clear_error();
    BF_TRY(validate_doa_dims(dims, slice));
    if (block_len == 0 || dims->n_time % block_len != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "block_len must divide n_time");
    }
    if (!(forgetting > 0.0 && forgetting <= 1.0)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "forgetting factor must be in (0, 1]");
    }
    if (!(diag_load >= 0.0) || n_points == 0 || n_points > (1u << 24)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "diag_load must be >= 0 and n_points in [1, 2^24]");
    }
    BF_TRY(check_ptr(covariance, 8, "covariance"));
    BF_TRY(check_ptr(positions, 4, "positions"));
    BF_TRY(check_ptr(wave_numbers, 8, "wave_numbers"));
    BF_TRY(check_ptr(bartlett, 8, "bartlett"));
    BF_TRY(check_ptr(capon, 8, "capon"));
    BF_TRY(check_ptr(l_est, 8, "l_est"));
    BF_TRY(check_ptr(workspace, 16, "workspace"));
    return launch_doa_scan(static_cast<cudaStream_t>(stream), covariance, positions, wave_numbers, *dims,
                           block_len, subarray, forgetting, diag_load, l_first, l_step, n_points, m_fixed,
                           bartlett, capon, l_est, workspace);
}

BF_API bf_status bf_doa_scan(void* stream, const int32_t* covariance, const float* positions,
                             const double* wave_numbers, const bf_dims* dims, uint64_t block_len,
                             uint64_t subarray, double forgetting, double diag_load, double l_first,
                             double l_step, uint64_t n_points, double m_fixed, double* bartlett,
                             double* capon, double* l_est, void* workspace) {
    return doa_scan_impl(stream, covariance, positions, wave_numbers, dims, block_len, subarray, forgetting,
                         diag_load, l_first, l_step, n_points, m_fixed, bartlett, capon, l_est, workspace, false);
}

BF_API bf_status bf_doa_scan_slice(void* stream, const int32_t* covariance, const float* positions,
                                   const double* wave_numbers, const bf_dims* dims, uint64_t block_len,
                                   uint64_t subarray, double forgetting, double diag_load, double l_first,
                                   double l_step, uint64_t n_points, double m_fixed, double* bartlett,
                                   double* capon, double* l_est, void* workspace) {
    return doa_scan_impl(stream, covariance, positions, wave_numbers, dims, block_len, subarray, forgetting,
                         diag_load, l_first, l_step, n_points, m_fixed, bartlett, capon, l_est, workspace, true);
}

BF_API bf_status bf_doa_peak(void* stream, const double* bartlett, const double* capon, uint64_t n_blocks,
                             uint64_t n_points, double l_first, double l_step, double* l_est) {
    clear_error();
    if (n_blocks == 0 || n_blocks > 65535 || n_points == 0 || n_points > (1u << 24)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "n_blocks must be in [1, 65535] and n_points in [1, 2^24]");
    }
    BF_TRY(check_ptr(bartlett, 8, "bartlett"));
    BF_TRY(check_ptr(capon, 8, "capon"));
    BF_TRY(check_ptr(l_est, 8, "l_est"));
    return launch_doa_peak(static_cast<cudaStream_t>(stream), bartlett, capon, n_blocks, n_points, l_first, l_step,
                           l_est);
}

static bf_status check_track(const bf_dims* dims, const bf_doa_track_config* c) {
    BF_TRY(validate_dims(dims));
    if (c == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "config must not be null");
    if (dims->n_beams != 1) return set_error(BF_ERR_INVALID_ARGUMENT, "the DOA path takes n_beams == 1");
    if (dims->n_ant > 64) return set_error(BF_ERR_UNSUPPORTED, "the DOA covariance supports n_ant 32 or 64");
    if (c->block_len == 0 || c->block_len % 128 != 0 || dims->n_time % c->block_len != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "block_len must be a multiple of 128 dividing n_time");
    }
    const uint64_t M = (c->subarray > 0 && c->subarray < dims->n_ant) ? c->subarray : dims->n_ant;
    if (M > 16) return set_error(BF_ERR_UNSUPPORTED, "the DOA search supports at most 16 elements after smoothing");
    if (c->estimator > 1) return set_error(BF_ERR_INVALID_ARGUMENT, "estimator must be 0 (Bartlett) or 1 (Capon)");
    if (c->grid < 2 || c->grid > 64 || c->levels > 16) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "grid must be 2 to 64 and levels at most 16");
    }
    if (!(c->fov_l >= 0.f) || !(c->fov_m >= 0.f) || !(c->forgetting > 0.f && c->forgetting <= 1.f) ||
        !(c->diag_load >= 0.f) || !std::isfinite(c->prior_l) || !std::isfinite(c->prior_m) ||
        c->prior_l * c->prior_l + c->prior_m * c->prior_m > 1.f) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "invalid field of view, forgetting, loading or prior");
    }
    if (dims->n_time / c->block_len > 65535) return set_error(BF_ERR_OVERFLOW, "at most 65535 windows");
    return BF_OK;
}

BF_API uint64_t bf_doa_track_workspace_bytes(const bf_dims* dims, const bf_doa_track_config* config) {
    if (check_track(dims, config) != BF_OK) return 0;
    return doa_track_workspace_bytes(*dims, config->block_len, config->subarray);
}

BF_API bf_status bf_doa_track(void* stream, const uint8_t* packed_voltage, const float* positions,
                              const double* wave_numbers, const bf_dims* dims, const bf_doa_track_config* config,
                              float* window_directions, float* intensity, void* workspace) {
    clear_error();
    BF_TRY(check_track(dims, config));
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    BF_TRY(check_ptr(positions, 4, "positions"));
    BF_TRY(check_ptr(wave_numbers, 8, "wave_numbers"));
    BF_TRY(check_ptr(window_directions, 4, "window_directions"));
    if (intensity != nullptr) BF_TRY(check_ptr(intensity, 4, "intensity"));
    BF_TRY(check_ptr(workspace, 256, "workspace"));
    return launch_doa_track(static_cast<cudaStream_t>(stream), packed_voltage, positions, wave_numbers, *dims,
                            *config, window_directions, intensity, workspace);
}

BF_API bf_status bf_take_device_error(uint32_t* code) {
    clear_error();
    return take_tc_error(code);
}

BF_API bf_status bf_generate_voltage(void* stream, uint64_t seed, uint64_t sample_offset,
                                     float scale, const float* mu, uint64_t epoch_len,
                                     uint8_t* out, const bf_dims* dims) {
    clear_error();
    if (dims == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "dims must not be null");
    if (out == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "out must not be null");
    if (mu != nullptr && epoch_len == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "epoch_len must be positive when mu is given");
    }
    if (mu != nullptr) BF_TRY(check_ptr(mu, 8, "mu"));
    return launch_generate(static_cast<cudaStream_t>(stream), seed, sample_offset, scale, mu,
                           epoch_len, out, *dims);
}

BF_API bf_status bf_apply_loss_mask(void* stream, uint8_t* packed_voltage, const uint8_t* loss_mask,
                                    const bf_dims* dims, uint64_t integration_spectra, uint32_t* valid_counts) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (integration_spectra == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    if (loss_mask == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "loss_mask must not be null");
    BF_TRY(check_ptr(packed_voltage, 16, "packed_voltage"));
    if (valid_counts != nullptr) BF_TRY(check_ptr(valid_counts, 4, "valid_counts"));
    return launch_apply_loss_mask(static_cast<cudaStream_t>(stream), packed_voltage, loss_mask, dims->n_time,
                                  dims->n_freq, dims->n_ant, integration_spectra, valid_counts);
}

BF_API bf_status bf_generate_weights(void* stream, const float* positions, const float* frequencies,
                                     const float* directions, float* weights, const bf_dims* dims,
                                     uint64_t n_shards) {
    clear_error();
    BF_TRY(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (positions == nullptr || frequencies == nullptr || directions == nullptr || weights == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "positions, frequencies, directions and weights must not be null");
    }
    BF_TRY(check_ptr(weights, 8, "weights"));
    return launch_generate_weights(static_cast<cudaStream_t>(stream), positions, frequencies, directions, weights,
                                   n_shards, dims->n_freq, dims->n_beams, dims->n_ant);
}

}  // extern "C"
