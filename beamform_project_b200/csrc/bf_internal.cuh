// bf_internal.cuh -- shared helpers for the B200 beamformer library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/bf_b200.h"

namespace bf {

// Per-thread error text behind bf_last_error().
bf_status set_error(bf_status code, const std::string& message);
bf_status clear_error();

inline bf_status cuda_status(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return BF_OK;
    return set_error(BF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

// validate_dimensions (include/beamformer/config.hpp:81-94).
bf_status validate_dims(const bf_dims* dims);

inline uint64_t window_count(uint64_t n_time, uint64_t spectra) {
    return n_time / spectra + (n_time % spectra == 0 ? 0 : 1);
}

// Signed nibble decode of include/beamformer/int4.hpp:19-30 (two's complement).
__device__ __forceinline__ int nibble_lo(uint32_t byte) {
    return static_cast<int>(byte << 28) >> 28;
}
__device__ __forceinline__ int nibble_hi(uint32_t byte) {
    return static_cast<int>(byte << 24) >> 28;
}

// One complex multiply-accumulate in the reference's float32 order
// (src/cpu_beamformer.cpp:71-72), written with round-to-nearest intrinsics so
// the compiler cannot contract it into FMA:
//   sr += wr*xr - wi*xi ;  si += wr*xi + wi*xr
__device__ __forceinline__ void cmac_ref(float& sr, float& si, float wr, float wi, float xr,
                                         float xi) {
    sr = __fadd_rn(sr, __fsub_rn(__fmul_rn(wr, xr), __fmul_rn(wi, xi)));
    si = __fadd_rn(si, __fadd_rn(__fmul_rn(wr, xi), __fmul_rn(wi, xr)));
}

__device__ __forceinline__ float power_ref(float sr, float si) {
    return __fadd_rn(__fmul_rn(sr, sr), __fmul_rn(si, si));
}

// Kernel launchers (each returns a status, never throws).
bf_status launch_grid_exact(int kernel, cudaStream_t stream, const uint8_t* v, const float* w,
                            float* out, const bf_dims& d, uint64_t spectra, bool integrate);
bf_status launch_quantize(cudaStream_t stream, const float* in, int8_t* codes, float* params,
                          const bf_dims& d);
bf_status launch_generate(cudaStream_t stream, uint64_t seed, uint64_t offset, float scale,
                          const float* mu, uint64_t epoch_len, uint8_t* out, const bf_dims& d);
bf_status launch_tracker(cudaStream_t stream, int mode, const uint8_t* v, const float* pos,
                         const double* k, const float* dirs, float* intensity, float* integrated,
                         const bf_dims& d, uint64_t spectra);
uint64_t split_weight_bytes(const bf_dims& d, uint64_t n_shards);
bf_status launch_prepare_split(cudaStream_t stream, const float* w, void* split, const bf_dims& d,
                               uint64_t n_shards);
bf_status take_tc_error(uint32_t* code);
bf_status launch_grid_tensor(cudaStream_t stream, const uint8_t* v, const void* split,
                             float* integrated, int8_t* codes, float* params, const bf_dims& d,
                             uint64_t spectra, uint64_t n_shards);

}  // namespace bf
