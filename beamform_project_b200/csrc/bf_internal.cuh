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

#define BF_RETURN_IF(expr)              \
    do {                                \
        const bf_status bf_s_ = (expr); \
        if (bf_s_ != BF_OK) return bf_s_; \
    } while (0)

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

// One warp quantizes one 1x16x16 chunk (window w, channels 16*ft.., beams
// 16*bt..) of integrated [W][F][B] exactly as cpu_quantize_integrated_intensity
// (src/quantization.cpp:61-161): min/max over the finite values,
// scale = (max - min) / 255, offset = min - (-127.5 * scale), codes
// clamp(rint((v - offset) / scale), -127, 127), -128 for non-finite values and
// a zero parameter pair for a chunk holding one.  Correctly rounded
// intrinsics keep codes and parameters bit-identical to the CPU reference.
// kCoherent reads through L2 (values written by other CTAs of a running grid).
template <bool kCoherent>
__device__ __forceinline__ void quantize_chunk(const float* __restrict in, int8_t* __restrict codes,
                                               float2* __restrict params, size_t param_index, int win,
                                               int n_freq, int n_beams, int ft, int bt, int lane) {
    float vals[8];
    bool valid[8];
    float mn = INFINITY, mx = -INFINITY;
    bool nonfinite = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int s = lane + 32 * i;  // local_freq * 16 + local_beam
        const int f = ft * 16 + (s >> 4), b = bt * 16 + (s & 15);
        valid[i] = f < n_freq && b < n_beams;
        vals[i] = 0.f;
        if (valid[i]) {
            const float* src = in + (static_cast<size_t>(win) * n_freq + f) * n_beams + b;
            vals[i] = kCoherent ? __ldcg(src) : *src;
            if (!isfinite(vals[i])) {
                nonfinite = true;
            } else {
                mn = fminf(mn, vals[i]);
                mx = fmaxf(mx, vals[i]);
            }
        }
    }
    nonfinite = __any_sync(0xffffffffu, nonfinite);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    float offset = 0.f, scale = 0.f;
    if (!nonfinite && isfinite(mn) && isfinite(mx)) {
        scale = __fdiv_rn(__fsub_rn(mx, mn), 255.0f);
        offset = __fsub_rn(mn, __fmul_rn(-127.5f, scale));
        if (!isfinite(offset) || !isfinite(scale)) offset = scale = 0.f;
    }
    if (lane == 0) params[param_index] = make_float2(offset, scale);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        const int s = lane + 32 * i;
        const int f = ft * 16 + (s >> 4), b = bt * 16 + (s & 15);
        int code = 0;
        if (!isfinite(vals[i])) {
            code = -128;
        } else if (scale != 0.f) {
            code = __float2int_rn(__fdiv_rn(__fsub_rn(vals[i], offset), scale));
            code = max(-127, min(127, code));
        }
        codes[(static_cast<size_t>(win) * n_freq + f) * n_beams + b] = static_cast<int8_t>(code);
    }
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
bf_status launch_doa_covariance(cudaStream_t stream, const uint8_t* v, int32_t* out, const bf_dims& d,
                                uint64_t block_len);
bf_status launch_apply_loss_mask(cudaStream_t stream, uint8_t* v, const uint8_t* mask, uint64_t n_time,
                                 uint64_t n_freq, uint64_t n_ant, uint64_t spectra, uint32_t* counts);
uint64_t doa_workspace_bytes(uint64_t n_blocks, uint64_t n_freq, uint64_t M);
bf_status launch_doa_scan(cudaStream_t stream, const int32_t* R, const float* pos, const double* kw,
                          const bf_dims& d, uint64_t block_len, uint64_t subarray, double lam, double load,
                          double l_first, double l_step, uint64_t n, double m_fixed, double* bartlett,
                          double* capon, double* l_est, void* workspace);
// nb_pad > 0 pads the beams to nb_pad columns (a multiple of 16 >= n_beams)
// instead of the next multiple of 16.
uint64_t split_weight_bytes(const bf_dims& d, uint64_t n_shards, int nb_pad = 0);
bf_status launch_prepare_split(cudaStream_t stream, const float* w, void* split, const bf_dims& d,
                               uint64_t n_shards, int nb_pad = 0);
bf_status take_tc_error(uint32_t* code);
unsigned* device_error_word();
uint64_t grid_tensor_counter_count(const bf_dims& d, uint64_t spectra, uint64_t n_shards);
// counters == nullptr: quantize (when codes is given) with a second launch;
// otherwise quantization is fused into the tensor kernel's epilogue and
// `counters` (grid_tensor_counter_count entries) is its scratch.
bf_status launch_grid_tensor(cudaStream_t stream, const uint8_t* v, const void* split,
                             float* integrated, int8_t* codes, float* params, const bf_dims& d,
                             uint64_t spectra, uint64_t n_shards, unsigned* counters);

}  // namespace bf
