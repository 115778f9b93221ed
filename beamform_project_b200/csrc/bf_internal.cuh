// bf_internal.cuh -- shared helpers for the B200 beamformer library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
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

// Device address of a file-scope __device__ variable on the current device.
// In host code the variable's name is only a host-side stand-in, so its
// device address is looked up with cudaGetSymbolAddress.  The lookup runs
// again on every call made while `stream` is not capturing: a cudaDeviceReset
// (or any teardown of the primary context) reloads the module, possibly at
// another address, and a cached pointer would then send the kernel to freed
// memory.  While `stream` captures, the last address found on this device is
// used (the lookup may load the module, which capture forbids), so the first
// call on a device, and the first after a reset, must come before any
// capture.
struct SymbolAddressCache {
    static constexpr int kMaxDevices = 64;
    std::mutex mu;
    void* addr[kMaxDevices] = {};
};

inline bf_status device_symbol_address(const void* symbol, SymbolAddressCache& cache, cudaStream_t stream,
                                       void** out, const char* what) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
    if (dev < 0 || dev >= SymbolAddressCache::kMaxDevices) {
        return set_error(BF_ERR_UNSUPPORTED, std::string("device ordinal beyond the address table of ") + what);
    }
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(stream, &capture);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamIsCapturing");
    std::lock_guard<std::mutex> lock(cache.mu);
    if (capture == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, symbol);
        if (e != cudaSuccess) return cuda_status(e, (std::string("cudaGetSymbolAddress(") + what + ")").c_str());
        cache.addr[dev] = p;
    } else if (cache.addr[dev] == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         std::string("the first call on a device must come before stream capture (") + what + ")");
    }
    *out = cache.addr[dev];
    return BF_OK;
}

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

// rint((v - offset) / scale) clamped to [-127, 127], with the quotient of the
// reference's correctly rounded float division.  The quotient comes from the
// reciprocal and one fused correction step, which is within one ulp of the
// correctly rounded value, so its nearest integer is the same unless the
// value lies within 2^-14 of a half-integer (|q| <= 127.5 here: one ulp is at
// most 2^-16); only those values take the correctly rounded division.
__device__ __forceinline__ int quantize_code(float v, float offset, float scale, float rcp) {
    const float d = __fsub_rn(v, offset);
    const float q0 = __fmul_rn(d, rcp);
    float q = __fmaf_rn(__fmaf_rn(-q0, scale, d), rcp, q0);
    const float frac = __fsub_rn(q, floorf(q));
    if (fabsf(__fsub_rn(frac, 0.5f)) < 0x1p-14f) q = __fdiv_rn(d, scale);
    return max(-127, min(127, __float2int_rn(q)));
}

// One warp quantizes one 1x16x16 chunk (window w, channels 16*ft.., beams
// 16*bt..) of integrated [W][F][B] exactly as cpu_quantize_integrated_intensity
// (src/quantization.cpp:61-161): min/max over the finite values,
// scale = (max - min) / 255, offset = min - (-127.5 * scale), codes
// clamp(rint((v - offset) / scale), -127, 127), -128 for non-finite values and
// a zero parameter pair for a chunk holding one.  Correctly rounded
// intrinsics keep codes and parameters bit-identical to the CPU reference.
// kCoherent reads through L2 (values written by other CTAs of a running grid).
// A lane holds four consecutive beams of two channels (16-byte loads and
// 4-byte code stores when the beam count is a multiple of four and the
// buffers are aligned for them, scalar accesses otherwise).
template <bool kCoherent>
__device__ __forceinline__ void quantize_chunk(const float* __restrict in, int8_t* __restrict codes,
                                               float2* __restrict params, size_t param_index, int win,
                                               int n_freq, int n_beams, int ft, int bt, int lane) {
    const bool vec = (n_beams & 3) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(codes) & 3) == 0;
    const int b0 = bt * 16 + 4 * (lane & 3);
    float vals[8];
    bool valid[8];
    float mn = INFINITY, mx = -INFINITY;
    bool nonfinite = false;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int f = ft * 16 + (lane >> 2) + 8 * h;
        const size_t row = (static_cast<size_t>(win) * n_freq + f) * n_beams;
        if (vec) {
            const bool ok = f < n_freq && b0 < n_beams;
            float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
            if (ok) {
                const float4* src = reinterpret_cast<const float4*>(in + row + b0);
                x = kCoherent ? __ldcg(src) : *src;
            }
            vals[4 * h] = x.x;
            vals[4 * h + 1] = x.y;
            vals[4 * h + 2] = x.z;
            vals[4 * h + 3] = x.w;
#pragma unroll
            for (int j = 0; j < 4; ++j) valid[4 * h + j] = ok;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool ok = f < n_freq && b0 + j < n_beams;
                valid[4 * h + j] = ok;
                vals[4 * h + j] = 0.f;
                if (ok) vals[4 * h + j] = kCoherent ? __ldcg(in + row + b0 + j) : in[row + b0 + j];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        if (!isfinite(vals[i])) {
            nonfinite = true;
        } else {
            mn = fminf(mn, vals[i]);
            mx = fmaxf(mx, vals[i]);
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
    const float rcp = scale != 0.f ? __frcp_rn(scale) : 0.f;
    int c[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        c[i] = 0;
        if (!isfinite(vals[i])) c[i] = -128;
        else if (scale != 0.f) c[i] = quantize_code(vals[i], offset, scale, rcp);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int f = ft * 16 + (lane >> 2) + 8 * h;
        const size_t row = (static_cast<size_t>(win) * n_freq + f) * n_beams;
        if (vec) {
            if (valid[4 * h]) {
                const uint32_t packed = (static_cast<uint32_t>(c[4 * h]) & 0xFFu) |
                                        ((static_cast<uint32_t>(c[4 * h + 1]) & 0xFFu) << 8) |
                                        ((static_cast<uint32_t>(c[4 * h + 2]) & 0xFFu) << 16) |
                                        ((static_cast<uint32_t>(c[4 * h + 3]) & 0xFFu) << 24);
                *reinterpret_cast<uint32_t*>(codes + row + b0) = packed;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (valid[4 * h + j]) codes[row + b0 + j] = static_cast<int8_t>(c[4 * h + j]);
            }
        }
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
// The DOA fold (doa_scan.cu) of every (block, channel) cell, cell = block *
// n_freq + f, into the head of `workspace` (doa_fold_bytes): S [cells][M][M]
// and Q = (S + E I)^{-1} [cells][M][M] as (re, im) double pairs, E [cells]
// double, ok [cells] int (the loaded Cholesky succeeded).
uint64_t doa_fold_bytes(uint64_t cells, uint64_t M);
bf_status launch_doa_fold(cudaStream_t stream, const int32_t* R, const bf_dims& d, uint64_t block_len, int M,
                          double lam, double load, void* workspace);
// The adaptive tracker (doa_track.cu).
uint64_t doa_track_workspace_bytes(const bf_dims& d, uint64_t block_len, uint64_t subarray);
bf_status launch_doa_track(cudaStream_t stream, const uint8_t* v, const float* pos, const double* kw,
                           const bf_dims& d, const bf_doa_track_config& c, float* dirs, float* intensity,
                           void* workspace);
bf_status launch_doa_scan(cudaStream_t stream, const int32_t* R, const float* pos, const double* kw,
                          const bf_dims& d, uint64_t block_len, uint64_t subarray, double lam, double load,
                          double l_first, double l_step, uint64_t n, double m_fixed, double* bartlett,
                          double* capon, double* l_est, void* workspace);
// argmax and parabolic peak of each block's Bartlett and Capon spectra
bf_status launch_doa_peak(cudaStream_t stream, const double* bartlett, const double* capon, uint64_t n_blocks,
                          uint64_t n_points, double l_first, double l_step, double* l_est);
// nb_pad > 0 pads the beams to nb_pad columns (a multiple of 16 >= n_beams)
// instead of the next multiple of 16.
uint64_t split_weight_bytes(const bf_dims& d, uint64_t n_shards, int nb_pad = 0);
bf_status launch_prepare_split(cudaStream_t stream, const float* w, void* split, const bf_dims& d,
                               uint64_t n_shards, int nb_pad = 0);
bf_status take_tc_error(uint32_t* code);
// Device address of the error word (grid_tc.cu) for kernels in other
// translation units; null when it cannot be found (bf_last_error says why).
unsigned* device_error_word(cudaStream_t stream);
// covariance-form grid (grid_cov.cu)
uint64_t cov_weight_bytes(const bf_dims& d, uint64_t n_shards);
bf_status check_grid_cov(const bf_dims& d, uint64_t spectra, uint64_t n_shards);
bf_status launch_prepare_cov(cudaStream_t stream, const float* w, void* out, const bf_dims& d, uint64_t n_shards);
bf_status launch_grid_cov(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated,
                          int8_t* codes, float* params, const bf_dims& d, uint64_t spectra, uint64_t n_shards);
uint64_t grid_tensor_counter_count(const bf_dims& d, uint64_t spectra, uint64_t n_shards);
// Launch choices of the grid path that leave every value bit-identical (the
// split kernel's unit size and channel order) or within the same bar (the
// checked form's kernel), picked per (n_ant, padded beams, integration) by
// the autotuner (autotune.cu).
struct GridTuning {
    int form = 1;        // bf_grid_auto_integrated: 0 split kernel, 1 checked covariance form
    int group_mult = 1;  // split kernel: units of group_mult x the smallest whole-window unit
    int paired = 1;      // split kernel: CTA pairs walk channel pairs
};
// The tuned choice for a class, or the defaults; true when a tuned entry exists.
bool tuned_grid_config(int n_ant, int nb_pad, uint64_t spectra, GridTuning* out);

// counters == nullptr: quantize (when codes is given) with a second launch;
// otherwise quantization is fused into the tensor kernel's epilogue and
// `counters` (grid_tensor_counter_count entries) is its scratch.  tune ==
// nullptr uses the tuned (or default) choice for the class.
bf_status launch_grid_tensor(cudaStream_t stream, const uint8_t* v, const void* split,
                             float* integrated, int8_t* codes, float* params, const bf_dims& d,
                             uint64_t spectra, uint64_t n_shards, unsigned* counters,
                             const GridTuning* tune = nullptr);
// The split kernel over the units of a device-written list (no quantizer).
bf_status launch_grid_tensor_list(cudaStream_t stream, const uint8_t* v, const void* split, float* integrated,
                                  const bf_dims& d, uint64_t spectra, uint64_t n_shards, const int* unit_list,
                                  const int* unit_count);
// Units of a plain split-kernel launch: (shard, channel, group) with
// groups_per_channel groups of windows_per_group windows (S >= 32).
long long grid_tensor_unit_layout(const bf_dims& d, uint64_t spectra, uint64_t n_shards, int* groups_per_channel,
                                  int* windows_per_group);
// Checked covariance form (grid_cov.cu): the covariance kernel with error
// estimates, then the split kernel over the units whose estimate exceeds the
// calibrated limit.  Weights: the covariance image, then the split image.
uint64_t auto_weight_bytes(const bf_dims& d, uint64_t n_shards);
bool auto_uses_cov(const bf_dims& d, uint64_t spectra, uint64_t n_shards);
uint64_t auto_workspace_bytes(const bf_dims& d, uint64_t spectra, uint64_t n_shards);
bf_status launch_prepare_auto(cudaStream_t stream, const float* w, void* out, const bf_dims& d, uint64_t n_shards);
bf_status launch_grid_auto(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated, int8_t* codes,
                           float* params, void* workspace, const bf_dims& d, uint64_t spectra, uint64_t n_shards,
                           const struct GridTuning* tune = nullptr);
bf_status launch_grid_cov_estimate(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated,
                                   float* estimate, const bf_dims& d, uint64_t spectra, uint64_t n_shards);

}  // namespace bf
