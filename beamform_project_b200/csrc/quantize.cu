// quantize.cu -- int8 chunk quantizer (drop-in for
// launch_quantize_integrated_intensity, reference include/beamformer/
// cuda_stage_api.hpp:37-42).
//
// Semantics follow cpu_quantize_integrated_intensity (src/quantization.cpp:
// 61-161) operation for operation, with correctly rounded intrinsics so the
// codes and the (offset, scale) pairs are bit-identical to the CPU reference:
//   scale  = (max - min) / 255        (255 = 127.5 - (-127.5))
//   offset = min - (-127.5 * scale)
//   code   = clamp(rint((v - offset) / scale), -127, 127)   (half to even)
//   non-finite value -> -128; a chunk holding one gets (0, 0); scale 0 -> 0.
// One warp per 1x16x16 chunk, 8 values per lane, shuffle min/max.
#include "bf_internal.cuh"

namespace bf {
namespace {

constexpr int kChunkWarps = 8;

__global__ void __launch_bounds__(kChunkWarps * 32)
quantize_kernel(const float* __restrict__ in, int8_t* __restrict__ codes,
                float2* __restrict__ params, int n_win, int n_freq, int n_beams, int ftiles,
                int btiles, long long n_chunks) {
    const long long chunk = static_cast<long long>(blockIdx.x) * kChunkWarps + (threadIdx.x >> 5);
    if (chunk >= n_chunks) return;
    const int lane = threadIdx.x & 31;
    const int bt = static_cast<int>(chunk % btiles);
    const long long rest = chunk / btiles;
    const int ft = static_cast<int>(rest % ftiles);
    const int win = static_cast<int>(rest / ftiles);

    float vals[8];
    bool valid[8];
    float mn = INFINITY, mx = -INFINITY;
    bool nonfinite = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int s = lane + 32 * i;  // 0..255 = local_freq * 16 + local_beam
        const int f = ft * 16 + (s >> 4), b = bt * 16 + (s & 15);
        valid[i] = f < n_freq && b < n_beams;
        vals[i] = 0.f;
        if (valid[i]) {
            vals[i] = in[(static_cast<size_t>(win) * n_freq + f) * n_beams + b];
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
    if (lane == 0) params[chunk] = make_float2(offset, scale);
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

}  // namespace

bf_status launch_quantize(cudaStream_t stream, const float* in, int8_t* codes, float* params,
                          const bf_dims& d) {
    const uint64_t ftiles = (d.n_freq + 15) / 16, btiles = (d.n_beams + 15) / 16;
    const uint64_t n_chunks = d.n_time * ftiles * btiles;
    const uint64_t blocks = (n_chunks + kChunkWarps - 1) / kChunkWarps;
    if (blocks > 0x7fffffffull || d.n_time > 0x7fffffffull) {
        return set_error(BF_ERR_OVERFLOW, "CUDA quantization grid exceeds the supported size");
    }
    if (blocks == 0) return BF_OK;
    quantize_kernel<<<static_cast<unsigned>(blocks), kChunkWarps * 32, 0, stream>>>(
        in, codes, reinterpret_cast<float2*>(params), static_cast<int>(d.n_time),
        static_cast<int>(d.n_freq), static_cast<int>(d.n_beams), static_cast<int>(ftiles),
        static_cast<int>(btiles), static_cast<long long>(n_chunks));
    return cuda_status(cudaGetLastError(), "quantize_kernel launch");
}

}  // namespace bf
