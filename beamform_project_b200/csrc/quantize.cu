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
    quantize_chunk<false>(in, codes, params, static_cast<size_t>(chunk), win, n_freq, n_beams, ft, bt, lane);
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
