// grid_exact.cu -- fixed-grid beamformer in the reference's float32 order.
//
// This is the plain drop-in for launch_packed_beamformer and
// launch_packed_integrated_beamformer (reference include/beamformer/
// cuda_stage_api.hpp:21-35, kernels src/cuda_beamformer.cu:108-354).  Each
// output is the same sequence of correctly rounded float32 operations as
// cpu_beamform_packed_intensity (src/cpu_beamformer.cpp:56-78) followed by
// cpu_integrate_intensity (src/temporal_integration.cpp:95-109), so results
// are bit-identical to the reference CPU core built without FMA contraction.
//
// Work decomposition (not the reference's): one warp owns one
// (channel, 32-beam tile, time unit) where a time unit is one integration
// window (integrated output) or 32 spectra (per-spectrum output).  Lanes are
// beams.  The CTA's four warps share the tile's weights in shared memory
// ([A][32] float2, conflict-free across lanes); each warp decodes its
// voltage rows once into a private float2 staging area that all 32 lanes
// then read as a broadcast.  Four spectra are accumulated in flight per lane
// (independent chains, each in antenna order) and their powers are added to
// the window sum strictly in increasing time.
#include "bf_internal.cuh"

namespace bf {
namespace {

constexpr int kWarps = 4;
constexpr int kRows = 8;          // spectra staged per warp per step
constexpr int kUnitSpectra = 32;  // time unit of the per-spectrum output

template <bool kTiled, bool kIntegrate>
__global__ void __launch_bounds__(kWarps * 32)
grid_exact_kernel(const uint8_t* __restrict__ v, const float2* __restrict__ w,
                  float* __restrict__ out, int n_time, int n_freq, int n_ant, int n_beams,
                  int unit_len, int n_units) {
    extern __shared__ float2 smem[];
    float2* ws = smem;                                  // [A][32]
    float2* xs = smem + n_ant * 32 + (threadIdx.x >> 5) * kRows * n_ant;  // [kRows][A]

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int tile = blockIdx.x;
    const int f = blockIdx.y;
    const int beam_tiles = (n_beams + 31) / 32;

    for (int i = threadIdx.x; i < n_ant * 32; i += blockDim.x) {
        const int a = i >> 5, lb = i & 31, b = tile * 32 + lb;
        float2 val = make_float2(0.f, 0.f);
        if (b < n_beams) {
            val = kTiled ? w[((static_cast<size_t>(f) * beam_tiles + tile) * n_ant + a) * 32 + lb]
                         : w[(static_cast<size_t>(b) * n_freq + f) * n_ant + a];
        }
        ws[i] = val;
    }
    __syncthreads();

    const int unit = blockIdx.z * kWarps + warp;
    if (unit >= n_units) return;
    const int b = tile * 32 + lane;
    const int t_begin = unit * unit_len;
    const int t_end = min(t_begin + unit_len, n_time);
    const int chunks_per_row = n_ant / 16;  // 16-byte loads per voltage row
    float acc = 0.f;

    for (int tc = t_begin; tc < t_end; tc += kRows) {
        const int rows = min(kRows, t_end - tc);
        for (int c = lane; c < rows * chunks_per_row; c += 32) {
            const int r = c / chunks_per_row, q = c % chunks_per_row;
            const uint4 raw = __ldg(reinterpret_cast<const uint4*>(
                v + (static_cast<size_t>(tc + r) * n_freq + f) * n_ant + q * 16));
            const uint32_t words[4] = {raw.x, raw.y, raw.z, raw.w};
            float2* dst = xs + r * n_ant + q * 16;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const uint32_t byte = (words[j >> 2] >> (8 * (j & 3))) & 0xFFu;
                dst[j] = make_float2(static_cast<float>(nibble_lo(byte)),
                                     static_cast<float>(nibble_hi(byte)));
            }
        }
        __syncwarp();
        for (int r0 = 0; r0 < rows; r0 += 4) {
            float sr[4] = {0.f, 0.f, 0.f, 0.f}, si[4] = {0.f, 0.f, 0.f, 0.f};
            for (int a = 0; a < n_ant; ++a) {
                const float2 wv = ws[a * 32 + lane];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float2 x = xs[(r0 + u) * n_ant + a];
                    cmac_ref(sr[u], si[u], wv.x, wv.y, x.x, x.y);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (r0 + u < rows) {
                    const float p = power_ref(sr[u], si[u]);
                    if (kIntegrate) {
                        acc = __fadd_rn(acc, p);
                    } else if (b < n_beams) {
                        out[(static_cast<size_t>(tc + r0 + u) * n_freq + f) * n_beams + b] = p;
                    }
                }
            }
        }
        __syncwarp();
    }
    if (kIntegrate && b < n_beams) {
        out[(static_cast<size_t>(unit) * n_freq + f) * n_beams + b] = acc;
    }
}

template <bool kTiled, bool kIntegrate>
bf_status launch_variant(cudaStream_t stream, const uint8_t* v, const float* w, float* out,
                         const bf_dims& d, int unit_len, int n_units) {
    const int A = static_cast<int>(d.n_ant);
    const size_t smem = static_cast<size_t>(A) * 32 * sizeof(float2)
                        + static_cast<size_t>(kWarps) * kRows * A * sizeof(float2);
    auto kern = grid_exact_kernel<kTiled, kIntegrate>;
    cudaError_t err =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return cuda_status(err, "grid_exact_kernel smem attribute");
    const dim3 grid(static_cast<unsigned>((d.n_beams + 31) / 32),
                    static_cast<unsigned>(d.n_freq),
                    static_cast<unsigned>((n_units + kWarps - 1) / kWarps));
    kern<<<grid, kWarps * 32, smem, stream>>>(v, reinterpret_cast<const float2*>(w), out,
                                              static_cast<int>(d.n_time),
                                              static_cast<int>(d.n_freq), A,
                                              static_cast<int>(d.n_beams), unit_len, n_units);
    return cuda_status(cudaGetLastError(), "grid_exact_kernel launch");
}

}  // namespace

bf_status launch_grid_exact(int kernel, cudaStream_t stream, const uint8_t* v, const float* w,
                            float* out, const bf_dims& d, uint64_t spectra, bool integrate) {
    const uint64_t unit_len = integrate ? spectra : kUnitSpectra;
    const uint64_t n_units = window_count(d.n_time, unit_len);
    if (n_units > (1ull << 31) / kWarps || d.n_time > (1ull << 31)) {
        return set_error(BF_ERR_OVERFLOW, "CUDA grid exceeds the supported size");
    }
    const bool tiled = kernel == BF_KERNEL_TILED;
    const int ul = static_cast<int>(unit_len), nu = static_cast<int>(n_units);
    if (tiled) {
        return integrate ? launch_variant<true, true>(stream, v, w, out, d, ul, nu)
                         : launch_variant<true, false>(stream, v, w, out, d, ul, nu);
    }
    return integrate ? launch_variant<false, true>(stream, v, w, out, d, ul, nu)
                     : launch_variant<false, false>(stream, v, w, out, d, ul, nu);
}

}  // namespace bf
