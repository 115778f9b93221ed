// tracker_stream.cu -- HBM streaming tracker kernel (bf_tracker mode 1).
//
// Same product as the reference trackers (src/beam_tracker.cpp:90-146 on the
// CPU, src/cuda_beam_tracker_v5.cu:137-273 on the GPU): one steering weight
// set per integration window, per-spectrum power |sum_a w_a x_a|^2 for a
// single beam, plus (new) the per-window sum.
//
// The kernel reads every voltage byte exactly once with 128-bit loads and is
// meant to run at HBM speed.  At 64 antennas a scalar complex MAC costs about
// 12 ALU instructions per input byte, which would make the kernel ALU-bound,
// so the MAC runs on the tensor pipe instead with the voltage fed straight
// from registers:
//   * Packed bytes are turned into fp16 pairs with two LOP3s (the nibble is
//     placed in the mantissa of 1024.0 with its sign bit flipped) and one
//     half2 subtract / fma -- int4 values are exact in fp16.
//   * The weights are generated in registers once per window: FP64 delay
//     and phase, reduced mod 2*pi in FP64, then float sin/cos, and split
//     into an fp16 hi + lo pair (w = hi + lo to ~2^-22).
//   * One mma.m16n8k16 (fp16 x fp16 -> fp32) multiplies 16 spectra x 8
//     antennas by an 8-column weight matrix whose columns are (re, im) x
//     (hi, lo) of the beam.  The hi and lo partial sums are added in fp32,
//     then |.|^2.
//   * Lanes (g, q) of the fragment map to spectra g, g+8 and to the q-th
//     quarter of the antenna row, so each thread loads its A/4 contiguous
//     bytes of two rows; the K order of the contraction is permuted to match
//     the decode (only the weights need to follow it).
// A CTA of 8 warps takes 8 consecutive channels (512 contiguous bytes per
// spectrum at 64 antennas) for one window; per-spectrum powers are staged in
// shared memory so each spectrum's 8 channels are written as one 32-byte
// sector.
#include "bf_internal.cuh"
#include "tracker_common.cuh"

#include <cuda_fp16.h>

namespace bf {
namespace {

using namespace trk;

constexpr int kChannelsPerCta = 8;

template <int A>
__global__ void __launch_bounds__(kChannelsPerCta * 32)
tracker_stream_kernel(const uint8_t* __restrict__ v, const float* __restrict__ pos,
                      const double* __restrict__ kw, const float* __restrict__ dirs,
                      float* __restrict__ intensity, float* __restrict__ integrated, int n_time,
                      int n_freq, int spectra) {
    constexpr int NW = A / 16;          // 32-bit words per thread per spectrum
    constexpr int kBytes = A / 4;       // bytes per thread per spectrum
    __shared__ float stage[16][kChannelsPerCta];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int win = blockIdx.x;
    const int f = blockIdx.y * kChannelsPerCta + warp;
    const bool fvalid = f < n_freq;

    // B fragments for this window: column g in (re_hi, im_hi, re_lo, im_lo, 0...).
    uint32_t bfrag[NW][2][2];
    {
        const bool used = g < 4 && fvalid;
        const bool is_im = (g & 1) != 0, is_lo = (g >> 1) != 0;
        const double k = fvalid ? kw[f] : 0.0;
        const double dx = dirs[3 * win], dy = dirs[3 * win + 1], dz = dirs[3 * win + 2];
#pragma unroll
        for (int j = 0; j < NW; ++j) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int a0 = q * kBytes + 4 * j + s, a1 = a0 + 2;
                uint32_t xr = 0, xi = 0;
                if (used) {
                    const float2 w0 = steering_weight(pos, a0, k, dx, dy, dz);
                    const float2 w1 = steering_weight(pos, a1, k, dx, dy, dz);
                    // re: xr*wr - xi*wi ; im: xr*wi + xi*wr
                    const float cr0 = is_im ? w0.y : w0.x, cr1 = is_im ? w1.y : w1.x;
                    const float ci0 = is_im ? w0.x : -w0.y, ci1 = is_im ? w1.x : -w1.y;
                    xr = split_part(cr0, is_lo) | (static_cast<uint32_t>(split_part(cr1, is_lo)) << 16);
                    xi = split_part(ci0, is_lo) | (static_cast<uint32_t>(split_part(ci1, is_lo)) << 16);
                }
                bfrag[j][s][0] = xr;
                bfrag[j][s][1] = xi;
            }
        }
    }

    const int t_begin = win * spectra;
    const int t_end = min(t_begin + spectra, n_time);
    float acc = 0.f;
    // Rows g and g+8 of the 16-spectrum block starting at tb (zero past the window).
    auto load_rows = [&](int tb, uint32_t (&wg)[NW], uint32_t (&wg8)[NW]) {
        const int tg = tb + g, tg8 = tb + g + 8;
        const uint8_t* rg = v + (static_cast<size_t>(tg) * n_freq + f) * A + q * kBytes;
        const uint8_t* rg8 = v + (static_cast<size_t>(tg8) * n_freq + f) * A + q * kBytes;
        const bool vg = fvalid && tg < t_end, vg8 = fvalid && tg8 < t_end;
        if constexpr (A == 32) {
            const uint2 x0 = vg ? __ldg(reinterpret_cast<const uint2*>(rg)) : make_uint2(0, 0);
            const uint2 x1 = vg8 ? __ldg(reinterpret_cast<const uint2*>(rg8)) : make_uint2(0, 0);
            wg[0] = x0.x; wg[1] = x0.y; wg8[0] = x1.x; wg8[1] = x1.y;
        } else {
#pragma unroll
            for (int c = 0; c < NW / 4; ++c) {
                const uint4 x0 = vg ? __ldg(reinterpret_cast<const uint4*>(rg) + c) : make_uint4(0, 0, 0, 0);
                const uint4 x1 = vg8 ? __ldg(reinterpret_cast<const uint4*>(rg8) + c) : make_uint4(0, 0, 0, 0);
                wg[4 * c] = x0.x; wg[4 * c + 1] = x0.y; wg[4 * c + 2] = x0.z; wg[4 * c + 3] = x0.w;
                wg8[4 * c] = x1.x; wg8[4 * c + 1] = x1.y; wg8[4 * c + 2] = x1.z; wg8[4 * c + 3] = x1.w;
            }
        }
    };
    auto process = [&](const uint32_t (&wg)[NW], const uint32_t (&wg8)[NW], int tb) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            uint32_t re02g, im02g, re13g, im13g, re02h, im02h, re13h, im13h;
            decode_word(wg[j], re02g, im02g, re13g, im13g);
            decode_word(wg8[j], re02h, im02h, re13h, im13h);
            mma_16816(d, re02g, re02h, im02g, im02h, bfrag[j][0][0], bfrag[j][0][1]);
            mma_16816(d, re13g, re13h, im13g, im13h, bfrag[j][1][0], bfrag[j][1][1]);
        }
        // q == 0 holds (re_hi, im_hi), q == 1 holds (re_lo, im_lo) for rows g, g+8.
        float p[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) p[i] = __shfl_xor_sync(0xffffffffu, d[i], 1);
        const float re_g = d[0] + p[0], im_g = d[1] + p[1];
        const float re_h = d[2] + p[2], im_h = d[3] + p[3];
        const float pow_g = re_g * re_g + im_g * im_g;
        const float pow_h = re_h * re_h + im_h * im_h;
        if (q == 0) acc += pow_g + pow_h;
        if (intensity != nullptr) {
            if (q == 0) {
                stage[g][warp] = pow_g;
                stage[g + 8][warp] = pow_h;
            }
            __syncthreads();
            if (threadIdx.x < 16 * kChannelsPerCta) {
                const int r = threadIdx.x / kChannelsPerCta, c = threadIdx.x % kChannelsPerCta;
                const int fo = blockIdx.y * kChannelsPerCta + c;
                if (tb + r < t_end && fo < n_freq) {
                    intensity[static_cast<size_t>(tb + r) * n_freq + fo] = stage[r][c];
                }
            }
            __syncthreads();
        }
    };
    // software pipeline: the next two blocks' loads are in flight while two
    // blocks compute (blocks are still summed one by one in increasing time)
    uint32_t wa[NW], wa8[NW], wb[NW], wb8[NW];
    load_rows(t_begin, wa, wa8);
    load_rows(t_begin + 16, wb, wb8);
    for (int tb = t_begin; tb < t_end; tb += 32) {
        uint32_t na[NW], na8[NW], nb[NW], nb8[NW];
        load_rows(tb + 32, na, na8);
        load_rows(tb + 48, nb, nb8);
        process(wa, wa8, tb);
        if (tb + 16 < t_end) process(wb, wb8, tb + 16);  // uniform across the CTA
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            wa[j] = na[j];
            wa8[j] = na8[j];
            wb[j] = nb[j];
            wb8[j] = nb8[j];
        }
    }
    if (integrated != nullptr) {
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        acc += __shfl_xor_sync(0xffffffffu, acc, 8);
        acc += __shfl_xor_sync(0xffffffffu, acc, 16);
        if (lane == 0 && fvalid) integrated[static_cast<size_t>(win) * n_freq + f] = acc;
    }
}

}  // namespace

bf_status launch_tracker_stream(cudaStream_t stream, const uint8_t* v, const float* pos,
                                const double* k, const float* dirs, float* intensity,
                                float* integrated, const bf_dims& d, uint64_t spectra) {
    const uint64_t W = window_count(d.n_time, spectra);
    if (W > 0x7fffffffull || d.n_time > 0x7fffffffull) {
        return set_error(BF_ERR_OVERFLOW, "CUDA tracker grid exceeds the supported size");
    }
    const dim3 grid(static_cast<unsigned>(W),
                    static_cast<unsigned>((d.n_freq + kChannelsPerCta - 1) / kChannelsPerCta));
    const dim3 block(kChannelsPerCta * 32);
    const int T = static_cast<int>(d.n_time), F = static_cast<int>(d.n_freq);
    const int S = static_cast<int>(spectra);
    switch (d.n_ant) {
        case 32:
            tracker_stream_kernel<32><<<grid, block, 0, stream>>>(v, pos, k, dirs, intensity, integrated, T, F, S);
            break;
        case 64:
            tracker_stream_kernel<64><<<grid, block, 0, stream>>>(v, pos, k, dirs, intensity, integrated, T, F, S);
            break;
        case 128:
            tracker_stream_kernel<128><<<grid, block, 0, stream>>>(v, pos, k, dirs, intensity, integrated, T, F, S);
            break;
        case 256:
            tracker_stream_kernel<256><<<grid, block, 0, stream>>>(v, pos, k, dirs, intensity, integrated, T, F, S);
            break;
        default:
            return set_error(BF_ERR_INVALID_ARGUMENT, "n_ant must be 32, 64, 128, or 256");
    }
    return cuda_status(cudaGetLastError(), "tracker_stream_kernel launch");
}

}  // namespace bf
