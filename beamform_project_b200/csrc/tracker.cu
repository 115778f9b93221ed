// tracker.cu -- dynamic single-beam tracker (n_beams == 1).
//
// Reference behaviour: beam_tracker_cpu_packed_intensity_into
// (src/beam_tracker.cpp:90-146) computes one weight set per integration
// window from the window's direction (evaluated at the window's first sample,
// src/beam_tracker.cpp:52-76) and writes the per-spectrum power [T][F][1].
// The reference GPU trackers (src/cuda_beam_tracker_v5.cu:137-273) compute
// the same weights on the device in FP64.
//
// mode 0 (this file): reference float32 operation order.  One CTA per
//   (window, 32-channel block); the window's weights are generated once into
//   shared memory ([A][32] float2) with the FP64 delay, FP64 phase and FP64
//   sin/cos rounded to float exactly as src/weights.cpp:42-55.  Each of the 8
//   warps takes every 8th spectrum of the window (lanes = channels, 64-byte
//   coalesced rows); the optional per-window sum is taken in increasing time
//   through a small shared-memory stage, as src/temporal_integration.cpp:
//   95-109 would sum the per-spectrum output.
// mode 1 (tracker_stream.cu): the HBM streaming kernel.
#include "bf_internal.cuh"

namespace bf {

bf_status launch_tracker_stream(cudaStream_t stream, const uint8_t* v, const float* pos,
                                const double* k, const float* dirs, float* intensity,
                                float* integrated, const bf_dims& d, uint64_t spectra);

namespace {

constexpr int kSlots = 8;

__global__ void __launch_bounds__(kSlots * 32)
tracker_exact_kernel(const uint8_t* __restrict__ v, const float* __restrict__ pos,
                     const double* __restrict__ kw, const float* __restrict__ dirs,
                     float* __restrict__ intensity, float* __restrict__ integrated, int n_time,
                     int n_freq, int n_ant, int spectra) {
    extern __shared__ float2 ws[];  // [A][32]
    __shared__ float pw[kSlots][32];
    const int win = blockIdx.x;
    const int f0 = blockIdx.y * 32;
    const int lane = threadIdx.x & 31, slot = threadIdx.x >> 5;

    const double dx = dirs[3 * win], dy = dirs[3 * win + 1], dz = dirs[3 * win + 2];
    for (int i = threadIdx.x; i < n_ant * 32; i += blockDim.x) {
        const int a = i >> 5, f = f0 + (i & 31);
        float2 w = make_float2(0.f, 0.f);
        if (f < n_freq) {
            const double delay = __dadd_rn(__dadd_rn(__dmul_rn((double)pos[3 * a], dx),
                                                     __dmul_rn((double)pos[3 * a + 1], dy)),
                                           __dmul_rn((double)pos[3 * a + 2], dz));
            const double phase = __dmul_rn(kw[f], delay);
            double s, c;
            sincos(phase, &s, &c);
            w = make_float2(static_cast<float>(c), static_cast<float>(s));
        }
        ws[i] = w;
    }
    __syncthreads();

    const int f = f0 + lane;
    const int t0 = win * spectra;
    const int t1 = min(t0 + spectra, n_time);
    float acc = 0.f;
    for (int tb = t0; tb < t1; tb += kSlots) {
        const int t = tb + slot;
        float p = 0.f;
        if (t < t1 && f < n_freq) {
            const uint8_t* row = v + (static_cast<size_t>(t) * n_freq + f) * n_ant;
            float sr = 0.f, si = 0.f;
            for (int a0 = 0; a0 < n_ant; a0 += 16) {
                const uint4 raw = __ldg(reinterpret_cast<const uint4*>(row + a0));
                const uint32_t words[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const uint32_t byte = (words[j >> 2] >> (8 * (j & 3))) & 0xFFu;
                    const float2 w = ws[(a0 + j) * 32 + lane];
                    cmac_ref(sr, si, w.x, w.y, static_cast<float>(nibble_lo(byte)),
                             static_cast<float>(nibble_hi(byte)));
                }
            }
            p = power_ref(sr, si);
            if (intensity != nullptr) intensity[static_cast<size_t>(t) * n_freq + f] = p;
        }
        if (integrated != nullptr) {
            pw[slot][lane] = p;
            __syncthreads();
            if (slot == 0) {
                for (int s = 0; s < kSlots && tb + s < t1; ++s) acc = __fadd_rn(acc, pw[s][lane]);
            }
            __syncthreads();
        }
    }
    if (integrated != nullptr && slot == 0 && f < n_freq) {
        integrated[static_cast<size_t>(win) * n_freq + f] = acc;
    }
}

}  // namespace

bf_status launch_tracker(cudaStream_t stream, int mode, const uint8_t* v, const float* pos,
                         const double* k, const float* dirs, float* intensity, float* integrated,
                         const bf_dims& d, uint64_t spectra) {
    if (mode == 1) {
        return launch_tracker_stream(stream, v, pos, k, dirs, intensity, integrated, d, spectra);
    }
    const uint64_t W = window_count(d.n_time, spectra);
    if (W > 0x7fffffffull || d.n_time > 0x7fffffffull) {
        return set_error(BF_ERR_OVERFLOW, "CUDA tracker grid exceeds the supported size");
    }
    const size_t smem = d.n_ant * 32 * sizeof(float2);
    cudaError_t err = cudaFuncSetAttribute(tracker_exact_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return cuda_status(err, "tracker_exact_kernel smem attribute");
    const dim3 grid(static_cast<unsigned>(W), static_cast<unsigned>((d.n_freq + 31) / 32));
    tracker_exact_kernel<<<grid, kSlots * 32, smem, stream>>>(
        v, pos, k, dirs, intensity, integrated, static_cast<int>(d.n_time),
        static_cast<int>(d.n_freq), static_cast<int>(d.n_ant), static_cast<int>(spectra));
    return cuda_status(cudaGetLastError(), "tracker_exact_kernel launch");
}

}  // namespace bf
