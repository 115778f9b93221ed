// loss_mask.cu -- consuming a shard's loss mask on the device.
//
// The reference defines the mask (include/beamformer/formats.hpp:22-30: one
// byte per [time][local frequency] frame, 0 = lost, the payload left as the
// RFSoC wrote it) and carries it with every shard, but nothing downstream
// reads it.  Here a lost frame's packed bytes become 0 (both nibbles zero),
// so it adds nothing to any beam, tracker or covariance sum, and the number
// of valid frames of every (integration window, channel) is counted so that
// integrated outputs can be normalised.  Any nonzero mask byte counts as
// valid.
//
// A thread takes one channel and a run of up to kRun consecutive frames;
// threads of a warp take consecutive channels, so mask reads coalesce and a
// lost frame's A bytes are cleared with 16-byte stores.  Counts go out with
// one atomic add per (thread, window touched).
#include "bf_internal.cuh"

#include <algorithm>

namespace bf {
namespace {

constexpr int kRun = 32;

__global__ void __launch_bounds__(256)
apply_loss_mask_kernel(uint8_t* __restrict v, const uint8_t* __restrict mask, long long n_time, int n_freq,
                       int n_ant, long long spectra, unsigned* __restrict counts) {
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long runs = (n_time + kRun - 1) / kRun;
    if (idx >= runs * n_freq) return;
    const int f = static_cast<int>(idx % n_freq);
    const long long t0 = (idx / n_freq) * kRun;
    const long long t1 = t0 + kRun < n_time ? t0 + kRun : n_time;
    const int words = n_ant / 16;
    unsigned valid = 0;
    long long win = t0 / spectra;
    for (long long t = t0; t < t1; ++t) {
        const long long w = t / spectra;
        if (w != win) {
            if (counts != nullptr && valid != 0) atomicAdd(&counts[win * n_freq + f], valid);
            valid = 0;
            win = w;
        }
        const long long frame = t * n_freq + f;
        if (mask[frame] != 0) {
            ++valid;
        } else {
            uint4* row = reinterpret_cast<uint4*>(v + frame * n_ant);
            for (int i = 0; i < words; ++i) row[i] = make_uint4(0, 0, 0, 0);
        }
    }
    if (counts != nullptr && valid != 0) atomicAdd(&counts[win * n_freq + f], valid);
}

}  // namespace

bf_status launch_apply_loss_mask(cudaStream_t stream, uint8_t* v, const uint8_t* mask, uint64_t n_time,
                                 uint64_t n_freq, uint64_t n_ant, uint64_t spectra, uint32_t* counts) {
    if (counts != nullptr) {
        const uint64_t n = window_count(n_time, spectra) * n_freq;
        BF_RETURN_IF(cuda_status(cudaMemsetAsync(counts, 0, n * sizeof(uint32_t), stream), "valid_counts clear"));
    }
    const uint64_t threads = (n_time + kRun - 1) / kRun * n_freq;
    const uint64_t blocks = (threads + 255) / 256;
    if (blocks > 0x7fffffffull) return set_error(BF_ERR_OVERFLOW, "loss mask grid too large");
    apply_loss_mask_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
        v, mask, static_cast<long long>(n_time), static_cast<int>(n_freq), static_cast<int>(n_ant),
        static_cast<long long>(spectra), reinterpret_cast<unsigned*>(counts));
    return cuda_status(cudaGetLastError(), "apply_loss_mask_kernel launch");
}

}  // namespace bf
