// generate.cu -- seeded synthetic complex int4 voltages on the device.
//
// Not a reference kernel: the reference draws uniform integers from
// std::mt19937 on the host (src/synthetic_data.cpp:107-119).  Inputs of the
// sizes benchmarked here (up to several GB) are produced on the GPU instead,
// with an integer-only counter hash (splitmix64 finaliser) feeding an
// Irwin-Hall sum of eight 16-bit uniforms.  The float32 steps are correctly
// rounded mul/add and a half-to-even round, so the CPU restatement in the
// oracle reproduces every byte.
#include "bf_internal.cuh"

#include <algorithm>

namespace bf {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ int irwin_hall8(uint64_t seed, uint64_t counter) {
    const uint64_t h0 = mix64(seed ^ mix64(2 * counter));
    const uint64_t h1 = mix64(seed ^ mix64(2 * counter + 1));
    int s = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        s += static_cast<int>((h0 >> (16 * i)) & 0xFFFFu);
        s += static_cast<int>((h1 >> (16 * i)) & 0xFFFFu);
    }
    return 2 * s - 8 * 65535;
}

__device__ __forceinline__ uint32_t round_clip_nibble(float x) {
    int i = __float2int_rn(x);
    i = max(-8, min(7, i));
    return static_cast<uint32_t>(i) & 0xFu;
}

__global__ void generate_kernel(uint64_t seed, uint64_t offset, float scale,
                                const float2* __restrict__ mu, uint64_t epoch_len,
                                uint8_t* __restrict__ out, uint64_t n_freq, uint64_t n_ant,
                                uint64_t total) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += stride) {
        float mr = 0.f, mi = 0.f;
        if (mu != nullptr) {
            const uint64_t a = i % n_ant;
            const uint64_t tf = i / n_ant;
            const uint64_t f = tf % n_freq, t = tf / n_freq;
            const float2 m = mu[((t / epoch_len) * n_freq + f) * n_ant + a];
            mr = m.x;
            mi = m.y;
        }
        const uint64_t c = offset + i;
        const float gr = static_cast<float>(irwin_hall8(seed, 2 * c));
        const float gi = static_cast<float>(irwin_hall8(seed, 2 * c + 1));
        const uint32_t re = round_clip_nibble(__fadd_rn(__fmul_rn(gr, scale), mr));
        const uint32_t im = round_clip_nibble(__fadd_rn(__fmul_rn(gi, scale), mi));
        out[i] = static_cast<uint8_t>(re | (im << 4));
    }
}

}  // namespace

bf_status launch_generate(cudaStream_t stream, uint64_t seed, uint64_t offset, float scale,
                          const float* mu, uint64_t epoch_len, uint8_t* out, const bf_dims& d) {
    const uint64_t total = d.n_time * d.n_freq * d.n_ant;
    if (total == 0) return BF_OK;
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((total + 255) / 256, 148ull * 64));
    generate_kernel<<<blocks, 256, 0, stream>>>(seed, offset, scale,
                                                reinterpret_cast<const float2*>(mu), epoch_len,
                                                out, d.n_freq, d.n_ant, total);
    return cuda_status(cudaGetLastError(), "generate_kernel launch");
}

}  // namespace bf
