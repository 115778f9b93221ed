// doa_cov.cu -- exact per-block array covariance on int8 tensor cores.
//
// Reference: CpuOptBeamTracker forms, per frequency and block of K snapshots,
// R[f] = (1/K) sum_k x_k x_k^H in std::complex<float>
// (src/cpu_opt_beam_tracker.cpp:559-602).  Here the block sums are formed
// exactly in INT32:
//   R_blk[b][f][i][j] = sum_{t in block b} x_i(t) * conj(x_j(t))
// (re, im) as int32, for the full A x A Hermitian matrix.  Spatial smoothing,
// forward-backward averaging, 1/K, diagonal loading and forgetting are linear
// and run afterwards in FP64 (doa_scan.cu).
//
// Formulation: with y(t) the 2A real components of x(t), the Gram matrix
// G = sum_t y(t) y(t)^T is one tcgen05 kind::i8 GEMM per (block, channel):
// M = N = 128 components (zero padded for 32 antennas), K = time.  The
// unpacked tile [t][128 bytes] is MN-major for both operands, so one
// shared-memory tile feeds A and B.  The tile holds the components in offset
// binary, u = y + 8 in 0..15 (one lop3 per four nibbles), and the MMA runs
// u8 x u8; the epilogue restores
//   G_ij = Gu_ij - 8 (S_i + S_j) + 64 K,   S_i = sum_t u_i(t),
// with S gathered by the unpack warps from the same bytes.  A 16-byte chunk
// of the tile holds 8 antennas as [re 0-3][im 0-3][re 4-7][im 4-7], so
// component m = 16 c + 4 h + k is antenna 8 c + 4 (h >> 1) + k, part h & 1.
// R assembles from G in the epilogue: Re R_ij = G(re i, re j) + G(im i, im j),
// Im R_ij = G(im i, re j) - G(re i, im j).  u <= 15, so Gu stays below 2^31
// for blocks of up to 2^23 spectra.
//
// CTA (one per SM): a unit is (block, channel pair), so every TMA box row is
// the pair's 2A contiguous bytes (a whole 128-byte line at 64 antennas; a
// single channel's 64 bytes would make DRAM fetch the neighbour twice).
// Warp 0 TMA producer (raw 128-spectrum tiles of both channels), warp 1 MMA
// issuer and TMEM owner, warps 2-19 unpack (int4 -> offset-binary bytes,
// 128-byte swizzle, one tile per channel; a warp reads two spectra of both
// channels, 256 contiguous bytes, so the raw loads are conflict free), warps
// 20-23 epilogue (two 128 x 128 int32 accumulators per unit, two TMEM stages
// of 256 columns).  All waits are bounded and report through the device
// error word.
#include "bf_internal.cuh"
#include "sm100.cuh"

#include <cuda.h>

#include <algorithm>
#include <mutex>

namespace bf {

namespace {

using namespace sm100;

constexpr int kThreads = 768;
constexpr int kUnpackWarps = 18;                 // nine per channel of the pair
constexpr int kEpiFirstWarp = 2 + kUnpackWarps;
constexpr int kRowStep = 32 * kUnpackWarps / 16; // rows between a thread's chunks
constexpr int kTile = 128;        // spectra per tile
constexpr int kRawStages = 5;
constexpr int kXStages = 3;
constexpr uint32_t kXBytes = 2 * kTile * 128;  // one unpacked tile per channel of the pair
constexpr uint64_t kWaitNs = 2000000000ull;

struct CovParams {
    int32_t* out;             // [blocks][F][A][A][2]
    unsigned* err;            // device error word (bits 16 and up)
    int n_freq, n_ant, block_len, n_blocks, tiles_per_block, n_pairs;
    long long n_units;        // n_blocks * n_pairs
};

__device__ __forceinline__ void cov_error(unsigned* err, unsigned code) {
    if (err != nullptr) atomicOr(err, code << 16);
}

// 8 packed bytes (antennas 8c..8c+7) -> 16 offset-binary components
// [re 0-3][im 0-3][re 4-7][im 4-7]: a two's-complement nibble n becomes
// u = n ^ 8 = n + 8 (mod 16), one lop3 ((w & 0x0F..) ^ 0x08..) per word.
__device__ __forceinline__ uint32_t offset4(uint32_t w) {
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(r) : "r"(w), "r"(0x0F0F0F0Fu), "r"(0x08080808u));
    return r;
}
__device__ __forceinline__ uint4 offset8(uint32_t w0, uint32_t w1) {
    return make_uint4(offset4(w0), offset4(w0 >> 4), offset4(w1), offset4(w1 >> 4));
}

template <int A>
__global__ void __launch_bounds__(kThreads, 1)
doa_cov_kernel(const __grid_constant__ CUtensorMap vmap, const CovParams p) {
    constexpr uint32_t RAW = kTile * 2 * A;              // [row][2 channels][A]
    constexpr uint32_t IDESC = idesc_u8_s32_mn(128, 128);
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* xs = smem;                                  // kXStages x 2 x 16 KiB
    uint8_t* raw = smem + kXStages * kXBytes;            // kRawStages x RAW
    uint64_t* bars = reinterpret_cast<uint64_t*>(raw + kRawStages * RAW);  // 512 bytes
    uint32_t* s_part = reinterpret_cast<uint32_t*>(raw + kRawStages * RAW + 512);  // [2][kUnpackWarps][2][128]
    uint32_t* s_sum = s_part + 2 * kUnpackWarps * 256;                             // [2][2][128]
    uint64_t* raw_full = bars;                           // [kRawStages]
    uint64_t* raw_empty = bars + kRawStages;             // [kRawStages]
    uint64_t* x_full = bars + 2 * kRawStages;            // [kXStages]
    uint64_t* x_empty = x_full + kXStages;               // [kXStages]
    uint64_t* acc_full = x_empty + kXStages;             // [2]
    uint64_t* acc_empty = acc_full + 2;                  // [2]
    uint64_t* mma_done = acc_empty + 2;
    uint64_t* part_full = mma_done + 1;                  // [2] unpack warps -> epilogue
    uint64_t* part_empty = part_full + 2;                // [2] epilogue -> unpack warps
    uint64_t* sum_ready = part_empty + 2;                // [2] among the epilogue warps
    uint32_t* tmem_ptr = reinterpret_cast<uint32_t*>(sum_ready + 2);
    volatile int* s_fail = reinterpret_cast<volatile int*>(sum_ready + 3);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRawStages; ++i) {
            mbar_init(&raw_full[i], 1);
            mbar_init(&raw_empty[i], kUnpackWarps);
        }
        for (int i = 0; i < kXStages; ++i) {
            mbar_init(&x_full[i], kUnpackWarps);
            mbar_init(&x_empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], 4);
        }
        mbar_init(mma_done, 1);
        for (int i = 0; i < 2; ++i) {
            mbar_init(&part_full[i], kUnpackWarps);
            mbar_init(&part_empty[i], 4);
            mbar_init(&sum_ready[i], 4);
        }
        *s_fail = 0;
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(tmem_ptr, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_ptr;

    const long long u_begin = p.n_units * blockIdx.x / gridDim.x;
    const long long u_end = p.n_units * (blockIdx.x + 1) / gridDim.x;
    auto fail = [&](unsigned code) {
        cov_error(p.err, code);
        *s_fail = 1;
    };

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int armed[kRawStages];
            for (int s = 0; s < kRawStages; ++s) armed[s] = -1;
            bool stop = false;
            for (long long u = u_begin; u < u_end && !stop; ++u) {
                const int b = static_cast<int>(u / p.n_pairs), fp = static_cast<int>(u % p.n_pairs);
                for (int k = 0; k < p.tiles_per_block; ++k) {
                    if (*s_fail) { stop = true; break; }
                    if (!mbar_wait(&raw_empty[stage], phase ^ 1, kWaitNs)) { fail(1); stop = true; break; }
                    mbar_expect_tx(&raw_full[stage], RAW);  // a missing odd channel arrives zero filled
                    tma_load_4d(raw + stage * RAW, &vmap, 0, 2 * fp, b * p.block_len + k * kTile, 0, &raw_full[stage]);
                    armed[stage] = static_cast<int>(phase);
                    if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                }
            }
            for (int s = 0; s < kRawStages; ++s) {
                if (armed[s] >= 0 && !mbar_wait(&raw_full[s], static_cast<uint32_t>(armed[s]), kWaitNs)) fail(2);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int xst = 0, ast = 0;
            uint32_t xph = 0, aph = 0;
            bool stop = false;
            for (long long u = u_begin; u < u_end && !stop; ++u) {
                if (!mbar_wait(&acc_empty[ast], aph ^ 1, kWaitNs)) { fail(4); break; }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + ast * 256;
                for (int k = 0; k < p.tiles_per_block; ++k) {
                    if (*s_fail) { stop = true; break; }
                    if (!mbar_wait(&x_full[xst], xph, kWaitNs)) { fail(8); stop = true; break; }
                    tc_fence_after();
#pragma unroll
                    for (int ch = 0; ch < 2; ++ch) {
                        const uint32_t xa = smem_u32(xs + xst * kXBytes + ch * (kTile * 128));
#pragma unroll
                        for (int kk = 0; kk < kTile / 32; ++kk) {
                            const uint64_t desc = smem_desc_sw128_mn(xa + kk * 32 * 128);
                            mma_i8_ss(d_tmem + ch * 128, desc, desc, IDESC, (k > 0 || kk > 0) ? 1u : 0u);
                        }
                    }
                    tc_commit(&x_empty[xst]);
                    if (++xst == kXStages) { xst = 0; xph ^= 1; }
                }
                if (stop) break;
                tc_commit(&acc_full[ast]);
                if (++ast == 2) { ast = 0; aph ^= 1; }
            }
            tc_commit(mma_done);
            if (!mbar_wait(mma_done, 0, kWaitNs)) fail(16);
        }
    } else if (warp < kEpiFirstWarp) {
        // thread = (chunk c of 8 antennas, channel, first row r0) from its
        // index bits (2..0, 3, 9..4); rows r0, r0 + kRowStep, ... of every
        // tile.  Component sums: bytes[] adds the
        // offset words (at most 4 rows x 15 per byte per tile, flushed every
        // 4 tiles), wide[] the even / odd bytes in 16-bit lanes (flushed to
        // total[] every 512 tiles), total[] the unit's sums.
        const int ut = threadIdx.x - 64;
        const int c = ut & 7, ch = (ut >> 3) & 1, r0 = ut >> 4;
        const bool live = c < A / 8;
        // rows r0 + i kRowStep, i < 4 (the fourth exists for r0 < 20); the
        // swizzle r & 7 alternates between two values since kRowStep % 8 == 4
        static_assert(kRowStep % 8 == 4 && 3 * kRowStep < kTile && 4 * kRowStep >= kTile, "row split");
        const bool has4 = r0 + 3 * kRowStep < kTile;
        const int raw_off = ch * A + c * 8 + r0 * 2 * A;
        const int x_off = ch * (kTile * 128) + r0 * 128;
        const int xsw_even = (c ^ (r0 & 7)) << 4, xsw_odd = xsw_even ^ 64;
        int stage = 0, xst = 0, pst = 0;
        uint32_t phase = 0, xph = 0, pph = 0;
        bool stop = false;
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            uint32_t bytes[4] = {0, 0, 0, 0}, wide[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t total[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) total[i] = 0;
            auto flush_bytes = [&]() {
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    wide[h] += bytes[h] & 0x00FF00FFu;
                    wide[4 + h] += (bytes[h] >> 8) & 0x00FF00FFu;
                    bytes[h] = 0;
                }
            };
            auto flush_wide = [&]() {
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    total[4 * h + 0] += wide[h] & 0xFFFFu;
                    total[4 * h + 2] += wide[h] >> 16;
                    total[4 * h + 1] += wide[4 + h] & 0xFFFFu;
                    total[4 * h + 3] += wide[4 + h] >> 16;
                    wide[h] = wide[4 + h] = 0;
                }
            };
            for (int k = 0; k < p.tiles_per_block; ++k) {
                if (*s_fail) { stop = true; break; }
                if (!mbar_wait(&raw_full[stage], phase, kWaitNs)) { fail(32); stop = true; break; }
                if (!mbar_wait(&x_empty[xst], xph ^ 1, kWaitNs)) { fail(64); stop = true; break; }
                const uint8_t* rsrc = raw + stage * RAW + raw_off;
                uint8_t* xdst = xs + xst * kXBytes + x_off;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (i < 3 || has4) {
                        uint4 v = make_uint4(0, 0, 0, 0);
                        if (live) {
                            const uint2 w = *reinterpret_cast<const uint2*>(rsrc + i * kRowStep * 2 * A);
                            v = offset8(w.x, w.y);
                            bytes[0] += v.x;
                            bytes[1] += v.y;
                            bytes[2] += v.z;
                            bytes[3] += v.w;
                        }
                        *reinterpret_cast<uint4*>(xdst + i * kRowStep * 128 + ((i & 1) != 0 ? xsw_odd : xsw_even)) = v;
                    }
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&raw_empty[stage]);
                    mbar_arrive(&x_full[xst]);
                }
                if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                if (++xst == kXStages) { xst = 0; xph ^= 1; }
                if ((k & 3) == 3) flush_bytes();
                if ((k & 511) == 511) flush_wide();
            }
            if (stop) break;
            flush_bytes();
            flush_wide();
            // the warp's two row groups share each (channel, chunk): lanes l, l + 16
#pragma unroll
            for (int i = 0; i < 16; ++i) total[i] += __shfl_xor_sync(0xffffffffu, total[i], 16);
            if (!mbar_wait(&part_empty[pst], pph ^ 1, kWaitNs)) { fail(256); break; }
            if (lane < 16) {
                uint32_t* dst = s_part + ((pst * kUnpackWarps + (warp - 2)) * 2 + ch) * 128 + 16 * c;
#pragma unroll
                for (int i = 0; i < 16; ++i) dst[i] = total[i];
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&part_full[pst]);
            if (++pst == 2) { pst = 0; pph ^= 1; }
        }
    } else {
        const int q4 = warp & 3;
        const int et = 32 * (warp - kEpiFirstWarp) + lane;  // 0 .. 127
        const int m = 32 * q4 + lane;                         // component row of G
        const int mc = m >> 4, mh = (m >> 2) & 3;
        const int i = 8 * mc + 4 * (mh >> 1) + (m & 3);       // antenna
        const int comp = mh & 1;                              // 0 = re / 1 = im part of R
        const uint32_t k64 = 64u * static_cast<uint32_t>(p.block_len);
        int ast = 0;
        uint32_t aph = 0;
        bool stop = false;
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            // component sums of the unit: one partial per unpack warp and channel
            if (!mbar_wait(&part_full[ast], aph, kWaitNs)) { fail(512); break; }
#pragma unroll
            for (int ch = 0; ch < 2; ++ch) {
                uint32_t acc = 0;
#pragma unroll
                for (int w = 0; w < kUnpackWarps; ++w) {
                    acc += s_part[((ast * kUnpackWarps + w) * 2 + ch) * 128 + et];
                }
                s_sum[(ast * 2 + ch) * 128 + et] = acc;
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&part_empty[ast]);
                mbar_arrive(&sum_ready[ast]);
            }
            if (!mbar_wait(&sum_ready[ast], aph, kWaitNs)) { fail(1024); break; }
            if (!mbar_wait(&acc_full[ast], aph, kWaitNs)) { fail(128); break; }
            tc_fence_after();
            const int b = static_cast<int>(u / p.n_pairs), fp = static_cast<int>(u % p.n_pairs);
#pragma unroll 1
            for (int ch = 0; ch < 2; ++ch) {
                const int f = 2 * fp + ch;
                if (f >= p.n_freq) break;
                const uint32_t* sums = s_sum + (ast * 2 + ch) * 128;
                // G = Gu - 8 (S_m + S_n) + 64 K, in wrapping 32-bit arithmetic
                const uint32_t bias_m = k64 - 8u * sums[m];
                int32_t* row = p.out + ((static_cast<size_t>(b) * p.n_freq + f) * A + i) * A * 2;
                const uint32_t taddr = tmem_base + ((32u * q4) << 16) + ast * 256 + ch * 128;
#pragma unroll 1
                for (int cc = 0; cc < 4; ++cc) {
                    uint32_t g[32];
                    tmem_ld_32x32b_x32(taddr + 32 * cc, g);
                    tmem_ld_wait();
#pragma unroll
                    for (int jl = 0; jl < 16; ++jl) {
                        // antenna j = 16 cc + jl: columns re j and im j of this 32-column chunk
                        const int j = 16 * cc + jl;
                        const int n_re = 16 * (jl >> 3) + 8 * ((jl >> 2) & 1) + (jl & 3), n_im = n_re + 4;
                        const uint32_t own = g[n_re] + bias_m - 8u * sums[32 * cc + n_re];
                        const uint32_t send = g[n_im] + bias_m - 8u * sums[32 * cc + n_im];
                        const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, 4);
                        const int32_t val = static_cast<int32_t>(comp == 0 ? own + recv : own - recv);
                        if (i < A && j < A) row[2 * j + comp] = val;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[ast]);
            if (++ast == 2) { ast = 0; aph ^= 1; }
            stop = *s_fail != 0;
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, 512);
    }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn_cov() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
        }
    });
    return fn;
}

template <int A>
bf_status launch_cov(cudaStream_t stream, const CUtensorMap& map, const CovParams& p) {
    // at least 120 KB, so that one CTA (512 TMEM columns) holds an SM and
    // tcgen05.alloc never has to wait for a column
    const size_t smem = std::max<size_t>(kXStages * kXBytes + kRawStages * kTile * 2 * A + 512 +
                                             (4 * kUnpackWarps + 4) * 128 * sizeof(uint32_t) + 1024,
                                         120 * 1024);
    auto kern = doa_cov_kernel<A>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "doa_cov_kernel smem attribute");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = static_cast<int>(std::min<long long>(sms, p.n_units));
    kern<<<grid, kThreads, smem, stream>>>(map, p);
    return cuda_status(cudaGetLastError(), "doa_cov_kernel launch");
}

}  // namespace

bf_status launch_doa_covariance(cudaStream_t stream, const uint8_t* v, int32_t* out, const bf_dims& d,
                                uint64_t block_len) {
    if (d.n_ant != 32 && d.n_ant != 64) {
        return set_error(BF_ERR_UNSUPPORTED, "the tensor-core covariance supports n_ant 32 or 64");
    }
    if (block_len == 0 || block_len % kTile != 0 || d.n_time % block_len != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         "block length must be a positive multiple of 128 that divides n_time");
    }
    if (block_len > (1ull << 23) || d.n_time >= (1ull << 31)) {
        return set_error(BF_ERR_OVERFLOW, "covariance block or stream too long for int32 sums");
    }
    EncodeTiledFn enc = encode_fn_cov();
    if (enc == nullptr) return set_error(BF_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    CUtensorMap map;
    const cuuint64_t dims[4] = {d.n_ant, d.n_freq, d.n_time, 1};
    const cuuint64_t strides[3] = {d.n_ant, d.n_freq * d.n_ant, d.n_time * d.n_freq * d.n_ant};
    const cuuint32_t box[4] = {static_cast<cuuint32_t>(d.n_ant), 2, static_cast<cuuint32_t>(kTile), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<uint8_t*>(v), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(BF_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(r));
    CovParams p{};
    p.out = out;
    p.err = device_error_word(stream);
    if (p.err == nullptr) return BF_ERR_CUDA;
    p.n_freq = static_cast<int>(d.n_freq);
    p.n_ant = static_cast<int>(d.n_ant);
    p.block_len = static_cast<int>(block_len);
    p.n_blocks = static_cast<int>(d.n_time / block_len);
    p.tiles_per_block = static_cast<int>(block_len / kTile);
    p.n_pairs = static_cast<int>((d.n_freq + 1) / 2);
    p.n_units = static_cast<long long>(p.n_blocks) * p.n_pairs;
    return d.n_ant == 32 ? launch_cov<32>(stream, map, p) : launch_cov<64>(stream, map, p);
}

}  // namespace bf
