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
// Formulation: with y(t) the 2A real components (re, im interleaved) of x(t),
// the Gram matrix G = sum_t y(t) y(t)^T is one tcgen05 kind::i8 GEMM per
// (block, channel): M = N = 128 components (zero padded for 32 antennas),
// K = time.  The unpacked tile [t][128 int8] is MN-major for both operands,
// so one shared-memory tile feeds A and B.  R assembles from G in the
// epilogue: Re R_ij = G_{2i,2j} + G_{2i+1,2j+1}, Im R_ij = G_{2i+1,2j} -
// G_{2i,2j+1}.  |x| <= 8 per component, so every sum stays below 2^31 for
// blocks of up to 2^24 spectra.
//
// CTA (one per SM): a unit is (block, channel pair), so every TMA box row is
// the pair's 2A contiguous bytes (a whole 128-byte line at 64 antennas; a
// single channel's 64 bytes would make DRAM fetch the neighbour twice).
// Warp 0 TMA producer (raw 128-spectrum tiles of both channels), warp 1 MMA
// issuer and TMEM owner, warps 2-11 unpack (int4 -> int8, 128-byte swizzle,
// one tile per channel), warps 12-15 epilogue (two 128 x 128 int32
// accumulators per unit, two TMEM stages of 256 columns).  All waits are
// bounded and report through the device error word.
#include "bf_internal.cuh"
#include "sm100.cuh"

#include <cuda.h>

#include <algorithm>
#include <mutex>

namespace bf {

namespace {

using namespace sm100;

constexpr int kThreads = 512;
constexpr int kUnpackWarps = 10;
constexpr int kTile = 128;        // spectra per tile
constexpr int kRawStages = 6;
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

// 8 packed bytes (antennas 8c..8c+7) -> 16 int8 components (re, im interleaved).
// A nibble n becomes the signed byte ((n ^ 8) + 0x78) ^ 0x80: n ^ 8 is in
// 0..15, + 0x78 stays below 0x100 (no carry into the next byte), and the
// final xor maps 0x78 + (n ^ 8) onto n - 16 * (n >= 8).
__device__ __forceinline__ uint4 expand8(uint32_t w0, uint32_t w1) {
    auto two = [](uint32_t w, uint32_t& a, uint32_t& b) {
        uint32_t lo, hi, x, y;
        asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(lo) : "r"(w), "r"(0x0F0F0F0Fu), "r"(0x08080808u));
        asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(hi) : "r"(w >> 4), "r"(0x0F0F0F0Fu), "r"(0x08080808u));
        lo = (lo + 0x78787878u) ^ 0x80808080u;
        hi = (hi + 0x78787878u) ^ 0x80808080u;
        asm("prmt.b32 %0, %1, %2, 0x5140;" : "=r"(x) : "r"(lo), "r"(hi));
        asm("prmt.b32 %0, %1, %2, 0x7362;" : "=r"(y) : "r"(lo), "r"(hi));
        a = x;
        b = y;
    };
    uint4 r;
    two(w0, r.x, r.y);
    two(w1, r.z, r.w);
    return r;
}

template <int A>
__global__ void __launch_bounds__(kThreads, 1)
doa_cov_kernel(const __grid_constant__ CUtensorMap vmap, const CovParams p) {
    constexpr uint32_t RAW = kTile * 2 * A;              // [row][2 channels][A]
    constexpr uint32_t IDESC = idesc_s8_s32_mn(128, 128);
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* xs = smem;                                  // kXStages x 2 x 16 KiB
    uint8_t* raw = smem + kXStages * kXBytes;            // kRawStages x RAW
    uint64_t* bars = reinterpret_cast<uint64_t*>(raw + kRawStages * RAW);
    uint64_t* raw_full = bars;                           // [kRawStages]
    uint64_t* raw_empty = bars + kRawStages;             // [kRawStages]
    uint64_t* x_full = bars + 2 * kRawStages;            // [kXStages]
    uint64_t* x_empty = x_full + kXStages;               // [kXStages]
    uint64_t* acc_full = x_empty + kXStages;             // [2]
    uint64_t* acc_empty = acc_full + 2;                  // [2]
    uint64_t* mma_done = acc_empty + 2;
    uint32_t* tmem_ptr = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* s_fail = reinterpret_cast<volatile int*>(mma_done + 2);

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
    } else if (warp < 2 + kUnpackWarps) {
        const int ut = threadIdx.x - 64;  // 0 .. 32 * kUnpackWarps - 1
        int stage = 0, xst = 0;
        uint32_t phase = 0, xph = 0;
        bool stop = false;
        constexpr int kChunks = A / 8;   // 8-antenna chunks per spectrum
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            for (int k = 0; k < p.tiles_per_block; ++k) {
                if (*s_fail) { stop = true; break; }
                if (!mbar_wait(&raw_full[stage], phase, kWaitNs)) { fail(32); stop = true; break; }
                if (!mbar_wait(&x_empty[xst], xph ^ 1, kWaitNs)) { fail(64); stop = true; break; }
                const uint8_t* rsrc = raw + stage * RAW;
                uint8_t* xdst = xs + xst * kXBytes;
                for (int idx = ut; idx < 2 * kTile * 8; idx += 32 * kUnpackWarps) {
                    const int ch = idx >> 10, r = (idx >> 3) & (kTile - 1), c = idx & 7;  // channel, spectrum, chunk
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (c < kChunks) {
                        const uint2 w = *reinterpret_cast<const uint2*>(rsrc + (r * 2 + ch) * A + c * 8);
                        v = expand8(w.x, w.y);
                    }
                    *reinterpret_cast<uint4*>(xdst + ch * (kTile * 128) + r * 128 + ((c ^ (r & 7)) << 4)) = v;
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&raw_empty[stage]);
                    mbar_arrive(&x_full[xst]);
                }
                if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                if (++xst == kXStages) { xst = 0; xph ^= 1; }
            }
        }
    } else {
        const int q4 = warp & 3;
        const int m = 32 * q4 + lane;       // component row of G
        const int i = m >> 1, comp = m & 1; // antenna, 0 = re / 1 = im part of R
        int ast = 0;
        uint32_t aph = 0;
        bool stop = false;
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            if (!mbar_wait(&acc_full[ast], aph, kWaitNs)) { fail(128); break; }
            tc_fence_after();
            const int b = static_cast<int>(u / p.n_pairs), fp = static_cast<int>(u % p.n_pairs);
#pragma unroll 1
            for (int ch = 0; ch < 2; ++ch) {
                const int f = 2 * fp + ch;
                if (f >= p.n_freq) break;
                int32_t* row = p.out + ((static_cast<size_t>(b) * p.n_freq + f) * A + i) * A * 2;
                const uint32_t taddr = tmem_base + ((32u * q4) << 16) + ast * 256 + ch * 128;
#pragma unroll 1
                for (int c = 0; c < 4; ++c) {
                    uint32_t g[32];
                    tmem_ld_32x32b_x32(taddr + 32 * c, g);
                    tmem_ld_wait();
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int j = 16 * c + jj;
                        const int32_t own = static_cast<int32_t>(g[2 * jj]);
                        const int32_t recv = __shfl_xor_sync(0xffffffffu, static_cast<int32_t>(g[2 * jj + 1]), 1);
                        const int32_t val = comp == 0 ? own + recv : own - recv;
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
    const size_t smem = std::max<size_t>(kXStages * kXBytes + kRawStages * kTile * 2 * A + 256 + 1024, 120 * 1024);
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
    if (block_len > (1ull << 24) || d.n_time >= (1ull << 31)) {
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
    p.err = device_error_word();
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
