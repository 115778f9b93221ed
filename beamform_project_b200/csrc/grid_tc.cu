// grid_tc.cu -- split-precision tcgen05 fixed-grid beamformer (sm_100a).
//
// Same product as the reference's fused grid path (launch_packed_integrated_
// beamformer + launch_quantize_integrated_intensity, reference
// src/cuda_beamformer.cu:488-543 and src/cuda_quantize_int8.cu:132-147):
//   I[w][f][b] = sum_{t in window w} | sum_a w[b][f][a] * x[t][f][a] |^2
// with the weights used as stored (no conjugate), windows of S spectra and a
// partial last window, then int8 chunk quantization.
//
// Formulation.  Per channel the complex contraction is one real GEMM
//   D[t][n] = sum_k X[t][k] * Wop[n][k],   M = time, K = 2A, N = 2B,
// where k enumerates (re, im) of every antenna and n = 2b + (0: re, 1: im)
// of every beam.  Voltages are exact in fp16; each weight coefficient is an
// fp16 pair hi + lo with hi = fp16(w), lo = fp16(w - hi), and both products
// accumulate into the same fp32 TMEM accumulator, so D carries about 22 bits
// of weight precision.  |.|^2 and the time integration run in the epilogue.
//
// CTA organisation (one persistent CTA per SM, 12 warps):
//   warp 0      TMA producer: raw voltage tiles (128 spectra x A bytes of one
//               channel, 4-D tensor map, zero fill past T; four quadrant boxes
//               of R rows for windows below 32 spectra) and the channel's
//               prepared weight image (1-D bulk copies).
//   warp 1      TMEM owner and MMA issuer (one thread): 2 x K/16
//               tcgen05.mma (M=128, N=2B, K=16) per tile, hi then lo.
//   unpack      raw int4 bytes -> fp16 in the 128-byte-swizzled K-major
//               layout the MMA reads (two LOP3s + one half2 op per value
//               pair; the K order follows the decode and the prepared
//               weights follow it): warps 2-3 (2-7 for 16 beams).  At 128
//               and 256 antennas warps 4-7, one per TMEM lane quadrant, write
//               the fp16 tile into TMEM instead and the MMAs read A there.
//   epilogue    the remaining warps, a multiple of four: TMEM -> registers
//               (tcgen05.ld 32x32b), power per (spectrum, beam), then either
//               a butterfly reduce-scatter over each warp's 32 spectra into
//               running per-window sums (S >= 32) or a staging tile summed per
//               (window, beam) inside the warp's lane quadrant (S < 32), and
//               window totals over the four quadrants in a fixed order.
// Pipelines: 2 raw stages (4 at 128 antennas), 2 fp16 stages, 2 TMEM
// accumulators, all mbarrier driven; every wait is bounded and records an
// error code instead of hanging.
//
// Work split: units are (shard, channel, group of G tiles) with G tiles =
// lcm(128, S) spectra (a tile of 4 x R rows, R = 32 / S * S, below 32), so no
// integration window crosses a unit; each CTA takes a contiguous range of
// units (few channel switches, so few weight loads).  S is below 32 or a
// multiple of 32, so a window never straddles a warp's 32 spectra.
#include "bf_internal.cuh"
#include "grid_tc.cuh"
#include "sm100.cuh"

#include <cuda.h>
#include <cuda_fp16.h>

#include <climits>
#include <mutex>

namespace bf {

__device__ unsigned int g_tc_error = 0;

namespace {

using namespace sm100;

constexpr int kThreads = 384;             // 4 control / unpack warps + 8 epilogue warps
constexpr int kEpilogueThreads = 256;
constexpr int kTileM = 128;
constexpr int kRing = 8;                  // window partial-sum slots
constexpr uint32_t kMaxDynamicSmem = 232448;  // per CTA on sm_100
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s bound on any wait
constexpr int kMaxRawStages = 4;

struct TcParams {
    TcJob job;                  // plain launches
    const TcTableHeader* table; // served launches
    int8_t* codes;              // [shard][W][F][B] or null (no fused quantization)
    float2* params;             // [shard][W][ftiles][btiles]
    unsigned* counters;         // [shard][W][ftiles] arrival counts, zero at launch
    int ftiles, btiles;
    int paired;                 // plain launch: CTA pairs share channel pairs (see JobCursor)
    long long n_units;
    // plain launch over a device-written list of units (the checked
    // covariance form's fallback): *unit_count entries of unit_list
    const int* unit_list;
    const int* unit_count;
};

// Index i of a CTA's range is unit i, or unit_list[i] in a list launch.
__device__ __forceinline__ long long unit_at(const TcParams& p, long long i) {
    return p.unit_list != nullptr ? static_cast<long long>(p.unit_list[i]) : i;
}


__device__ __forceinline__ void record_error(unsigned code) { atomicOr(&g_tc_error, code); }

// Decode one packed word (4 antennas) into the 8 fp16 K values of its slot:
// [re a0, re a2, im a0, im a2, re a1, re a3, im a1, im a3].
__device__ __forceinline__ uint4 decode4(uint32_t w) {
    const uint32_t w1 = w >> 8;
    uint32_t t0, t1, t2, t3;
    asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(t0) : "r"(w), "r"(0x000F000Fu), "r"(0x64086408u));
    asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(t1) : "r"(w), "r"(0x00F000F0u), "r"(0x64806480u));
    asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(t2) : "r"(w1), "r"(0x000F000Fu), "r"(0x64086408u));
    asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(t3) : "r"(w1), "r"(0x00F000F0u), "r"(0x64806480u));
    const __half2 bias_lo = __float2half2_rn(1032.0f);
    const __half2 sixteenth = __float2half2_rn(0.0625f);
    const __half2 bias_hi = __float2half2_rn(-72.0f);
    __half2 h0 = __hsub2(*reinterpret_cast<__half2*>(&t0), bias_lo);
    __half2 h1 = __hfma2(*reinterpret_cast<__half2*>(&t1), sixteenth, bias_hi);
    __half2 h2 = __hsub2(*reinterpret_cast<__half2*>(&t2), bias_lo);
    __half2 h3 = __hfma2(*reinterpret_cast<__half2*>(&t3), sixteenth, bias_hi);
    uint4 r;
    r.x = *reinterpret_cast<uint32_t*>(&h0);
    r.y = *reinterpret_cast<uint32_t*>(&h1);
    r.z = *reinterpret_cast<uint32_t*>(&h2);
    r.w = *reinterpret_cast<uint32_t*>(&h3);
    return r;
}

// 32 accumulator columns of this lane's spectrum = (re, im) of 16 beams.
// Returns the power summed over the warp's 32 spectra for beam (lane >> 1):
// |.|^2 per beam, then a butterfly reduce-scatter (16 shuffles in all) that
// leaves the sum for beam m in lanes 2m and 2m + 1.
__device__ __forceinline__ float beam_pair_sum(const uint32_t (&r)[32], int lane) {
    float v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const float re = __uint_as_float(r[2 * j]), im = __uint_as_float(r[2 * j + 1]);
        v[j] = re * re + im * im;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const bool up = lane & 16;
        const float send = up ? v[i] : v[i + 8];
        const float keep = up ? v[i + 8] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const bool up = lane & 8;
        const float send = up ? v[i] : v[i + 4];
        const float keep = up ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const bool up = lane & 4;
        const float send = up ? v[i] : v[i + 2];
        const float keep = up ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {
        const bool up = lane & 2;
        const float send = up ? v[0] : v[1];
        const float keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

struct Unit {
    int shard, f, tile_begin, tile_end;
    int key;  // (job, shard, channel): identifies the weight image
};

// Walks the units of a CTA's contiguous range in order, tracking which job
// each belongs to (a plain launch has the single job p.job).
template <bool kServed>
struct JobCursor {
    const TcJob* jobs = nullptr;
    int n_jobs = 1, j = 0;
    long long next_begin = 0;  // unit_begin of job j + 1
    TcJob jb;

    __device__ __forceinline__ void init(const TcParams& p, long long u) {
        if constexpr (kServed) {
            jobs = reinterpret_cast<const TcJob*>(p.table + 1);
            n_jobs = p.table->n_jobs;
            int lo = 0, hi = n_jobs - 1;  // last job with unit_begin <= u
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (jobs[mid].unit_begin <= u) lo = mid; else hi = mid - 1;
            }
            j = lo;
            jb = jobs[j];
            next_begin = j + 1 < n_jobs ? jobs[j + 1].unit_begin : LLONG_MAX;
        } else {
            jb = p.job;
            next_begin = LLONG_MAX;
        }
    }
    // Paired order (plain launches with an even channel count): CTAs 2m and
    // 2m + 1 walk the same (channel pair, group) sequence, taking the even and
    // the odd channel of each pair, so the two 64-byte halves of every
    // 128-byte voltage line are read at about the same time and DRAM fetches
    // each line once.  u then counts (shard, channel pair, group).
    int pair_parity = -1;

    // The decomposition of the last unit returned: every role walks its range
    // one unit at a time, so the next unit comes from a carry chain instead of
    // four 64-bit divisions (a full decode only at a job change or a jump).
    long long last_u = -2;
    int d_shard = 0, d_ch = 0, d_g = 0;  // d_ch: channel, or channel pair when paired

    __device__ __forceinline__ Unit at(long long u) {
        bool full = u != last_u + 1;
        if constexpr (kServed) {
            while (u >= next_begin) {
                ++j;
                jb = jobs[j];
                next_begin = j + 1 < n_jobs ? jobs[j + 1].unit_begin : LLONG_MAX;
                full = true;
            }
        }
        const int chans = pair_parity >= 0 ? jb.n_freq / 2 : jb.n_freq;
        if (u == last_u && !full) {
            // same unit again
        } else if (!full) {
            if (++d_g == jb.groups_per_channel) {
                d_g = 0;
                if (++d_ch == chans) {
                    d_ch = 0;
                    ++d_shard;
                }
            }
        } else {
            const long long local = u - (kServed ? jb.unit_begin : 0);
            const long long per_shard = static_cast<long long>(chans) * jb.groups_per_channel;
            d_shard = static_cast<int>(local / per_shard);
            const long long rem = local % per_shard;
            d_ch = static_cast<int>(rem / jb.groups_per_channel);
            d_g = static_cast<int>(rem % jb.groups_per_channel);
        }
        last_u = u;
        Unit r;
        r.shard = d_shard;
        r.f = pair_parity >= 0 ? 2 * d_ch + pair_parity : d_ch;
        r.tile_begin = d_g * jb.group_tiles;
        r.tile_end = min(r.tile_begin + jb.group_tiles, jb.tiles_per_channel);
        r.key = (j << 16) + r.shard * jb.n_freq + r.f;
        return r;
    }
};

// ---------------- fused quantization bookkeeping (epilogue thread 0) ----------
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* addr, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(addr), "r"(v) : "memory");
    return old;
}

// Counter bumps issued for the windows finalized in one tile (all of one
// (shard, channel) unit); windows w0 + i for the bits i of mask.
struct Pending {
    unsigned old[8];
    unsigned mask;
    int w0, shard, fg;
    unsigned group;
};

// Record the windows finalized in a tile (no memory traffic yet).
__device__ __forceinline__ void record_finalized(const TcParams& p, const Unit& un, int first_row, int tile_end_row,
                                                 Pending& pd) {
    const TcJob& jb = p.job;
    pd.mask = 0;
    if (first_row >= jb.n_time) return;
    pd.w0 = first_row / jb.spectra;
    pd.shard = un.shard;
    pd.fg = un.f / 16;
    pd.group = static_cast<unsigned>(min(16, jb.n_freq - 16 * pd.fg));
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int w = pd.w0 + i;
        const int w_last = min((w + 1) * jb.spectra, jb.n_time) - 1;
        if (w < jb.n_windows && w_last >= first_row && w_last < tile_end_row) pd.mask |= 1u << i;
    }
}

// Bump the counters of recorded windows (acq_rel at GPU scope: releases this
// CTA's stores of those windows, acquires the other CTAs' when last).
__device__ __forceinline__ void issue_arrivals(const TcParams& p, const Pending& rec, Pending& pd) {
    pd = rec;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if ((rec.mask >> i) & 1u) {
            const size_t ci = (static_cast<size_t>(rec.shard) * p.job.n_windows + rec.w0 + i) * p.ftiles + rec.fg;
            pd.old[i] = atom_add_acq_rel_gpu(&p.counters[ci], 1u);
        }
    }
}

// Publish the windows whose group this CTA completed (bump result == group - 1).
__device__ __forceinline__ void publish_ready(Pending& pd, volatile int* s_quant, volatile int* s_meta) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int w = -1;
        if (((pd.mask >> i) & 1u) && pd.old[i] + 1 == pd.group) w = pd.w0 + i;
        s_quant[i] = w;
    }
    s_meta[0] = pd.shard;
    s_meta[1] = pd.fg;
    pd.mask = 0;
}

// All epilogue threads: quantize every published window's chunks (one warp per
// 16-beam chunk).  The integrated values of the other CTAs were released by
// their bumps and acquired by ours; they are read through L2.
__device__ __forceinline__ void quantize_ready(const TcParams& p, volatile int* s_quant, volatile int* s_meta,
                                               int et, int lane, int epi_warps) {
    const TcJob& jb = p.job;
    const int shard = s_meta[0], fg = s_meta[1];
    for (int i = 0; i < 8; ++i) {
        const int w = s_quant[i];
        if (w < 0) continue;
        const size_t shard_off = static_cast<size_t>(shard) * jb.n_windows * jb.n_freq * jb.n_beams;
        for (int bt = et >> 5; bt < p.btiles; bt += epi_warps) {
            const size_t pidx = ((static_cast<size_t>(shard) * jb.n_windows + w) * p.ftiles + fg) * p.btiles + bt;
            quantize_chunk<true>(jb.integrated + shard_off, p.codes + shard_off, p.params, pidx, w, jb.n_freq,
                                 jb.n_beams, fg, bt, lane);
        }
    }
}

// Shared-memory plan (offsets from a 1024-aligned base).
struct Smem {
    uint32_t w_bytes = 0;    // one of hi / lo
    uint32_t w_stages = 1;   // weight images in flight (2 when they fit)
    uint32_t x_bytes = 0;    // one fp16 stage
    uint32_t raw_bytes = 0;  // one raw stage
    uint32_t raw_stages = 2;
    uint32_t off_w = 0, off_x = 0, off_raw = 0, off_slots = 0, off_bar = 0, total = 0;
};

__host__ __device__ constexpr Smem smem_plan(int n_ant, int n_beams_pad, bool served) {
    Smem s{};
    const uint32_t K = 2 * n_ant, N = 2 * n_beams_pad;
    s.w_bytes = (K / 64) * N * 128;
    // at 128 antennas the fp16 voltage operand is written to TMEM instead
    s.x_bytes = n_ant >= 128 ? 0 : (K / 64) * kTileM * 128;
    s.raw_bytes = kTileM * n_ant;
    // with the voltage operand in TMEM the shared memory has room for more raw
    // tiles in flight, which the short MMAs of small beam groups need
    s.raw_stages = n_ant == 128 ? kMaxRawStages : 2;
    // window partial sums (S >= 32) or the per-warp power staging of short
    // windows ([8 warps][16 beams][33] floats), which share the space
    const uint32_t ring = kRing * 4 * n_beams_pad * 4, staging = (kEpilogueThreads / 32) * 16 * 33 * 4;
    const uint32_t rest = 2 * s.x_bytes + s.raw_stages * s.raw_bytes + (ring > staging ? ring : staging) + 256;
    // A second weight image lets the next channel's weights load while the
    // MMAs of the current one run.  Served units (one window, a few tiles)
    // switch channel at every unit; measured per served class on a B200, the
    // second image helps at 64 antennas and up to 32 beams (-8 to -15 %
    // window time) and costs at 32 antennas (+6 to +20 %: the smaller image
    // loads quickly, and the space is lost to L1); plain launches switch
    // rarely.
    const bool two = served && n_ant == 64 && n_beams_pad <= 32;
    s.w_stages = two && 4 * s.w_bytes + rest + 1024 <= kMaxDynamicSmem ? 2 : 1;
    s.off_w = 0;
    s.off_x = s.off_w + s.w_stages * 2 * s.w_bytes;
    s.off_raw = s.off_x + 2 * s.x_bytes;
    s.off_slots = s.off_raw + s.raw_stages * s.raw_bytes;
    s.off_bar = s.off_slots + (ring > staging ? ring : staging);
    s.total = s.off_bar + 256;
    return s;
}

template <int A, int NB, bool kServed>  // A antennas, NB padded beams (multiple of 16)
__global__ void __launch_bounds__(kThreads, 1)
grid_tensor_kernel(const __grid_constant__ CUtensorMap vmap, const TcParams p) {
    constexpr int K = 2 * A;
    constexpr int N = 2 * NB;
    constexpr uint32_t ACC_COLS = N;          // fp32 columns per accumulator
    // At 128 and 256 antennas the fp16 voltage tile (128 rows x K, 64 or
    // 128 KB) lives in TMEM after the two accumulators, K / 2 columns per
    // stage (two stages at 128 antennas, one at 256): the unpack warps write
    // it with tcgen05.st (a warp reaches one lane quadrant, so four unpack
    // warps cover the 128 rows) and the MMAs read A from TMEM, which leaves
    // the shared memory to the weight images of up to 64 (32) beams.
    constexpr bool kTmemA = A >= 128;
    constexpr int kXStages = A == 256 ? 1 : 2;
    constexpr int kHalvesA = A >= 128 ? A / 128 : 1;   // 128-byte halves of a raw row
    constexpr uint32_t A_COL0 = 2 * ACC_COLS;
    static_assert(!kTmemA || A_COL0 + kXStages * (K / 2) <= 512, "TMEM holds two accumulators and the voltage");
    constexpr uint32_t TMEM_COLS = kTmemA ? 512 : (2 * N <= 32) ? 32 : (2 * N <= 64) ? 64 : (2 * N <= 128) ? 128
                                   : (2 * N <= 256) ? 256 : 512;
    constexpr uint32_t IDESC = idesc_f16_f32(kTileM, N);
    constexpr Smem S = smem_plan(A, NB, kServed);
    // Warp roles: 0 producer, 1 MMA, then unpack warps, then epilogue warps
    // (a multiple of four, so epilogue warp w reads TMEM lane quadrant w % 4).
    // The narrowest beam set (one 32-column load per quadrant) has little
    // epilogue work and is unpack-bound, so it trades four epilogue warps for
    // unpack warps (measured: at 32 beams the epilogue would then bind).
    // With the voltage in TMEM: warps 2 and 3 idle, unpack warps 4-7 (one
    // per lane quadrant), epilogue warps 8-11.
    constexpr int kUnpackWarps = kTmemA ? 4 : NB <= 16 ? 6 : 2;
    constexpr int kUnpackFirst = kTmemA ? 4 : 2;
    constexpr int kEpiWarps = kThreads / 32 - kUnpackFirst - kUnpackWarps;   // 4 or 8
    constexpr int kEpiThreads = 32 * kEpiWarps;
    constexpr int kEpiFirstWarp = kUnpackFirst + kUnpackWarps;
    static_assert(kEpiWarps % 4 == 0 && kEpiFirstWarp % 4 == 0, "epilogue warps cover whole lane quadrants");

    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* w_img = smem + S.off_w;   // [w_stages][hi | lo]
    uint8_t* xs = smem + S.off_x;
    uint8_t* raw = smem + S.off_raw;
    float* slots = reinterpret_cast<float*>(smem + S.off_slots);   // [kRing][4][NB] or staging
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S.off_bar);
    constexpr int kRawStages = static_cast<int>(S.raw_stages);
    uint64_t* raw_full = bars + 0;    // [kRawStages]
    uint64_t* raw_empty = bars + 4;   // [kRawStages]
    uint64_t* x_full = bars + 8;      // [2]
    uint64_t* x_empty = bars + 10;    // [2]
    uint64_t* acc_full = bars + 12;   // [2]
    uint64_t* acc_empty = bars + 14;  // [2]
    uint64_t* w_full = bars + 16;     // [w_stages]
    uint64_t* w_empty = bars + 18;    // [w_stages]
    uint64_t* mma_done = bars + 20;
    uint32_t* tmem_ptr = reinterpret_cast<uint32_t*>(bars + 22);
    volatile int* s_fail = reinterpret_cast<volatile int*>(bars + 23);
    volatile int* s_quant = reinterpret_cast<volatile int*>(bars + 24);  // [8] windows to quantize
    volatile int* s_meta = reinterpret_cast<volatile int*>(bars + 28);   // [2] their shard, channel group
    static_assert(kRawStages <= kMaxRawStages && 29 * 8 <= 256, "barrier block");
    // A list launch with an empty list (the checked form's common case) ends
    // before any set-up; every thread reads the same count.
    if (!kServed && p.unit_list != nullptr && *p.unit_count == 0) return;
    Pending pend, recorded;                                               // epilogue thread 0 only
    pend.mask = 0;
    recorded.mask = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 8; ++i) s_quant[i] = -1;
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kRawStages; ++i) {
            mbar_init(&raw_full[i], 1);
            mbar_init(&raw_empty[i], kUnpackWarps);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&x_full[i], kUnpackWarps);
            mbar_init(&x_empty[i], 1);
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], kEpiWarps);
        }
        for (uint32_t i = 0; i < S.w_stages; ++i) {
            mbar_init(&w_full[i], 1);
            mbar_init(&w_empty[i], 1);
        }
        mbar_init(mma_done, 1);
        *s_fail = 0;
        fence_mbar_init();
    }
    for (int i = threadIdx.x; i < kRing * 4 * NB; i += kThreads) slots[i] = 0.f;
    if (warp == 1) tmem_alloc(tmem_ptr, TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_ptr;

    long long n_units = p.n_units;
    if constexpr (kServed) n_units = p.table->n_units;
    if (!kServed && p.unit_list != nullptr) n_units = *p.unit_count;
    long long u_begin = n_units * blockIdx.x / gridDim.x;
    long long u_end = n_units * (blockIdx.x + 1) / gridDim.x;
    int pair_parity = -1;
    if (!kServed && p.paired) {  // host guarantees an even channel count and grid
        const long long pair_units = n_units / 2;
        const int slots = static_cast<int>(gridDim.x / 2), m = static_cast<int>(blockIdx.x / 2);
        u_begin = pair_units * m / slots;
        u_end = pair_units * (m + 1) / slots;
        pair_parity = static_cast<int>(blockIdx.x & 1);
    }
    // A failed (timed-out) wait records its code, raises the CTA-wide flag and
    // makes every role stop at its next check; nothing waits unboundedly.
    auto fail = [&](unsigned code) {
        record_error(code);
        *s_fail = 1;
    };

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int armed[kRawStages];     // parity of the last load issued per raw stage
#pragma unroll
            for (int i = 0; i < kRawStages; ++i) armed[i] = -1;
            uint32_t w_loads = 0;      // weight images loaded; image i goes to stage i % w_stages
            uint32_t w_uses[2] = {0, 0};
            int prev_key = -1;
            bool stop = false;
            JobCursor<kServed> cur;
            if (u_begin < u_end) cur.init(p, u_begin);
            cur.pair_parity = pair_parity;
            for (long long u = u_begin; u < u_end && !stop; ++u) {
                const Unit un = cur.at(unit_at(p, u));
                const TcJob& jb = cur.jb;
                if (un.key != prev_key) {
                    const uint32_t ws = w_loads % S.w_stages;
                    // the stage's previous image must be done with (its n-th
                    // reuse waits for the n-th release, parity (n - 1) & 1)
                    if (w_uses[ws] > 0) {
                        if (!mbar_wait(&w_empty[ws], (w_uses[ws] - 1) & 1, kWaitNs)) { fail(1); break; }
                    }
                    mbar_expect_tx(&w_full[ws], 2 * S.w_bytes);
                    const uint8_t* src =
                        jb.split + static_cast<size_t>(un.shard * jb.n_freq + un.f) * 2 * S.w_bytes;
                    uint8_t* dst = w_img + ws * 2 * S.w_bytes;
                    constexpr uint32_t kChunk = 32768;
                    for (uint32_t off = 0; off < 2 * S.w_bytes; off += kChunk) {
                        const uint32_t n = min(kChunk, 2 * S.w_bytes - off);
                        bulk_g2s(dst + off, src + off, n, &w_full[ws]);
                    }
                    ++w_uses[ws];
                    ++w_loads;
                    prev_key = un.key;
                }
                const int R = jb.rows_q;
                for (int k = un.tile_begin; k < un.tile_end; ++k) {
                    if (*s_fail) { stop = true; break; }
                    if (!mbar_wait(&raw_empty[stage], phase ^ 1, kWaitNs)) { fail(2); stop = true; break; }
                    uint8_t* dst = raw + stage * S.raw_bytes;
                    if constexpr (kTmemA) {
                        // [half][128 rows][128 bytes], 128-byte swizzled boxes of 128 antennas
                        mbar_expect_tx(&raw_full[stage], R == 32 ? S.raw_bytes : 4 * R * A);
#pragma unroll
                        for (int h = 0; h < kHalvesA; ++h) {
                            uint8_t* dh = dst + h * (kTileM * 128);
                            if (R == 32) {
                                tma_load_4d(dh, &vmap, 128 * h, un.f, jb.t0 + k * kTileM, un.shard, &raw_full[stage]);
                            } else {
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    tma_load_4d(dh + q * 32 * 128, &vmap, 128 * h, un.f, jb.t0 + (4 * k + q) * R,
                                                un.shard, &raw_full[stage]);
                                }
                            }
                        }
                    } else if (R == 32) {
                        mbar_expect_tx(&raw_full[stage], S.raw_bytes);
                        tma_load_4d(dst, &vmap, 0, un.f, jb.t0 + k * kTileM, un.shard, &raw_full[stage]);
                    } else {
                        // four R-row boxes, one at the start of each lane quadrant
                        mbar_expect_tx(&raw_full[stage], 4 * R * A);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            tma_load_4d(dst + q * 32 * A, &vmap, 0, un.f, jb.t0 + (4 * k + q) * R, un.shard,
                                        &raw_full[stage]);
                        }
                    }
                    armed[stage] = static_cast<int>(phase);
                    if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                }
            }
            // let every copy this thread issued land before the CTA can exit
            for (int s = 0; s < kRawStages; ++s) {
                if (armed[s] >= 0 && !mbar_wait(&raw_full[s], static_cast<uint32_t>(armed[s]), kWaitNs)) fail(256);
            }
            for (uint32_t ws = 0; ws < S.w_stages; ++ws) {
                if (w_uses[ws] > 0 && !mbar_wait(&w_full[ws], (w_uses[ws] - 1) & 1, kWaitNs)) fail(512);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int xs_stage = 0, acc_stage = 0;
            uint32_t x_phase = 0, acc_phase = 0;
            uint32_t w_switches = 0, w_seen[2] = {0, 0}, ws = 0;
            int prev_key = -1;
            bool stop = false;
            uint32_t w_hi_addr = smem_u32(w_img), w_lo_addr = w_hi_addr + S.w_bytes;
            JobCursor<kServed> cur;
            if (u_begin < u_end) cur.init(p, u_begin);
            cur.pair_parity = pair_parity;
            for (long long u = u_begin; u < u_end && !stop; ++u) {
                const Unit un = cur.at(unit_at(p, u));
                if (un.key != prev_key) {
                    ws = w_switches % S.w_stages;
                    if (!mbar_wait(&w_full[ws], w_seen[ws] & 1, kWaitNs)) { fail(4); break; }
                    ++w_seen[ws];
                    ++w_switches;
                    w_hi_addr = smem_u32(w_img + ws * 2 * S.w_bytes);
                    w_lo_addr = w_hi_addr + S.w_bytes;
                    prev_key = un.key;
                }
                bool next_switches = true;
                if (u + 1 < u_end) {
                    JobCursor<kServed> ahead = cur;
                    next_switches = ahead.at(unit_at(p, u + 1)).key != un.key;
                }
                for (int k = un.tile_begin; k < un.tile_end; ++k) {
                    if (*s_fail) { stop = true; break; }
                    if (!mbar_wait(&x_full[xs_stage], x_phase, kWaitNs)) { fail(8); stop = true; break; }
                    if (!mbar_wait(&acc_empty[acc_stage], acc_phase ^ 1, kWaitNs)) { fail(16); stop = true; break; }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + acc_stage * ACC_COLS;
                    // descriptors once per tile; the start address field (bits 0-13,
                    // 16-byte units) then advances by plain adds (shared addresses stay
                    // below 2^18 bytes, so the field never carries)
                    const uint64_t a0 = kTmemA ? 0 : smem_desc_sw128(smem_u32(xs + xs_stage * S.x_bytes));
                    const uint32_t a_t = tmem_base + A_COL0 + xs_stage * (K / 2);  // voltage stage in TMEM
                    const uint64_t bh0 = smem_desc_sw128(w_hi_addr), bl0 = smem_desc_sw128(w_lo_addr);
#pragma unroll
                    for (int kk = 0; kk < K / 16; ++kk) {
                        const uint32_t kb = kk / 4, koff = (kk % 4) * 32;
                        const uint64_t a = a0 + ((kb * (kTileM * 128) + koff) >> 4);
                        const uint64_t bh = bh0 + ((kb * (N * 128) + koff) >> 4);
                        const uint64_t bl = bl0 + ((kb * (N * 128) + koff) >> 4);
                        if constexpr (kTmemA) {
                            // 16 K values = 8 columns of the TMEM voltage stage
                            mma_f16_ts(d_tmem, a_t + 8 * kk, bh, IDESC, kk > 0 ? 1u : 0u);
                            mma_f16_ts(d_tmem, a_t + 8 * kk, bl, IDESC, 1u);
                        } else {
                            mma_f16_ss(d_tmem, a, bh, IDESC, kk > 0 ? 1u : 0u);
                            mma_f16_ss(d_tmem, a, bl, IDESC, 1u);
                        }
                    }
                    tc_commit(&x_empty[xs_stage]);
                    tc_commit(&acc_full[acc_stage]);
                    if (k + 1 == un.tile_end && next_switches) tc_commit(&w_empty[ws]);
                    if (++xs_stage == kXStages) { xs_stage = 0; x_phase ^= 1; }
                    if (++acc_stage == 2) { acc_stage = 0; acc_phase ^= 1; }
                }
            }
            // every MMA this thread issued completes before TMEM is released
            tc_commit(mma_done);
            if (!mbar_wait(mma_done, 0, kWaitNs)) fail(1024);
        }
    } else if (warp < kUnpackFirst) {
        // idle (the TMEM voltage form places its unpack warps on lane quadrants 0-3)
    } else if (warp < kEpiFirstWarp) {
      if constexpr (kTmemA) {
        // ------------------------------------------------- unpack into TMEM
        // Thread = tile row 32 q4 + lane of this warp's lane quadrant: its raw
        // row (A bytes in 128-byte halves, each 128-byte swizzled by the TMA)
        // becomes K / 2 columns of fp16 pairs in K order (raw word i ->
        // columns 4 i .. 4 i + 3, the order decode4 and the prepared weights
        // share).
        const int q4 = warp & 3;
        const int r = 32 * q4 + lane;
        int stage = 0, xs_stage = 0;
        uint32_t phase = 0, x_phase = 0;
        bool stop = false;
        JobCursor<kServed> cur;
        if (u_begin < u_end) cur.init(p, u_begin);
        cur.pair_parity = pair_parity;
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            const Unit un = cur.at(unit_at(p, u));
            const bool zero = (r & 31) >= cur.jb.rows_q;  // spare quadrant rows of short windows
            for (int k = un.tile_begin; k < un.tile_end; ++k) {
                if (*s_fail) { stop = true; break; }
                if (!mbar_wait(&raw_full[stage], phase, kWaitNs)) { fail(32); stop = true; break; }
                if (!mbar_wait(&x_empty[xs_stage], x_phase ^ 1, kWaitNs)) { fail(64); stop = true; break; }
                tc_fence_after();  // the MMAs that read this TMEM stage are complete
                const uint8_t* row = raw + stage * S.raw_bytes + r * 128;
                const uint32_t tbase = tmem_base + ((32u * q4) << 16) + A_COL0 + xs_stage * (K / 2);
#pragma unroll
                for (int g4 = 0; g4 < A / 32; ++g4) {  // 32 columns: two 16-byte chunks of the row
                    uint32_t col[32];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = 2 * g4 + h;        // chunk c of the row: half c / 8, chunk c % 8 there
                        uint4 w4 = *reinterpret_cast<const uint4*>(row + (c >> 3) * (kTileM * 128) +
                                                                   (((c & 7) ^ (r & 7)) << 4));
                        if (zero) w4 = make_uint4(0u, 0u, 0u, 0u);
                        const uint32_t words[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const uint4 d4 = decode4(words[j]);
                            col[16 * h + 4 * j + 0] = d4.x;
                            col[16 * h + 4 * j + 1] = d4.y;
                            col[16 * h + 4 * j + 2] = d4.z;
                            col[16 * h + 4 * j + 3] = d4.w;
                        }
                    }
                    tmem_st_32x32b_x32(tbase + 32 * g4, col);
                }
                tmem_st_wait();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&raw_empty[stage]);
                    mbar_arrive(&x_full[xs_stage]);
                }
                if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                if (++xs_stage == kXStages) { xs_stage = 0; x_phase ^= 1; }
            }
        }
      } else {
        // ------------------------------------------------------------ unpack
        const int ut = threadIdx.x - 64;  // 0 .. 32 * kUnpackWarps - 1
        int stage = 0, xs_stage = 0;
        uint32_t phase = 0, x_phase = 0;
        bool stop = false;
        constexpr int kChunks = A / 16;  // 16-byte raw chunks per spectrum
        JobCursor<kServed> cur;
        if (u_begin < u_end) cur.init(p, u_begin);
        cur.pair_parity = pair_parity;
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            const Unit un = cur.at(unit_at(p, u));
            const int R = cur.jb.rows_q;
            for (int k = un.tile_begin; k < un.tile_end; ++k) {
                if (*s_fail) { stop = true; break; }
                if (!mbar_wait(&raw_full[stage], phase, kWaitNs)) { fail(32); stop = true; break; }
                if (!mbar_wait(&x_empty[xs_stage], x_phase ^ 1, kWaitNs)) { fail(64); stop = true; break; }
                const uint8_t* rsrc = raw + stage * S.raw_bytes;
                uint8_t* xdst = xs + xs_stage * S.x_bytes;
#pragma unroll 4
                for (int idx = ut; idx < kTileM * kChunks; idx += 32 * kUnpackWarps) {
                    const int r = idx / kChunks, q = idx % kChunks;
                    uint4 w4 = *reinterpret_cast<const uint4*>(rsrc + r * A + q * 16);
                    if ((r & 31) >= R) w4 = make_uint4(0u, 0u, 0u, 0u);  // spare quadrant rows
                    const uint32_t words[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int kslot = 4 * q + j;           // 16-byte K slot (8 values)
                        const int kb = kslot >> 3, c16 = kslot & 7;
                        uint8_t* dst = xdst + kb * (kTileM * 128) + r * 128 + ((c16 ^ (r & 7)) << 4);
                        *reinterpret_cast<uint4*>(dst) = decode4(words[j]);
                    }
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&raw_empty[stage]);
                    mbar_arrive(&x_full[xs_stage]);
                }
                if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                if (++xs_stage == 2) { xs_stage = 0; x_phase ^= 1; }
            }
        }
      }
    } else {
        // ------------------------------------------------------------ epilogue
        // Warp w reads TMEM lane quadrant w % 4 (32 tile rows) and, with eight
        // epilogue warps, one half of the accumulator columns (beams).
        const int q4 = warp & 3;
        constexpr int kHalves = kEpiWarps / 4;
        const int half = (warp - kEpiFirstWarp) >> 2;     // 0 .. kHalves - 1
        const int et = threadIdx.x - 32 * kEpiFirstWarp;  // 0 .. kEpiThreads - 1
        int acc_stage = 0;
        uint32_t acc_phase = 0;
        constexpr int kLoads = N / 32;                    // 16 beams per 32-column load
        constexpr int kHalfLoads = (kLoads + kHalves - 1) / kHalves;
        const int c_begin = half * kHalfLoads;
        const int c_count = min(kHalfLoads, kLoads - c_begin);
        float* stg = slots + (warp - kEpiFirstWarp) * 528;  // short windows: [16 beams][33]
        float acc[kHalfLoads];
#pragma unroll
        for (int c = 0; c < kHalfLoads; ++c) acc[c] = 0.f;
        int cur_win = -1;
        bool failed = false, stop = false;
        auto flush = [&](int w) {
            float* s = slots + ((w % kRing) * 4 + q4) * NB;
            if ((lane & 1) == 0) {
#pragma unroll
                for (int c = 0; c < kHalfLoads; ++c) {
                    if (c < c_count) s[16 * (c_begin + c) + (lane >> 1)] = acc[c];
                }
            }
#pragma unroll
            for (int c = 0; c < kHalfLoads; ++c) acc[c] = 0.f;
        };
        // Short windows (S < 32): every window lies inside one lane quadrant.
        // The 16 powers of each lane's spectrum go to the staging tile
        // [16 beams][33] (row pitch 33 floats: the stores of a beam and the
        // reads of a window both spread over the banks) and each lane sums a
        // (window, beam) pair of the quadrant, in increasing row order.  wq is
        // the quadrant's first window; the unit's window length sw and pair
        // count npairs (16 per window) are set once per unit.
        auto nwin_of = [](int npairs) { return npairs >> 4; };
        auto short_windows = [&](const uint32_t (&r)[32], int c, const TcJob& jb, const Unit& un, int wq, int sw,
                                 int npairs) {
            float* srow = stg + lane;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float re = __uint_as_float(r[2 * j]), im = __uint_as_float(r[2 * j + 1]);
                srow[j * 33] = re * re + im * im;
            }
            __syncwarp();
            const int b16 = 16 * (c_begin + c);
            const size_t row_base = static_cast<size_t>(un.shard) * jb.n_windows + jb.w0;
            // two pairs per lane at a time (p and p + 32), their sums interleaved;
            // a pair past the quadrant's reads the staging tile and is dropped
            for (int pb = 0; pb < npairs; pb += 64) {
                const int p0 = pb + lane, p1 = pb + 32 + lane;
                const int j0 = p0 & 15, j1 = p1 & 15;
                const int s0 = min(p0 >> 4, nwin_of(npairs) - 1), s1 = min(p1 >> 4, nwin_of(npairs) - 1);
                const float* x0 = stg + j0 * 33 + s0 * sw;
                const float* x1 = stg + j1 * 33 + s1 * sw;
                float sum0 = 0.f, sum1 = 0.f;
#pragma unroll 5
                for (int i = 0; i < sw; ++i) {
                    sum0 += x0[i];
                    sum1 += x1[i];
                }
                const int w0 = wq + s0, w1 = wq + s1;
                if (p0 < npairs && w0 * sw < jb.n_time && b16 + j0 < jb.n_beams) {
                    jb.integrated[((row_base + w0) * jb.n_freq + un.f) * jb.beam_stride + b16 + j0] = sum0;
                }
                if (p1 < npairs && w1 * sw < jb.n_time && b16 + j1 < jb.n_beams) {
                    jb.integrated[((row_base + w1) * jb.n_freq + un.f) * jb.beam_stride + b16 + j1] = sum1;
                }
            }
            __syncwarp();
        };
        JobCursor<kServed> cur;
        if (u_begin < u_end) cur.init(p, u_begin);
        cur.pair_parity = pair_parity;
        for (long long u = u_begin; u < u_end && !stop; ++u) {
            const Unit un = cur.at(unit_at(p, u));
            const TcJob& jb = cur.jb;
            const bool short_win = jb.spectra < 32;
            const int sw = jb.spectra, nwin = short_win ? jb.rows_q / sw : 0, npairs = nwin * 16;
            for (int k = un.tile_begin; k < un.tile_end; ++k) {
                if (!failed && !mbar_wait(&acc_full[acc_stage], acc_phase, kWaitNs)) { fail(128); failed = true; }
                tc_fence_after();
                const uint32_t taddr = tmem_base + ((32u * q4) << 16) + acc_stage * ACC_COLS + 32 * c_begin;
                if (short_win) {
                    const int sq = (4 * k + q4) * jb.rows_q;  // first spectrum of this quadrant
                    const int wq = (4 * k + q4) * nwin;         // its first window (rows_q = nwin * sw)
                    if (!failed && sq < jb.n_time && kHalfLoads % 2 == 0) {
                        // one load at a time: with two loads in flight beside the
                        // staging sums, two loads per half spilled registers and
                        // four ran 2-3 % slower (three stay faster paired)
#pragma unroll 1
                        for (int c = 0; c < c_count; ++c) {
                            uint32_t r0[32];
                            tmem_ld_32x32b_x32(taddr + 32 * c, r0);
                            tmem_ld_wait();
                            short_windows(r0, c, jb, un, wq, sw, npairs);
                        }
                    } else if (!failed && sq < jb.n_time) {
#pragma unroll
                        for (int c = 0; c < kHalfLoads; c += 2) {
                            uint32_t r0[32];
                            if (c < c_count) tmem_ld_32x32b_x32(taddr + 32 * c, r0);
                            if constexpr (kHalfLoads > 1) {
                                uint32_t r1[32];
                                if (c + 1 < c_count) tmem_ld_32x32b_x32(taddr + 32 * (c + 1), r1);
                                tmem_ld_wait();
                                if (c < c_count) short_windows(r0, c, jb, un, wq, sw, npairs);
                                if (c + 1 < c_count) short_windows(r1, c + 1, jb, un, wq, sw, npairs);
                            } else {
                                tmem_ld_wait();
                                if (c < c_count) short_windows(r0, c, jb, un, wq, sw, npairs);
                            }
                        }
                    }
                } else {
                    const int row0 = k * kTileM + 32 * q4;
                    const int my_win = row0 < jb.n_time ? row0 / jb.spectra : -1;
                    if (my_win != cur_win && cur_win >= 0) { flush(cur_win); cur_win = -1; }
                    if (my_win >= 0 && !failed) {
#pragma unroll
                        for (int c = 0; c < kHalfLoads; c += 2) {
                            // two loads in flight per wait
                            uint32_t r0[32];
                            if (c < c_count) tmem_ld_32x32b_x32(taddr + 32 * c, r0);
                            if constexpr (kHalfLoads > 1) {
                                uint32_t r1[32];
                                if (c + 1 < c_count) tmem_ld_32x32b_x32(taddr + 32 * (c + 1), r1);
                                tmem_ld_wait();
                                if (c < c_count) acc[c] += beam_pair_sum(r0, lane);
                                if (c + 1 < c_count) acc[c + 1] += beam_pair_sum(r1, lane);
                            } else {
                                tmem_ld_wait();
                                if (c < c_count) acc[c] += beam_pair_sum(r0, lane);
                            }
                        }
                        cur_win = my_win;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0 && !failed) mbar_arrive(&acc_empty[acc_stage]);
                if (++acc_stage == 2) { acc_stage = 0; acc_phase ^= 1; }

                const int tile_end_row = min((k + 1) * kTileM, jb.n_time);
                const int first_row = k * kTileM;
                const bool fused = !kServed && p.codes != nullptr;
                if (!short_win) {
                    if (cur_win >= 0 && min((cur_win + 1) * jb.spectra, jb.n_time) <= tile_end_row) {
                        flush(cur_win);
                        cur_win = -1;
                    }
                    // Does a window end in this tile (the same for every warp)?  Only
                    // then (or with fused quantization) do the slots need a barrier.
                    bool ends = false;
                    if (first_row < jb.n_time) {
                        const int w_last_row = tile_end_row - 1;
                        const int wl = w_last_row / jb.spectra;
                        ends = min((wl + 1) * jb.spectra, jb.n_time) - 1 == w_last_row ||
                               (wl > 0 && wl * jb.spectra - 1 >= first_row);
                    }
                    if (ends || fused) named_barrier(1, kEpiThreads);
                    // quantize the groups this CTA completed one tile ago (list published
                    // by epilogue thread 0 before the barrier)
                    if (fused) quantize_ready(p, s_quant, s_meta, et, lane, kEpiWarps);
                    // finalize every window whose last spectrum lies in this tile
                    if (ends) {
                        const int w_first = first_row / jb.spectra;
                        const int w_last_in = (tile_end_row - 1) / jb.spectra;
                        for (int w = w_first; w <= w_last_in; ++w) {
                            const int w_last = min((w + 1) * jb.spectra, jb.n_time) - 1;
                            if (w_last < first_row || w_last >= tile_end_row) continue;
                            float* s = slots + (w % kRing) * 4 * NB;
                            for (int b = et; b < NB; b += kEpiThreads) {
                                const float total = ((s[b] + s[NB + b]) + s[2 * NB + b]) + s[3 * NB + b];
                                s[b] = s[NB + b] = s[2 * NB + b] = s[3 * NB + b] = 0.f;
                                if (b < jb.n_beams) {
                                    jb.integrated[((static_cast<size_t>(un.shard) * jb.n_windows + jb.w0 + w) *
                                                       jb.n_freq + un.f) * jb.beam_stride + b] = total;
                                }
                            }
                        }
                    }
                }
                // one decision for all epilogue warps, at the end of each unit (and
                // every tile with fused quantization): stop together or go on
                // together; a failed wait only makes the remaining tiles of the
                // unit skip their work
                if ((k + 1 == un.tile_end || fused) &&
                    named_barrier_or(1, kEpiThreads, failed || *s_fail != 0)) {
                    stop = true;
                    break;
                }
                if (fused && !short_win && et == 0) {
                    // Fused int8 quantization.  A 1x16x16 chunk spans 16 channels that
                    // other CTAs own: each finished (window, channel) bumps its
                    // 16-channel group's counter, and the CTA whose bump completes the
                    // group quantizes the group's chunks for that window.  A GPU-scope
                    // release waits for the releasing thread's outstanding stores, so the
                    // bump for a tile's windows is issued one tile after their stores
                    // (ordered by the barriers in between; the release is cumulative) and
                    // its result is published one tile later still: both waits overlap
                    // the tensor work instead of stalling the epilogue.
                    publish_ready(pend, s_quant, s_meta);
                    issue_arrivals(p, recorded, pend);
                    record_finalized(p, un, first_row, tile_end_row, recorded);
                }
            }
        }
        if (!kServed && p.codes != nullptr && !stop) {
            // drain the three stages: published list, bumps in flight, recorded windows
            for (int round = 0; round < 3; ++round) {
                named_barrier(1, kEpiThreads);
                quantize_ready(p, s_quant, s_meta, et, lane, kEpiWarps);
                named_barrier(1, kEpiThreads);
                if (et == 0) {
                    publish_ready(pend, s_quant, s_meta);
                    issue_arrivals(p, recorded, pend);
                    recorded.mask = 0;
                }
            }
            named_barrier(1, kEpiThreads);
            quantize_ready(p, s_quant, s_meta, et, lane, kEpiWarps);
        }
    }

    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TMEM_COLS);
    }
}

// ------------------------------------------------------------------------
// weight preparation: canonical complex64 -> split fp16 swizzled image
// ------------------------------------------------------------------------
// n_beams beams from b0 of canonical weights holding b_total beams per shard.
__global__ void prepare_split_kernel(const float2* __restrict__ w, uint8_t* __restrict__ out,
                                     int n_freq, int n_ant, int n_beams, int nb_pad, int n_shards, int b0,
                                     int b_total) {
    const int K = 2 * n_ant, N = 2 * nb_pad;
    const long long per_channel = static_cast<long long>(N) * K;
    const long long total = per_channel * n_freq * n_shards;
    const uint32_t w_bytes = (K / 64) * N * 128;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long ch = i / per_channel;  // shard * F + f
        const int rem = static_cast<int>(i % per_channel);
        const int n = rem / K, k = rem % K;
        const int shard = static_cast<int>(ch / n_freq), f = static_cast<int>(ch % n_freq);
        // inverse of the decode order: k -> (antenna, component)
        const int q = k / 32, j = (k % 32) / 8, pslot = k % 8;
        static constexpr int kAnt[8] = {0, 2, 0, 2, 1, 3, 1, 3};
        static constexpr int kIm[8] = {0, 0, 1, 1, 0, 0, 1, 1};
        const int a = 16 * q + 4 * j + kAnt[pslot];
        const int comp = kIm[pslot];
        const int b = n >> 1, out_im = n & 1;
        float coef = 0.f;
        if (b < n_beams) {
            const float2 wv = w[((static_cast<size_t>(shard) * b_total + b0 + b) * n_freq + f) * n_ant + a];
            // re out: x_re*wr - x_im*wi ; im out: x_re*wi + x_im*wr
            coef = out_im ? (comp ? wv.x : wv.y) : (comp ? -wv.y : wv.x);
        }
        const __half hi = __float2half_rn(coef);
        const __half lo = __float2half_rn(coef - __half2float(hi));
        const int kb = k / 64, kk = k % 64;
        const uint32_t off = kb * (N * 128) + n * 128 + ((((kk >> 3) ^ (n & 7))) << 4) + (kk & 7) * 2;
        uint8_t* base = out + ch * 2 * w_bytes;
        *reinterpret_cast<__half*>(base + off) = hi;
        *reinterpret_cast<__half*>(base + w_bytes + off) = lo;
    }
}

// ------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<EncodeTiledFn>(p);
        }
    });
    return fn;
}

int padded_beams(uint64_t b) { return static_cast<int>((b + 15) / 16 * 16); }

// At 128 and 256 antennas the voltage operand lives in TMEM and the shared
// memory holds one channel's hi + lo weight images for at most 64 beams
// (K = 256: 32 KB per 16 beams) or 32 beams (K = 512), so more beams run in
// groups: one launch per group over the same voltage, each writing its
// columns of the integrated rows.  The operand holds the groups' images one
// after the other, each padded to a multiple of 16 beams.
bool beam_groups(uint64_t n_ant) { return n_ant >= 128; }
// 64 beams at 128 antennas; at 256 (K = 512) an image of 32 beams is 128 KB
int group_size(const bf_dims& d) { return d.n_ant == 256 ? 32 : 64; }
int group_count(const bf_dims& d) { return static_cast<int>((d.n_beams + group_size(d) - 1) / group_size(d)); }
int group_beams(const bf_dims& d, int g) {
    return static_cast<int>(
        std::min<uint64_t>(group_size(d), d.n_beams - static_cast<uint64_t>(g) * group_size(d)));
}
uint64_t group_image_bytes(const bf_dims& d, uint64_t n_shards, int nb_pad) {
    return n_shards * d.n_freq * 2ull * (2 * d.n_ant) * (2ull * nb_pad) * 2ull;
}

template <int A, int NB, bool kServed>
bf_status launch_tc(cudaStream_t stream, const CUtensorMap& map, const TcParams& p, int grid,
                    bool set_attribute = true) {
    const Smem s = smem_plan(A, NB, kServed);
    const size_t smem = s.total + 1024;
    auto kern = grid_tensor_kernel<A, NB, kServed>;
    if (set_attribute) {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return cuda_status(err, "grid_tensor_kernel smem attribute");
    }
    if (grid == 0) return BF_OK;
    kern<<<grid, kThreads, smem, stream>>>(map, p);
    return cuda_status(cudaGetLastError(), "grid_tensor_kernel launch");
}

template <int A>
bf_status dispatch_nb(cudaStream_t stream, const CUtensorMap& map, const TcParams& p, int nb_pad, int grid) {
    switch (nb_pad) {
        case 16: return launch_tc<A, 16, false>(stream, map, p, grid);
        case 32: return launch_tc<A, 32, false>(stream, map, p, grid);
        case 48: return launch_tc<A, 48, false>(stream, map, p, grid);
        case 64: return launch_tc<A, 64, false>(stream, map, p, grid);
        case 80: return launch_tc<A, 80, false>(stream, map, p, grid);
        case 96: return launch_tc<A, 96, false>(stream, map, p, grid);
        case 112: return launch_tc<A, 112, false>(stream, map, p, grid);
        case 128: return launch_tc<A, 128, false>(stream, map, p, grid);
        default: return set_error(BF_ERR_INVALID_ARGUMENT, "n_beams must be between 1 and 128");
    }
}

// Served launches are captured in CUDA graphs: the shared-memory attribute is
// set once beforehand (grid == 0 sets it without launching) and not during
// capture.
template <int A>
bf_status dispatch_served(cudaStream_t stream, const CUtensorMap& map, const TcParams& p, int nb_pad, int grid) {
    const bool attr = grid == 0;
    switch (nb_pad) {
        case 16: return launch_tc<A, 16, true>(stream, map, p, grid, attr);
        case 32: return launch_tc<A, 32, true>(stream, map, p, grid, attr);
        case 64: return launch_tc<A, 64, true>(stream, map, p, grid, attr);
        case 128: return launch_tc<A, 128, true>(stream, map, p, grid, attr);
        default: return set_error(BF_ERR_INVALID_ARGUMENT, "served beam classes are 16, 32, 64 and 128");
    }
}

long long gcd_ll(long long a, long long b) { return b == 0 ? a : gcd_ll(b, a % b); }

}  // namespace

uint64_t split_weight_bytes(const bf_dims& d, uint64_t n_shards, int nb_pad) {
    const uint64_t K = 2 * d.n_ant;
    const uint64_t N = 2 * static_cast<uint64_t>(nb_pad > 0 ? nb_pad : padded_beams(d.n_beams));
    return n_shards * d.n_freq * 2ull * K * N * 2ull;
}

bf_status launch_prepare_split(cudaStream_t stream, const float* w, void* split, const bf_dims& d,
                               uint64_t n_shards, int nb_pad) {
    if (beam_groups(d.n_ant)) {
        if (nb_pad > 0) return set_error(BF_ERR_UNSUPPORTED, "served jobs use 32 or 64 antennas");
        uint8_t* out = static_cast<uint8_t*>(split);
        for (int g = 0; g < group_count(d); ++g) {
            const int nb = group_beams(d, g), nbp = padded_beams(nb);
            const long long total = static_cast<long long>(n_shards) * d.n_freq * 2 * nbp * 2 * d.n_ant;
            const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 32));
            prepare_split_kernel<<<blocks, 256, 0, stream>>>(
                reinterpret_cast<const float2*>(w), out, static_cast<int>(d.n_freq), static_cast<int>(d.n_ant), nb,
                nbp, static_cast<int>(n_shards), g * group_size(d), static_cast<int>(d.n_beams));
            BF_RETURN_IF(cuda_status(cudaGetLastError(), "prepare_split_kernel launch"));
            out += group_image_bytes(d, n_shards, nbp);
        }
        return BF_OK;
    }
    const int nbp = nb_pad > 0 ? nb_pad : padded_beams(d.n_beams);
    const long long total = static_cast<long long>(n_shards) * d.n_freq * 2 * nbp * 2 * d.n_ant;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 32));
    prepare_split_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const float2*>(w),
                                                     static_cast<uint8_t*>(split), static_cast<int>(d.n_freq),
                                                     static_cast<int>(d.n_ant), static_cast<int>(d.n_beams),
                                                     nbp, static_cast<int>(n_shards), 0,
                                                     static_cast<int>(d.n_beams));
    return cuda_status(cudaGetLastError(), "prepare_split_kernel launch");
}

uint64_t grid_tensor_counter_count(const bf_dims& d, uint64_t spectra, uint64_t n_shards) {
    return n_shards * window_count(d.n_time, spectra) * ((d.n_freq + 15) / 16);
}

long long tc_job_tiling(TcJob& job, int n_time, int spectra, int n_freq, int n_shards, int group_mult) {
    job.n_time = n_time;
    job.spectra = spectra;
    job.n_freq = n_freq;
    job.n_shards = n_shards;
    job.rows_q = small_window_rows(spectra);
    const int rows_per_tile = 4 * job.rows_q;
    job.tiles_per_channel = (n_time + rows_per_tile - 1) / rows_per_tile;
    if (spectra < 32) {
        job.group_tiles = 1;  // windows never cross a tile
    } else {
        const long long lcm = static_cast<long long>(spectra) / gcd_ll(spectra, kTileM) * kTileM;
        job.group_tiles = static_cast<int>(lcm / kTileM);
    }
    job.group_tiles *= std::max(1, group_mult);
    job.groups_per_channel = (job.tiles_per_channel + job.group_tiles - 1) / job.group_tiles;
    return static_cast<long long>(n_shards) * n_freq * job.groups_per_channel;
}

int tc_padded_beams(uint64_t b) { return padded_beams(b); }

bf_status encode_voltage_map(CUtensorMap* map, const uint8_t* base, uint64_t n_ant, uint64_t n_freq,
                             uint64_t n_rows, uint64_t n_shards, uint64_t row_stride, uint64_t shard_stride,
                             int rows_q) {
    EncodeTiledFn enc = encode_fn();
    if (enc == nullptr) return set_error(BF_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    const cuuint64_t dims[4] = {n_ant, n_freq, n_rows, n_shards};
    const cuuint64_t strides[3] = {n_ant, row_stride, shard_stride};
    const cuuint32_t box_rows = static_cast<cuuint32_t>(rows_q == 32 ? kTileM : rows_q);
    // rows of 128 antennas and more arrive in 128-byte boxes, swizzled
    const cuuint32_t box[4] = {static_cast<cuuint32_t>(n_ant >= 128 ? 128 : n_ant), 1, box_rows, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<uint8_t*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     // 128-antenna rows are read one row per thread: 128-byte swizzle
                     n_ant >= 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(BF_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(r));
    return BF_OK;
}

namespace {

bf_status launch_grid_tensor_impl(cudaStream_t stream, const uint8_t* v, const void* split, float* integrated,
                                  int8_t* codes, float* params, const bf_dims& d, uint64_t spectra,
                                  uint64_t n_shards, unsigned* counters, const int* unit_list,
                                  const int* unit_count, const GridTuning& tune) {
    if (d.n_time >= (1ull << 31) || n_shards > 1024 || spectra >= (1ull << 30)) {
        return set_error(BF_ERR_OVERFLOW, "CUDA tensor-core grid exceeds the supported size");
    }
    if (d.n_ant != 32 && d.n_ant != 64 && d.n_ant != 128 && d.n_ant != 256) {
        return set_error(BF_ERR_UNSUPPORTED, "the tensor-core kernel supports n_ant 32, 64, 128 or 256");
    }
    const bool groups = beam_groups(d.n_ant);
    if (groups && unit_list != nullptr) {
        return set_error(BF_ERR_UNSUPPORTED, "unit lists cover 32 or 64 antennas");
    }
    const int S = static_cast<int>(spectra);
    TcParams p{};
    p.job.split = static_cast<const uint8_t*>(split);
    p.job.integrated = integrated;
    p.job.n_beams = static_cast<int>(d.n_beams);
    p.job.beam_stride = static_cast<int>(d.n_beams);
    p.job.n_windows = static_cast<int>(window_count(d.n_time, spectra));
    p.job.w0 = 0;
    p.job.t0 = 0;
    p.job.unit_begin = 0;
    p.n_units = tc_job_tiling(p.job, static_cast<int>(d.n_time), S, static_cast<int>(d.n_freq),
                              static_cast<int>(n_shards), unit_list != nullptr ? 1 : tune.group_mult);
    p.ftiles = static_cast<int>((d.n_freq + 15) / 16);
    p.btiles = static_cast<int>((d.n_beams + 15) / 16);

    CUtensorMap map;
    bf_status st = encode_voltage_map(&map, v, d.n_ant, d.n_freq, d.n_time, n_shards, d.n_freq * d.n_ant,
                                      d.n_time * d.n_freq * d.n_ant, p.job.rows_q);
    if (st != BF_OK) return st;

    // Fused quantization runs in the long-window epilogue; short windows
    // and beam groups (a chunk is complete only after every group) quantize
    // with the separate kernel.
    const bool fused = codes != nullptr && counters != nullptr && S >= 32 && !groups;
    if (fused) {
        p.codes = codes;
        p.params = reinterpret_cast<float2*>(params);
        p.counters = counters;
        const cudaError_t e = cudaMemsetAsync(counters, 0,
                                              grid_tensor_counter_count(d, spectra, n_shards) * sizeof(unsigned),
                                              stream);
        if (e != cudaSuccess) return cuda_status(e, "clear quantization counters");
    }

    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = static_cast<int>(std::min<long long>(sms, p.n_units));
    p.paired = (tune.paired && d.n_freq % 2 == 0 && grid % 2 == 0 && grid >= 2) ? 1 : 0;
    if (unit_list != nullptr) {
        // the list's length is known on the device only: one CTA per SM, each
        // taking its share of the list (none when it is empty)
        p.unit_list = unit_list;
        p.unit_count = unit_count;
        p.paired = 0;
        grid = sms;
    }
    if (grid > 0 && groups) {
        const uint8_t* img = p.job.split;
        for (int g = 0; g < group_count(d); ++g) {
            TcParams pg = p;
            const int nb = group_beams(d, g), nbp = padded_beams(nb);
            pg.job.split = img;
            pg.job.integrated = integrated + g * group_size(d);
            pg.job.n_beams = nb;
            pg.btiles = (nb + 15) / 16;
            if (d.n_ant == 256) {
                st = nbp == 16 ? launch_tc<256, 16, false>(stream, map, pg, grid)
                               : launch_tc<256, 32, false>(stream, map, pg, grid);
            } else {
                switch (nbp) {
                    case 16: st = launch_tc<128, 16, false>(stream, map, pg, grid); break;
                    case 32: st = launch_tc<128, 32, false>(stream, map, pg, grid); break;
                    case 48: st = launch_tc<128, 48, false>(stream, map, pg, grid); break;
                    default: st = launch_tc<128, 64, false>(stream, map, pg, grid); break;
                }
            }
            if (st != BF_OK) return st;
            img += group_image_bytes(d, n_shards, nbp);
        }
    } else if (grid > 0) {
        const int nbp = padded_beams(d.n_beams);
        st = d.n_ant == 32 ? dispatch_nb<32>(stream, map, p, nbp, grid) : dispatch_nb<64>(stream, map, p, nbp, grid);
        if (st != BF_OK) return st;
    }
    if (codes == nullptr || fused) return BF_OK;
    bf_dims qd{n_shards * static_cast<uint64_t>(p.job.n_windows), d.n_freq, d.n_ant, d.n_beams};
    return launch_quantize(stream, integrated, codes, params, qd);
}

}  // namespace

bf_status launch_grid_tensor(cudaStream_t stream, const uint8_t* v, const void* split, float* integrated,
                             int8_t* codes, float* params, const bf_dims& d, uint64_t spectra,
                             uint64_t n_shards, unsigned* counters, const GridTuning* tune) {
    GridTuning t;
    if (tune != nullptr) {
        t = *tune;
    } else {
        tuned_grid_config(static_cast<int>(d.n_ant), padded_beams(d.n_beams), spectra, &t);
    }
    return launch_grid_tensor_impl(stream, v, split, integrated, codes, params, d, spectra, n_shards, counters,
                                   nullptr, nullptr, t);
}

bf_status launch_grid_tensor_list(cudaStream_t stream, const uint8_t* v, const void* split, float* integrated,
                                  const bf_dims& d, uint64_t spectra, uint64_t n_shards, const int* unit_list,
                                  const int* unit_count) {
    return launch_grid_tensor_impl(stream, v, split, integrated, nullptr, nullptr, d, spectra, n_shards, nullptr,
                                   unit_list, unit_count, GridTuning{});
}

long long grid_tensor_unit_layout(const bf_dims& d, uint64_t spectra, uint64_t n_shards, int* groups_per_channel,
                                  int* windows_per_group) {
    TcJob job{};
    const long long n = tc_job_tiling(job, static_cast<int>(d.n_time), static_cast<int>(spectra),
                                      static_cast<int>(d.n_freq), static_cast<int>(n_shards));
    *groups_per_channel = job.groups_per_channel;
    *windows_per_group = spectra < 32 ? 0 : static_cast<int>(job.group_tiles * kTileM / spectra);
    return n;
}

bf_status launch_grid_tensor_served(cudaStream_t stream, const CUtensorMap& map, int n_ant, int nb_pad,
                                    const TcTableHeader* table, int grid) {
    TcParams p{};
    p.table = table;
    if (n_ant == 32) return dispatch_served<32>(stream, map, p, nb_pad, grid);
    if (n_ant == 64) return dispatch_served<64>(stream, map, p, nb_pad, grid);
    return set_error(BF_ERR_UNSUPPORTED, "served jobs use 32 or 64 antennas");
}

// Device address of the error word for kernels in other translation units
// (device globals are per translation unit without relocatable device code).
unsigned* device_error_word(cudaStream_t stream) {
    static SymbolAddressCache cache;
    void* p = nullptr;
    if (device_symbol_address(&g_tc_error, cache, stream, &p, "device error word") != BF_OK) return nullptr;
    return static_cast<unsigned*>(p);
}

bf_status take_tc_error(uint32_t* code) {
    unsigned v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(v));
    if (e != cudaSuccess) return cuda_status(e, "read device error word");
    e = cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(zero));
    if (e != cudaSuccess) return cuda_status(e, "clear device error word");
    if (code) *code = v;
    return BF_OK;
}

}  // namespace bf
