// grid_cov.cu -- the fixed-grid beamformer in covariance form, for long
// integration windows.
//
// The reference integrates I[w][f][b] = sum_{t in w} |sum_a w_a x_a(t)|^2
// spectrum by spectrum (src/cuda_beamformer.cu:108-354,
// src/temporal_integration.cpp:16-110).  The same window sum is a quadratic
// form in the window's array covariance:
//   I[w][f][b] = v_b^T E v_b,   E = [[Rr, -Ri], [Ri, Rr]],
//   R = sum_{t in w} x(t) x(t)^H,  v_b = [Re w_b ; -Im w_b]
// (w x = conj(w)^H x, so the beam is conj(w)^H R conj(w)), and E is the real
// 2A x 2A form of the Hermitian R.  Per (window, channel) this kernel runs
//   1. the Gram G = sum_t y(t) y(t)^T of the real components y (16 x the int4
//      values, so one mask per four components unpacks them) as tcgen05
//      kind::i8 MMAs: M = N = 128 components, K = the window's spectra, exact
//      int32 in TMEM;
//   2. E from G (E_mn = (G_mn +- G_m'n') / 256 with m' the other part of the
//      same antenna, one warp shuffle per element) split into fp16 hi + lo
//      (E = hi + lo exactly: E is an integer below 2^16 after scaling), written
//      back over G in TMEM as the A operand of
//   3. Y = E V on kind::f16 with A from TMEM and B = V (hi and lo) from shared
//      memory: hi*Vhi + hi*Vlo + lo*Vhi, fp32 in TMEM (the dropped lo*Vlo is
//      below 2^-22 of the product);
//   4. I_b = sum_m V[m][b] Y[m][b] in fp32 (fixed butterfly order).
// The fp32 sums in 3 and 4 carry terms as large as |v_b|^2 tr(E) (E is
// positive semidefinite, so |E_mn| <= sqrt(E_mm E_nn) and, by Cauchy-Schwarz,
// sum_mn |V_mb E_mn V_nb| <= |v_b|^2 tr(E)), so the relative error of a beam
// scales with est_b = 2^-23 |v_b|^2 tr(E) / I_b: small for beams that carry
// the window's power, large for deep sidelobes of a strong source.  On
// request the kernel writes est_b per value and lists, for the split direct
// kernel (grid_tc.cu) to recompute, every unit holding a value whose estimate
// exceeds a limit calibrated against FP64 (the checked form,
// bf_grid_auto_integrated).
// Tensor work per (window, channel) at A = 64, B = 128: 128 x 128 x S int8
// MACs + 3 x 128^3 fp16 MACs, against 2 x 128 x 256 x S fp16 MACs for the
// split direct form: 2.35x less at S = 320.  The covariance is exact, so the
// only rounding is in the fp16 split of V (2^-22) and fp32 sums.
//
// CTA (one per SM, 768 threads): warp 0 TMA producer (64-spectrum tiles of one
// channel, 64 bytes per row; CTAs 2c and 2c + 1 walk the same windows of the
// even and odd channel of a pair, so both halves of each 128-byte line are
// read together), warp 1 MMA issuer and TMEM owner, warps 2-4, 6-8, 10 and 11
// unpack, warps 12-19 convert (two per TMEM lane quadrant), warps 20-23 form
// the beam sums.
// TMEM: two 128-column E stages (Gram accumulator, then A operand) and two
// 128-column Y stages.  Shared memory: the channel's V image (fp16 hi, fp16 lo in the
// 128-byte-swizzled K-major layout, fp32 [component][beam] in rows of 132), voltage stages.
// Every wait is bounded and reports through the device error word.
#include "bf_internal.cuh"
#include "grid_tc.cuh"
#include "sm100.cuh"

#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <mutex>

namespace bf {

namespace {

using namespace sm100;

// Warp roles.  A warp runs on SM sub-partition (warp id % 4), and the MMA
// issuer (warp 1) shares sub-partition 1 with every warp whose id is 1 mod 4:
// the unpack warps, which have no TMEM lane constraint, avoid it (warps 5 and
// 9 stay idle), so the issuer competes with three compute warps (one convert
// pair member and one beam-sum warp per quadrant must sit there), not five.
constexpr int kThreads = 768;
constexpr int kUnpackWarps = 8;        // warps 2-4, 6-8, 10, 11
constexpr int kConvFirst = 12, kConvWarps = 8;
constexpr int kDotFirst = 20, kDotWarps = 4;
__host__ __device__ constexpr bool unpack_warp(int w) { return w >= 2 && w < kConvFirst && w != 5 && w != 9; }
// 0..7 over the unpack warps
__host__ __device__ constexpr int unpack_slot(int w) { return w - 2 - (w > 5) - (w > 9); }
constexpr int kRows = 64;                             // spectra per voltage tile
constexpr int kRawStages = 8, kXStages = 6;
constexpr uint32_t kRawBytes = kRows * 64;            // one channel, 64 antennas
constexpr uint32_t kXBytes = kRows * 128;             // [row][128 components] int8
constexpr uint32_t kWHalf = 128 * 256;                // [128 beams][128 K] fp16
constexpr int kVPitch = 132;                          // floats per component row of the fp32 V
constexpr uint32_t kVBytes = 128 * kVPitch * 4;       // [component][beam] fp32, rows padded
constexpr uint32_t kWImage = 2 * kWHalf + kVBytes;    // per channel
constexpr uint32_t kYCol = 256;                       // TMEM columns of the two Y stages
constexpr uint64_t kWaitNs = 2000000000ull;
// trace partials of unit j sit in slot j % kTrSlots until the beam sums of
// unit j read them, after freeing Y of unit j; the converters reach unit
// j + kTrSlots only after Y of unit j + kTrSlots - 4 was freed, so any ring of
// at least five slots is safe
constexpr int kTrSlots = 8;
// mbarriers, TMEM address, fail flag, per-unit trace partials [kTrSlots][4]
constexpr uint32_t kBarBytes = (2 * kRawStages + 2 * kXStages + 11 + kTrSlots) * 8 + 8 + kTrSlots * 16;
constexpr uint32_t kSmemBytes = kWImage + kXStages * kXBytes + kRawStages * kRawBytes + 2 * 4 * 128 * 4 + 512 + 1024;
static_assert(kBarBytes <= 512, "barrier block");
static_assert(kSmemBytes <= 232448, "shared memory per CTA");

struct CovGridParams {
    const uint8_t* wimg;     // [shard][F][kWImage]
    float* out;              // [shard][W][F][B]
    unsigned* err;
    int n_freq, n_beams, n_windows, n_time, spectra;
    long long n_pair_units;  // shards x F/2 x windows
    float out_scale;         // 2^k
    // E scaled by 2^-k as one integer add and one subtract: the float
    // 1.5 x 2^(23 - k) has mantissa steps of 2^-k, so adding e (|e| < 2^22) to
    // its bits and subtracting it again is exact
    int e_magic_bits;
    float e_magic;
    // error estimates (checked form): est [shard][W][F][B] or null; with
    // est_limit > 0 every split-kernel unit (shard, channel, group of
    // split_gw windows; split_gpc groups per channel) holding an estimate
    // above the limit is appended once to unit_list
    float* est;
    float est_limit;
    unsigned* unit_flags;    // [split units], zero at launch
    int* unit_list;
    int* unit_count;         // zero at launch
    int split_gpc, split_gw;
};

// est_b = kEstScale |v_b|^2 tr(E) / I_b
constexpr float kEstScale = 0x1p-23f;

__device__ __forceinline__ void cov_grid_error(unsigned* err, unsigned code) {
    if (err != nullptr) atomicOr(err, 0x80000000u | (code << 16));
}

// A CTA's pair-units in order -- the windows of a channel pair, then the next
// pair, then the next shard -- without a division per unit.
struct CovCursor {
    int s, fp, w;
    __device__ __forceinline__ void start(long long pu, const CovGridParams& p) {
        const long long per_shard = static_cast<long long>(p.n_freq / 2) * p.n_windows;
        s = static_cast<int>(pu / per_shard);
        const long long r = pu % per_shard;
        fp = static_cast<int>(r / p.n_windows);
        w = static_cast<int>(r % p.n_windows);
    }
    __device__ __forceinline__ void next(const CovGridParams& p) {
        if (++w == p.n_windows) {
            w = 0;
            if (++fp == p.n_freq / 2) {
                fp = 0;
                ++s;
            }
        }
    }
    // the channel (and its weight image) changes after this unit
    __device__ __forceinline__ bool ends_run(const CovGridParams& p) const { return w + 1 == p.n_windows; }
};

__device__ __forceinline__ int cov_tiles(int w, const CovGridParams& p) {
    const int len = min(p.spectra, p.n_time - w * p.spectra);
    return (len + kRows - 1) / kRows;
}

// lane l ends with sum over the warp's lanes of v[l]
__device__ __forceinline__ float reduce_scatter32(float (&v)[32], int lane) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < o; ++i) {
            const float send = up ? v[i] : v[i + o];
            const float keep = up ? v[i + o] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

__global__ void __launch_bounds__(kThreads, 1)
grid_cov_kernel(const __grid_constant__ CUtensorMap vmap, const CovGridParams p) {
    constexpr uint32_t IDESC_G = idesc_s8_s32_mn(128, 128);
    constexpr uint32_t IDESC_Q = idesc_f16_f32(128, 128);
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* wsm = smem;                                   // V image
    uint8_t* xs = smem + kWImage;                          // kXStages x kXBytes
    uint8_t* raw = xs + kXStages * kXBytes;                // kRawStages x kRawBytes
    float* s_dot = reinterpret_cast<float*>(raw + kRawStages * kRawBytes);  // [2][4][128]
    uint64_t* bars = reinterpret_cast<uint64_t*>(s_dot + 2 * 4 * 128);
    uint64_t* raw_full = bars;                   // [kRawStages]
    uint64_t* raw_empty = raw_full + kRawStages; // [kRawStages]
    uint64_t* x_full = raw_empty + kRawStages;   // [kXStages]
    uint64_t* x_empty = x_full + kXStages;       // [kXStages]
    uint64_t* gram_done = x_empty + kXStages;    // [2]
    uint64_t* conv_done = gram_done + 2;         // [2]
    uint64_t* quad_done = conv_done + 2;         // [2]
    uint64_t* y_free = quad_done + 2;            // [2]
    uint64_t* w_full = y_free + 2;
    uint64_t* w_empty = w_full + 1;
    uint64_t* mma_done = w_empty + 1;
    uint64_t* tr_ready = mma_done + 1;           // [kTrSlots] trace partials of unit j in slot j % kTrSlots
    uint32_t* tmem_ptr = reinterpret_cast<uint32_t*>(tr_ready + kTrSlots);
    volatile int* s_fail = reinterpret_cast<volatile int*>(tmem_ptr + 1);
    float* s_trq = reinterpret_cast<float*>(tmem_ptr + 2);  // [kTrSlots][4 quadrants]
    const bool estimate = p.est != nullptr || p.est_limit > 0.f;

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
            mbar_init(&gram_done[i], 1);
            mbar_init(&conv_done[i], kConvWarps);
            mbar_init(&quad_done[i], 1);
            mbar_init(&y_free[i], kDotWarps);
        }
        mbar_init(w_full, 1);
        mbar_init(w_empty, 1 + kDotWarps);
        mbar_init(mma_done, 1);
        for (int i = 0; i < kTrSlots; ++i) mbar_init(&tr_ready[i], 4);
        *s_fail = 0;
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(tmem_ptr, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_ptr;

    // CTA pair c walks pair-units [begin, end); the even CTA takes the even channel
    const int odd = blockIdx.x & 1;
    const long long n_cp = gridDim.x / 2, cp = blockIdx.x / 2;
    const long long u_begin = p.n_pair_units * cp / n_cp;
    const long long u_end = p.n_pair_units * (cp + 1) / n_cp;
    auto fail = [&](unsigned code) {
        cov_grid_error(p.err, code);
        *s_fail = 1;
    };

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int armed[kRawStages];
            for (int s = 0; s < kRawStages; ++s) armed[s] = -1;
            int runs = 0;
            bool stop = false;
            CovCursor cur;
            cur.start(u_begin, p);
            for (long long pu = u_begin; pu < u_end && !stop; ++pu, cur.next(p)) {
                const int f = 2 * cur.fp + odd;
                const int nt = cov_tiles(cur.w, p);
                for (int k = 0; k < nt; ++k) {
                    if (*s_fail) { stop = true; break; }
                    if (!mbar_wait(&raw_empty[stage], phase ^ 1, kWaitNs)) { fail(1); stop = true; break; }
                    mbar_expect_tx(&raw_full[stage], kRawBytes);  // rows past the stream arrive zero filled
                    tma_load_4d(raw + stage * kRawBytes, &vmap, 0, f, cur.w * p.spectra + k * kRows, cur.s,
                                &raw_full[stage]);
                    armed[stage] = static_cast<int>(phase);
                    if (++stage == kRawStages) { stage = 0; phase ^= 1; }
                }
                if (stop) break;
                if (pu == u_begin || cur.w == 0) {
                    // after this unit's tiles, so the MMA can run its Gram while the
                    // previous channel's last beam sums finish
                    if (runs > 0 && !mbar_wait(w_empty, (runs - 1) & 1, kWaitNs)) { fail(2); break; }
                    mbar_expect_tx(w_full, kWImage);
                    const uint8_t* src = p.wimg + (static_cast<size_t>(cur.s) * p.n_freq + f) * kWImage;
                    for (uint32_t c = 0; c < kWImage; c += 32768) {
                        bulk_g2s(wsm + c, src + c, kWImage - c < 32768 ? kWImage - c : 32768u, w_full);
                    }
                    ++runs;
                }
            }
            for (int s = 0; s < kRawStages; ++s) {
                if (armed[s] >= 0 && !mbar_wait(&raw_full[s], static_cast<uint32_t>(armed[s]), kWaitNs)) fail(3);
            }
            if (runs > 0 && !mbar_wait(w_full, (runs - 1) & 1, kWaitNs)) fail(4);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int xst = 0;
            uint32_t xph = 0;
            bool stop = false;
            int runs = 0;
            // the quad of unit j - 1 is issued after the Gram of unit j
            long long q_idx = -1;
            bool q_first = false, q_ends = false;
            int q_run = 0;
            const uint64_t w_hi_desc = smem_desc_sw128(smem_u32(wsm));
            const uint64_t w_lo_desc = smem_desc_sw128(smem_u32(wsm) + kWHalf);
            const uint64_t x_desc = smem_desc_sw128_mn(smem_u32(xs));
            auto issue_quad = [&](long long i, bool first, bool last, int run) -> bool {
                const int eb = static_cast<int>(i & 1);
                const uint32_t par = static_cast<uint32_t>((i >> 1) & 1);
                if (!mbar_wait(&conv_done[eb], par, kWaitNs)) { fail(5); return false; }
                // Y[eb] was last read by the beam sums of unit i - 2
                if (i >= 2 && !mbar_wait(&y_free[eb], par ^ 1, kWaitNs)) { fail(6); return false; }
                if (first && !mbar_wait(w_full, static_cast<uint32_t>(run & 1), kWaitNs)) { fail(7); return false; }
                tc_fence_after();
                const uint32_t e_tm = tmem_base + eb * 128, y_tm = tmem_base + kYCol + eb * 128;
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) {
                    const uint32_t a_hi = e_tm + 32 * (kk >> 1) + 8 * (kk & 1), a_lo = a_hi + 16;
                    // descriptor start addresses advance in 16-byte units
                    const uint64_t off = ((kk >> 2) * (128 * 128) + (kk & 3) * 32) >> 4;
                    const uint64_t bh = w_hi_desc + off, bl = w_lo_desc + off;
                    mma_f16_ts(y_tm, a_hi, bh, IDESC_Q, kk > 0 ? 1u : 0u);
                    mma_f16_ts(y_tm, a_hi, bl, IDESC_Q, 1u);
                    mma_f16_ts(y_tm, a_lo, bh, IDESC_Q, 1u);
                }
                tc_commit(&quad_done[eb]);
                if (last) tc_commit(w_empty);
                return true;
            };
            long long j = 0;
            CovCursor cur;
            cur.start(u_begin, p);
            for (long long pu = u_begin; pu < u_end && !stop; ++pu, ++j, cur.next(p)) {
                const bool first = pu == u_begin || cur.w == 0;
                if (first) ++runs;
                const int eb = static_cast<int>(j & 1);
                // E[eb] was last read by the quad of unit j - 2, issued just before:
                // waiting for it lets the tensor pipe drain once per unit
                if (j >= 2 && !mbar_wait(&quad_done[eb], static_cast<uint32_t>(((j - 2) >> 1) & 1), kWaitNs)) {
                    fail(8);
                    break;
                }
                tc_fence_after();
                const uint32_t e_tm = tmem_base + eb * 128;
                const int nt = cov_tiles(cur.w, p);
                for (int k = 0; k < nt; ++k) {
                    if (*s_fail) { stop = true; break; }
                    if (!mbar_wait(&x_full[xst], xph, kWaitNs)) { fail(9); stop = true; break; }
                    tc_fence_after();
#pragma unroll
                    for (int kk = 0; kk < kRows / 32; ++kk) {
                        const uint64_t desc = x_desc + ((xst * kXBytes + kk * 32 * 128) >> 4);
                        mma_i8_ss(e_tm, desc, desc, IDESC_G, (k > 0 || kk > 0) ? 1u : 0u);
                    }
                    tc_commit(&x_empty[xst]);
                    if (++xst == kXStages) { xst = 0; xph ^= 1; }
                }
                if (stop) break;
                tc_commit(&gram_done[eb]);
                if (q_idx >= 0 && !issue_quad(q_idx, q_first, q_ends, q_run)) { stop = true; break; }
                q_idx = j;
                q_first = first;
                q_run = runs - 1;
                q_ends = cur.ends_run(p);
            }
            if (!stop && q_idx >= 0) issue_quad(q_idx, q_first, true, q_run);
            tc_commit(mma_done);
            if (!mbar_wait(mma_done, 0, kWaitNs)) fail(10);
        }
    } else if (unpack_warp(warp)) {
        // unpack: thread = (chunk c of 8 antennas, rows r0 and r0 + 32)
        const int ut = 32 * unpack_slot(warp) + lane;
        const int c = ut & 7, r0 = ut >> 3;
        int stage = 0, xst = 0;
        uint32_t phase = 0, xph = 0;
        bool stop = false;
        CovCursor cur;
        cur.start(u_begin, p);
        for (long long pu = u_begin; pu < u_end && !stop; ++pu, cur.next(p)) {
            const int nt = cov_tiles(cur.w, p);
            for (int k = 0; k < nt; ++k) {
                if (*s_fail) { stop = true; break; }
                if (!mbar_wait(&raw_full[stage], phase, kWaitNs)) { fail(11); stop = true; break; }
                if (!mbar_wait(&x_empty[xst], xph ^ 1, kWaitNs)) { fail(12); stop = true; break; }
                const uint8_t* rsrc = raw + stage * kRawBytes + c * 8;
                uint8_t* xdst = xs + xst * kXBytes;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int r = r0 + 32 * i;
                    const uint2 wv = *reinterpret_cast<const uint2*>(rsrc + r * 64);
                    // 16 x (re, im) of antennas 8c..8c+3 and 8c+4..8c+7: the nibble
                    // moved to the top of its byte is 16 x the signed value
                    const uint4 v = make_uint4((wv.x << 4) & 0xF0F0F0F0u, wv.x & 0xF0F0F0F0u,
                                               (wv.y << 4) & 0xF0F0F0F0u, wv.y & 0xF0F0F0F0u);
                    *reinterpret_cast<uint4*>(xdst + r * 128 + ((c ^ (r & 7)) << 4)) = v;
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
    } else if (warp < kConvFirst) {
        // idle (sub-partition 1 is left to the MMA issuer)
    } else if (warp < kDotFirst) {
        // convert: E = (G +- G') / 256 -> fp16 hi + lo over the same TMEM columns
        const int q = warp & 3, half = (warp - kConvFirst) >> 2;
        const int m = 32 * q + lane;
        const int sgn0 = ((m >> 2) & 1) != 0 ? -1 : 1;
        // the warp whose column chunks hold its quadrant's diagonal forms that
        // quadrant's part of tr(E) (integers times a power of two: exact)
        const bool has_diag = estimate && (q >> 1) == half;
        long long j = 0;
        for (long long pu = u_begin; pu < u_end; ++pu, ++j) {
            const int eb = static_cast<int>(j & 1);
            if (!mbar_wait(&gram_done[eb], static_cast<uint32_t>((j >> 1) & 1), kWaitNs)) { fail(13); break; }
            tc_fence_after();
            float diag = 0.f;
#pragma unroll 1
            for (int cc = 2 * half; cc < 2 * half + 2; ++cc) {
                const uint32_t taddr = tmem_base + ((32u * q) << 16) + eb * 128 + 32 * cc;
                uint32_t g[32];
                tmem_ld_32x32b_x32(taddr, g);
                tmem_ld_wait();
                float ef[32];
#pragma unroll
                for (int n = 0; n < 32; ++n) {
                    const int partner = __shfl_xor_sync(0xffffffffu, static_cast<int>(g[n ^ 4]), 4);
                    const int sg = ((n >> 2) & 1) != 0 ? -sgn0 : sgn0;
                    const int e = (static_cast<int>(g[n]) + sg * partner) >> 8;  // exact: both are 256 x
                    ef[n] = __int_as_float(e + p.e_magic_bits) - p.e_magic;
                }
                if (has_diag && cc == q) {
                    // ef[lane] by a select tree on the lane's bits (31 selects)
                    float t16[16], t8[8], t4[4], t2[2];
#pragma unroll
                    for (int i = 0; i < 16; ++i) t16[i] = (lane & 16) ? ef[i + 16] : ef[i];
#pragma unroll
                    for (int i = 0; i < 8; ++i) t8[i] = (lane & 8) ? t16[i + 8] : t16[i];
#pragma unroll
                    for (int i = 0; i < 4; ++i) t4[i] = (lane & 4) ? t8[i + 4] : t8[i];
#pragma unroll
                    for (int i = 0; i < 2; ++i) t2[i] = (lane & 2) ? t4[i + 2] : t4[i];
                    diag = (lane & 1) ? t2[1] : t2[0];
                }
                uint32_t r[32];
#pragma unroll
                for (int n = 0; n < 16; ++n) {
                    const __half2 h = __floats2half2_rn(ef[2 * n], ef[2 * n + 1]);
                    const float2 hf = __half22float2(h);
                    const __half2 l = __floats2half2_rn(ef[2 * n] - hf.x, ef[2 * n + 1] - hf.y);
                    r[n] = *reinterpret_cast<const uint32_t*>(&h);
                    r[16 + n] = *reinterpret_cast<const uint32_t*>(&l);
                }
                tmem_st_32x32b_x32(taddr, r);
            }
            tmem_st_wait();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&conv_done[eb]);
            if (has_diag) {
                // slot j % kTrSlots (the ring's bound is at its definition)
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) diag += __shfl_xor_sync(0xffffffffu, diag, o);
                if (lane == 0) {
                    s_trq[(j % kTrSlots) * 4 + q] = diag;
                    mbar_arrive(&tr_ready[j % kTrSlots]);
                }
            }
            if (*s_fail) break;
        }
    } else {
        // beam sums: I_b = sum_m V[m][b] Y[m][b]
        const int q = warp & 3;
        const int m = 32 * q + lane;
        const int t = 32 * (warp - kDotFirst) + lane;  // output beam of the final sum
        // [component][beam] with kVPitch-float rows: a lane's 32 beams of one
        // chunk are eight 16-byte loads, the lanes' rows spread over all banks
        const float* vt = reinterpret_cast<const float*>(wsm + 2 * kWHalf);
        float vnorm = 0.f;  // |v_t|^2 of the current channel
        long long j = 0;
        CovCursor cur;
        cur.start(u_begin, p);
        for (long long pu = u_begin; pu < u_end; ++pu, ++j, cur.next(p)) {
            const bool last = pu + 1 == u_end || cur.ends_run(p);
            const int eb = static_cast<int>(j & 1);
            if (!mbar_wait(&quad_done[eb], static_cast<uint32_t>((j >> 1) & 1), kWaitNs)) { fail(14); break; }
            tc_fence_after();
            if (estimate && (pu == u_begin || cur.w == 0)) {
                // the channel's image is in place until this run's last unit
                float acc = 0.f;
#pragma unroll 8
                for (int i = 0; i < 128; ++i) {
                    const float v = vt[((i + lane) & 127) * kVPitch + t];
                    acc = fmaf(v, v, acc);
                }
                vnorm = acc;
            }
            float part[4];
#pragma unroll 1
            for (int cb = 0; cb < 4; ++cb) {
                uint32_t y[32];
                tmem_ld_32x32b_x32(tmem_base + ((32u * q) << 16) + kYCol + eb * 128 + 32 * cb, y);
                tmem_ld_wait();
                if (cb == 3) {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&y_free[eb]);
                }
                float pr[32];
#pragma unroll
                for (int b4 = 0; b4 < 8; ++b4) {
                    const float4 v4 = *reinterpret_cast<const float4*>(vt + m * kVPitch + 32 * cb + 4 * b4);
                    pr[4 * b4] = __uint_as_float(y[4 * b4]) * v4.x;
                    pr[4 * b4 + 1] = __uint_as_float(y[4 * b4 + 1]) * v4.y;
                    pr[4 * b4 + 2] = __uint_as_float(y[4 * b4 + 2]) * v4.z;
                    pr[4 * b4 + 3] = __uint_as_float(y[4 * b4 + 3]) * v4.w;
                }
                part[cb] = reduce_scatter32(pr, lane);
            }
            __syncwarp();
            if (last && lane == 0) mbar_arrive(w_empty);
            // tr(E) of this unit, formed by the converters before its Y existed: read
            // here, off the path from the Y hand-off to the TMEM loads
            float tr = 0.f;
            if (estimate) {
                if (!mbar_wait(&tr_ready[j % kTrSlots], static_cast<uint32_t>((j / kTrSlots) & 1), kWaitNs)) {
                    fail(15);
                    break;
                }
                const float* tq = s_trq + (j % kTrSlots) * 4;
                tr = ((tq[0] + tq[1]) + tq[2]) + tq[3];
            }
            float* sd = s_dot + (j & 1) * 512;
#pragma unroll
            for (int cb = 0; cb < 4; ++cb) sd[q * 128 + 32 * cb + lane] = part[cb];
            named_barrier(1, 32 * kDotWarps);
            const float sum = ((sd[t] + sd[128 + t]) + sd[256 + t]) + sd[384 + t];
            const size_t oidx =
                ((static_cast<size_t>(cur.s) * p.n_windows + cur.w) * p.n_freq + 2 * cur.fp + odd) * p.n_beams + t;
            if (t < p.n_beams) p.out[oidx] = sum * p.out_scale;
            if (estimate) {
                const float bound = kEstScale * tr * vnorm;  // est = bound / sum
                if (p.est != nullptr && t < p.n_beams) p.est[oidx] = sum > 0.f ? bound / sum : INFINITY;
                if (p.est_limit > 0.f) {
                    // est <= limit without the division (a non-positive or NaN sum is over)
                    const bool over = t < p.n_beams && !(sum > 0.f && bound <= p.est_limit * sum);
                    if (__any_sync(0xffffffffu, over) && lane == 0) {
                        const int f = 2 * cur.fp + odd;
                        const int unit = (cur.s * p.n_freq + f) * p.split_gpc + cur.w / p.split_gw;
                        if (atomicExch(&p.unit_flags[unit], 1u) == 0u) p.unit_list[atomicAdd(p.unit_count, 1)] = unit;
                    }
                }
            }
            if (*s_fail) break;
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, 512);
    }
}

// Per channel: V = [Re w ; -Im w] in the unpack's component order (component
// m = 16c + 4h + k is antenna 8c + 4 (h >> 1) + k, real part for even h), as
// fp16 hi and lo [beam][component] in the 128-byte-swizzled K-major layout and
// as fp32 [component][beam] in rows of kVPitch floats (zero padded).  Beams
// past n_beams are zero.
__global__ void prepare_cov_kernel(const float2* __restrict__ w, uint8_t* __restrict__ out, int n_freq,
                                   int n_beams, int n_shards) {
    const long long total = static_cast<long long>(n_shards) * n_freq * 128 * 128;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long ch = i >> 14;  // shard * F + f
        const int rem = static_cast<int>(i & 16383);
        const int b = rem >> 7, m = rem & 127;
        const int shard = static_cast<int>(ch / n_freq), f = static_cast<int>(ch % n_freq);
        const int a = 8 * (m >> 4) + 4 * (((m >> 2) & 3) >> 1) + (m & 3);
        const int im = (m >> 2) & 1;
        float coef = 0.f;
        if (b < n_beams) {
            const float2 wv = w[((static_cast<size_t>(shard) * n_beams + b) * n_freq + f) * 64 + a];
            coef = im ? -wv.y : wv.x;
        }
        const __half hi = __float2half_rn(coef);
        const __half lo = __float2half_rn(coef - __half2float(hi));
        const int kb = m >> 6, kk = m & 63;
        const uint32_t off = kb * (128 * 128) + b * 128 + (((kk >> 3) ^ (b & 7)) << 4) + (kk & 7) * 2;
        uint8_t* base = out + ch * kWImage;
        *reinterpret_cast<__half*>(base + off) = hi;
        *reinterpret_cast<__half*>(base + kWHalf + off) = lo;
        float* vrow = reinterpret_cast<float*>(base + 2 * kWHalf) + m * kVPitch;
        vrow[b] = coef;
        if (b < kVPitch - 128) vrow[128 + b] = 0.f;  // row padding
    }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn_grid_cov() {
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

}  // namespace

uint64_t cov_weight_bytes(const bf_dims& d, uint64_t n_shards) { return n_shards * d.n_freq * kWImage; }

bf_status check_grid_cov(const bf_dims& d, uint64_t spectra, uint64_t n_shards) {
    if (d.n_ant != 64) return set_error(BF_ERR_UNSUPPORTED, "the covariance-form grid supports n_ant 64");
    if (spectra < kRows || spectra % kRows != 0 || spectra > 16384) {
        return set_error(BF_ERR_UNSUPPORTED,
                         "the covariance-form grid needs integration_spectra a multiple of 64, at most 16384");
    }
    if (d.n_freq % 2 != 0) return set_error(BF_ERR_UNSUPPORTED, "the covariance-form grid needs an even n_freq");
    if (n_shards == 0 || n_shards > 1024 || d.n_time >= (1ull << 31)) {
        return set_error(BF_ERR_OVERFLOW, "covariance-form grid request out of range");
    }
    return BF_OK;
}

bf_status launch_prepare_cov(cudaStream_t stream, const float* w, void* out, const bf_dims& d, uint64_t n_shards) {
    if (d.n_ant != 64) return set_error(BF_ERR_UNSUPPORTED, "the covariance-form grid supports n_ant 64");
    const long long total = static_cast<long long>(n_shards) * d.n_freq * 128 * 128;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 16));
    prepare_cov_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const float2*>(w), static_cast<uint8_t*>(out),
                                                   static_cast<int>(d.n_freq), static_cast<int>(d.n_beams),
                                                   static_cast<int>(n_shards));
    return cuda_status(cudaGetLastError(), "prepare_cov_kernel launch");
}

namespace {

// Estimates and fallback bookkeeping of one covariance-form launch.
struct CovChecks {
    float* est = nullptr;
    float est_limit = 0.f;
    unsigned* unit_flags = nullptr;
    int* unit_list = nullptr;
    int* unit_count = nullptr;
    int split_gpc = 0, split_gw = 0;
};

bf_status launch_grid_cov_impl(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated,
                               const bf_dims& d, uint64_t spectra, uint64_t n_shards, const CovChecks& chk) {
    BF_RETURN_IF(check_grid_cov(d, spectra, n_shards));
    EncodeTiledFn enc = encode_fn_grid_cov();
    if (enc == nullptr) return set_error(BF_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    CUtensorMap map;
    const cuuint64_t dims[4] = {64, d.n_freq, d.n_time, n_shards};
    const cuuint64_t strides[3] = {64, d.n_freq * 64, d.n_time * d.n_freq * 64};
    const cuuint32_t box[4] = {64, 1, static_cast<cuuint32_t>(kRows), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<uint8_t*>(v), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(BF_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(r));
    CovGridParams p{};
    p.wimg = static_cast<const uint8_t*>(wimg);
    p.out = integrated;
    p.err = device_error_word(stream);
    if (p.err == nullptr) return BF_ERR_CUDA;
    p.n_freq = static_cast<int>(d.n_freq);
    p.n_beams = static_cast<int>(d.n_beams);
    p.n_windows = static_cast<int>(window_count(d.n_time, spectra));
    p.n_time = static_cast<int>(d.n_time);
    p.spectra = static_cast<int>(spectra);
    p.n_pair_units = static_cast<long long>(n_shards) * (d.n_freq / 2) * p.n_windows;
    // |E| <= 128 S: scale it below the fp16 range (powers of two: exact)
    int k = 0;
    while (128.0 * static_cast<double>(spectra) * std::ldexp(1.0, -k) > 65504.0) ++k;
    p.out_scale = std::ldexp(1.0f, k);
    p.e_magic_bits = 0x4B400000 - (k << 23);
    p.e_magic = std::ldexp(12582912.0f, -k);
    p.est = chk.est;
    p.est_limit = chk.est_limit;
    p.unit_flags = chk.unit_flags;
    p.unit_list = chk.unit_list;
    p.unit_count = chk.unit_count;
    p.split_gpc = chk.split_gpc;
    p.split_gw = chk.split_gw;
    cudaError_t e = cudaFuncSetAttribute(grid_cov_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kSmemBytes));
    if (e != cudaSuccess) return cuda_status(e, "grid_cov_kernel smem attribute");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long grid = std::min<long long>(sms & ~1, 2 * p.n_pair_units);
    if (grid >= 2) {
        grid_cov_kernel<<<static_cast<int>(grid), kThreads, kSmemBytes, stream>>>(map, p);
        BF_RETURN_IF(cuda_status(cudaGetLastError(), "grid_cov_kernel launch"));
    }
    return BF_OK;
}

// The checked form's limit on est_b (relative, 2^-23 |v_b|^2 tr(E) / I_b):
// values at or below it are kept, every unit holding one above it is
// recomputed by the split kernel.  Calibrated on a B200 against the FP64
// oracle over noise, steered grids on a point source and random-phase beams
// on a strong source (every beam a sidelobe): every kept value was within
// 1e-5 / 2 of FP64 (the GPU test prints the error per estimate decade).
constexpr float kEstRatio = 1.0f / 16.0f;
constexpr float kAutoEstLimit = 1e-5f / kEstRatio;

uint64_t cov_part_bytes(const bf_dims& d, uint64_t n_shards) {
    return d.n_ant == 64 && d.n_freq % 2 == 0 ? cov_weight_bytes(d, n_shards) : 0;
}

}  // namespace

bf_status launch_grid_cov(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated, int8_t* codes,
                          float* params, const bf_dims& d, uint64_t spectra, uint64_t n_shards) {
    BF_RETURN_IF(launch_grid_cov_impl(stream, v, wimg, integrated, d, spectra, n_shards, CovChecks{}));
    if (codes == nullptr) return BF_OK;
    const bf_dims qd{n_shards * window_count(d.n_time, spectra), d.n_freq, d.n_ant, d.n_beams};
    return launch_quantize(stream, integrated, codes, params, qd);
}

bf_status launch_grid_cov_estimate(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated,
                                   float* estimate, const bf_dims& d, uint64_t spectra, uint64_t n_shards) {
    CovChecks chk;
    chk.est = estimate;
    return launch_grid_cov_impl(stream, v, wimg, integrated, d, spectra, n_shards, chk);
}

uint64_t auto_weight_bytes(const bf_dims& d, uint64_t n_shards) {
    return cov_part_bytes(d, n_shards) + split_weight_bytes(d, n_shards);
}

bool auto_uses_cov(const bf_dims& d, uint64_t spectra, uint64_t n_shards) {
    return d.n_ant == 64 && d.n_freq % 2 == 0 && spectra >= kRows && spectra % kRows == 0 && spectra <= 16384 &&
           n_shards >= 1 && n_shards <= 1024 && d.n_time < (1ull << 31);
}

uint64_t auto_workspace_bytes(const bf_dims& d, uint64_t spectra, uint64_t n_shards) {
    if (!auto_uses_cov(d, spectra, n_shards)) return 0;
    int gpc = 0, gw = 0;
    const long long units = grid_tensor_unit_layout(d, spectra, n_shards, &gpc, &gw);
    // [count, padding to 256 bytes][flags: units x u32][list: units x i32]
    return 256 + 8 * static_cast<uint64_t>(units);
}

bf_status launch_prepare_auto(cudaStream_t stream, const float* w, void* out, const bf_dims& d, uint64_t n_shards) {
    const uint64_t cov = cov_part_bytes(d, n_shards);
    if (cov > 0) BF_RETURN_IF(launch_prepare_cov(stream, w, out, d, n_shards));
    return launch_prepare_split(stream, w, static_cast<uint8_t*>(out) + cov, d, n_shards);
}

bf_status launch_grid_auto(cudaStream_t stream, const uint8_t* v, const void* wimg, float* integrated, int8_t* codes,
                           float* params, void* workspace, const bf_dims& d, uint64_t spectra, uint64_t n_shards,
                           const GridTuning* tune) {
    const uint64_t cov = cov_part_bytes(d, n_shards);
    const uint8_t* split = static_cast<const uint8_t*>(wimg) + cov;
    GridTuning t;
    if (tune != nullptr) {
        t = *tune;
    } else {
        tuned_grid_config(static_cast<int>(d.n_ant), tc_padded_beams(d.n_beams), spectra, &t);
    }
    if (!auto_uses_cov(d, spectra, n_shards) || t.form == 0) {
        return launch_grid_tensor(stream, v, split, integrated, codes, params, d, spectra, n_shards, nullptr, &t);
    }
    CovChecks chk;
    const long long units = grid_tensor_unit_layout(d, spectra, n_shards, &chk.split_gpc, &chk.split_gw);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    chk.unit_count = reinterpret_cast<int*>(ws);
    chk.unit_flags = reinterpret_cast<unsigned*>(ws + 256);
    chk.unit_list = reinterpret_cast<int*>(ws + 256 + 4 * static_cast<uint64_t>(units));
    chk.est_limit = kAutoEstLimit;
    BF_RETURN_IF(cuda_status(cudaMemsetAsync(ws, 0, 256 + 4 * static_cast<uint64_t>(units), stream),
                             "clear the fallback list"));
    BF_RETURN_IF(launch_grid_cov_impl(stream, v, wimg, integrated, d, spectra, n_shards, chk));
    BF_RETURN_IF(launch_grid_tensor_list(stream, v, split, integrated, d, spectra, n_shards, chk.unit_list,
                                         chk.unit_count));
    if (codes == nullptr) return BF_OK;
    const bf_dims qd{n_shards * window_count(d.n_time, spectra), d.n_freq, d.n_ant, d.n_beams};
    return launch_quantize(stream, integrated, codes, params, qd);
}

}  // namespace bf
