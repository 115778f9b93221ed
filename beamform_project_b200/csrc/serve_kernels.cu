// serve_kernels.cu -- kernels of the served batch besides the tensor grid:
// the device weight generator, the multi-job streaming tracker, and the
// multi-job chunk quantizer.
#include "bf_internal.cuh"
#include "serve.cuh"
#include "tracker_common.cuh"

#include <climits>

namespace bf {
namespace {

using namespace trk;

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kSpeedOfLight = 299792458.0;

// generate_weights (reference src/weights.cpp:38-55) term by term in double:
// k = 2*pi*f / c, delay = (px*dx + py*dy) + pz*dz, phase = k * delay,
// then (float) cos / (float) sin of the double phase.
__global__ void weights_kernel(const float* __restrict__ pos, const float* __restrict__ freq,
                               const float* __restrict__ dirs, float2* __restrict__ out, int n_shards,
                               int f_shard, int n_beams, int n_ant) {
    const long long total = static_cast<long long>(n_shards) * n_beams * f_shard * n_ant;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int a = static_cast<int>(i % n_ant);
        long long rest = i / n_ant;
        const int f = static_cast<int>(rest % f_shard);
        rest /= f_shard;
        const int b = static_cast<int>(rest % n_beams);
        const int s = static_cast<int>(rest / n_beams);
        const double k = __ddiv_rn(__dmul_rn(kTwoPi, static_cast<double>(freq[s * f_shard + f])), kSpeedOfLight);
        const double delay = __dadd_rn(__dadd_rn(__dmul_rn(static_cast<double>(pos[3 * a]), static_cast<double>(dirs[3 * b])),
                                                 __dmul_rn(static_cast<double>(pos[3 * a + 1]),
                                                           static_cast<double>(dirs[3 * b + 1]))),
                                       __dmul_rn(static_cast<double>(pos[3 * a + 2]), static_cast<double>(dirs[3 * b + 2])));
        const double phase = __dmul_rn(k, delay);
        out[i] = make_float2(static_cast<float>(cos(phase)), static_cast<float>(sin(phase)));
    }
}

// tracker_direction (reference src/beam_tracker.cpp:52-65) at sample t:
// l = l0 + (float)t * dl, m = m0 + (float)t * dm, n = sqrt(1 - (l*l + m*m)).
__device__ __forceinline__ float3 trajectory_direction(const float* tr, long long t) {
    const float tf = __ll2float_rn(t);
    const float l = __fadd_rn(tr[0], __fmul_rn(tf, tr[2]));
    const float m = __fadd_rn(tr[1], __fmul_rn(tf, tr[3]));
    const float tsq = __fadd_rn(__fmul_rn(l, l), __fmul_rn(m, m));
    return make_float3(l, m, __fsqrt_rn(__fsub_rn(1.0f, tsq)));
}

__device__ __forceinline__ int find_job(const long long* begins, int stride_ll, int n_jobs, long long u) {
    int lo = 0, hi = n_jobs - 1;  // last job whose first unit is <= u
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (begins[static_cast<long long>(mid) * stride_ll] <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The streaming tracker of tracker_stream.cu generalised to a job table and
// to up to 8 sources per unit: the m16n8 tile's 8 columns carry
// (re, im) x (hi, lo) of two sources, so a unit runs up to four tiles over
// the same decoded voltage.  A unit is (job, window, 8 channels, 8 sources);
// warp w of the CTA owns channel 8 * group + w.  The unit's steering
// weights are computed once each: the CTA forms the FP64 delays of its 8
// sources (shared by the 8 channels), each warp the weights of its channel,
// split at once into the four fp16 parts (re hi, im hi, re lo, im lo) that
// the fragments hold.  A part row keeps antennas a and a + 2 in one 32-bit
// word, so each fragment register is one shared-memory load (the im part of
// a real-row column is the negated word).  Rows are XOR-swizzled so that the
// 32 lanes of a fragment load hit 32 banks.
// kShort (windows of at most 16 spectra: one row block) reads the fragments
// where the MMAs use them instead of holding all four tiles in registers,
// which leaves room for twice the resident CTAs.
// For one source the arithmetic (weights, fragments, MMA chain, hi + lo
// combination, window sum order) is that of tracker_stream_kernel, so
// results agree bit for bit (split(-x) is -split(x) except for the sign of a
// zero part, and the powers are sums of squares).
template <int A>
struct TrackerFrag {
    static constexpr int kWords = A / 2;         // 32-bit words of a part row
    static constexpr int kRowWords = kWords + 4;  // row pitch: 16 bytes of padding
    static constexpr int kBytes = A / 4;         // antennas per k-pair quad (lane q)
    // word of part row r holding antennas (a, a + 2), a % 4 in {0, 1}:
    // a = q kBytes + 4 jj + 2 h + s lies in 16-byte chunk 2 jj + s, word q,
    // half h, so one B fragment register of all four quads is one chunk.  The
    // padded pitch puts the same chunk of eight consecutive rows (what one
    // ldmatrix reads) on eight different bank groups, and leaves every row
    // offset a compile-time constant for the weight writer.
    __device__ static int lane_word(int a) { return 4 * ((((a % kBytes) >> 2) << 1) | (a & 1)) + a / kBytes; }
    __device__ static int word(int r, int a) { return r * kRowWords + lane_word(a); }
    __device__ static int half(int a) { return (a >> 1) & 1; }
};

// Four 8x8 b16 matrices from shared memory; lane L gives the address of row
// L % 8 of matrix L / 8, and thread t receives word t % 4 of row t / 4.
__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr)
                 : "memory");
}

template <int A, bool kShort>
__global__ void __launch_bounds__(256, kShort ? 4 : 2)
served_tracker_kernel(const uint8_t* __restrict__ pool, long long row_stride, const TableHeader* table) {
    constexpr int NW = A / 16;          // 32-bit words per thread per spectrum
    constexpr int kBytes = A / 4;       // bytes (antennas) per thread per spectrum
    using Frag = TrackerFrag<A>;
    constexpr int kWarpWords = 8 * 4 * Frag::kRowWords;  // 8 sources x 4 parts
    __shared__ double s_delay[2][8][A];  // by unit parity
    __shared__ __align__(16) uint32_t s_frag[8][kWarpWords];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const TrJob* jobs = reinterpret_cast<const TrJob*>(table + 1);
    const long long n_units = table->n_units;
    const int n_jobs = table->n_jobs;
    uint32_t* frag = s_frag[warp];
    // fragment column g of tile nt: part row 8 nt + g (part g & 3 of source
    // 2 nt + (g >> 2)); the xi word takes the other component (row
    // 8 nt + (g ^ 1)), negated for the real columns.  One ldmatrix per
    // (nt, jj) loads (xr, xi) for s = 0 and s = 1: lane L addresses row
    // L % 8 of matrix L / 8 = (s, re / im).  Columns of sources a unit does
    // not have read stale rows; their sums are never stored.
    const uint32_t neg_i = (g & 1) != 0 ? 0u : 0x80008000u;
    const int lrow = (lane & 8) != 0 ? ((lane & 7) ^ 1) : (lane & 7);
    const int ls = lane >> 4;
    const uint32_t frag_sa =
        static_cast<uint32_t>(__cvta_generic_to_shared(frag)) + 4u * (lrow * Frag::kRowWords + 4 * ls);
    auto frag_load = [&](int nt, int jj, uint32_t& b0r, uint32_t& b0i, uint32_t& b1r, uint32_t& b1i) {
        ldsm_x4(frag_sa + 4u * (8 * nt * Frag::kRowWords + 8 * jj), b0r, b0i, b1r, b1i);
        b0i ^= neg_i;
        b1i ^= neg_i;
    };
    // A CTA takes a contiguous range of units and walks it with a cursor
    // (source group, then channel group, then window, then job): one job
    // search and two 32-bit divisions per CTA instead of per unit.
    const long long u_begin = n_units * blockIdx.x / gridDim.x;
    const long long u_end = n_units * (blockIdx.x + 1) / gridDim.x;
    int j = 0, sg = 0, fg = 0, w = 0;
    auto seek = [&](long long u) {
        j = find_job(&jobs[0].unit_begin, sizeof(TrJob) / sizeof(long long), n_jobs, u);
        const unsigned local = static_cast<unsigned>(u - jobs[j].unit_begin);  // units of one job fit 32 bits
        const unsigned sgn = static_cast<unsigned>(jobs[j].src_groups), fgn = static_cast<unsigned>(jobs[j].fgroups);
        const unsigned rest = local / sgn, wq = rest / fgn;
        sg = static_cast<int>(local - rest * sgn);
        fg = static_cast<int>(rest - wq * fgn);
        w = static_cast<int>(wq);
    };
    if (u_begin < u_end) seek(u_begin);
    for (long long u = u_begin; u < u_end; ++u) {
        if (u > u_begin) {
            if (++sg == jobs[j].src_groups) {
                sg = 0;
                if (++fg == jobs[j].fgroups) {
                    fg = 0;
                    if (++w == jobs[j].n_win) seek(u);  // the next job with units
                }
            }
        }
        const TrJob& jb = jobs[j];
        const int f = fg * 8 + warp;
        const bool fvalid = f < jb.n_freq;
        const int n_src = jb.n_src, S = jb.spectra;
        const int n_here = min(8, n_src - 8 * sg);
        const int n_tiles = (n_here + 1) / 2;
        const long long wglob = static_cast<long long>(jb.w0) + w;

        const int t_begin = w * S, t_end = t_begin + S;  // rows of this launch
        const uint8_t* base = pool + static_cast<size_t>(f) * A + q * kBytes;
        auto load_rows = [&](int tb, uint32_t (&wg)[NW], uint32_t (&wg8)[NW]) {
            const int tg = tb + g, tg8 = tb + g + 8;
            const uint8_t* rg = base + (jb.t0 + tg) * row_stride;
            const uint8_t* rg8 = base + (jb.t0 + tg8) * row_stride;
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
        // the window's first rows are in flight while the weights are formed
        uint32_t wg[NW], wg8[NW];
        load_rows(t_begin, wg, wg8);

        // One barrier per unit: the delays alternate between two buffers, and a
        // warp writing this unit's buffer has passed the last unit's barrier,
        // which every warp reaches only after forming its weights from this
        // buffer two units ago.
        const int db = static_cast<int>((u - u_begin) & 1);
        for (int i = threadIdx.x; i < n_here * A; i += blockDim.x) {
            const int sl = i / A, a = i % A;
            const float3 d = trajectory_direction(jb.traj + 4 * (8 * sg + sl), wglob * S);
            s_delay[db][sl][a] = steering_delay(jb.pos, a, d.x, d.y, d.z);
        }
        __syncthreads();
        if (fvalid) {
            // lane owns antennas lane + 32 c (its 16-bit slot in every part row
            // fixed); sources go in pairs, each row's offset a constant
            const double k = jb.kw[f];
            uint16_t* slot[A / 32];
#pragma unroll
            for (int c = 0; c < A / 32; ++c) {
                const int a = lane + 32 * c;
                slot[c] = reinterpret_cast<uint16_t*>(frag) + 2 * Frag::lane_word(a) + Frag::half(a);
            }
#pragma unroll 1
            for (int sl0 = 0; sl0 < n_here; sl0 += 2) {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    if (sl0 + e < n_here) {
#pragma unroll
                        for (int c = 0; c < A / 32; ++c) {
                            const float2 wv = steering_from_delay(k, s_delay[db][sl0 + e][lane + 32 * c]);
                            // the parts split_part forms, two per packed conversion
                            const __half2 hi = __floats2half2_rn(wv.x, wv.y);
                            const float2 hf = __half22float2(hi);
                            const uint32_t hw = h2_bits(hi);
                            const uint32_t lw = h2_bits(__floats2half2_rn(__fsub_rn(wv.x, hf.x), __fsub_rn(wv.y, hf.y)));
                            uint16_t* r0 = slot[c] + 2 * (sl0 + e) * 4 * Frag::kRowWords;  // part rows 4 (sl0 + e) ..
                            r0[0] = static_cast<uint16_t>(hw);
                            r0[2 * Frag::kRowWords] = static_cast<uint16_t>(hw >> 16);
                            r0[4 * Frag::kRowWords] = static_cast<uint16_t>(lw);
                            r0[6 * Frag::kRowWords] = static_cast<uint16_t>(lw >> 16);
                        }
                    }
                }
            }
        }
        __syncwarp();

        // B fragments of the long form: column g of tile nt is (re, im) x
        // (hi, lo) of source 8 sg + 2 nt + (g >> 2).
        uint32_t bfrag[kShort ? 1 : 4][NW][2][2];
        if constexpr (!kShort) {
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
                for (int jj = 0; jj < NW; ++jj) {
                    frag_load(nt, jj, bfrag[nt][jj][0][0], bfrag[nt][jj][0][1], bfrag[nt][jj][1][0],
                              bfrag[nt][jj][1][1]);
                }
            }
        }

        float pw[4] = {0.f, 0.f, 0.f, 0.f};
        for (int tb = t_begin; tb < t_end; tb += 16) {
            uint32_t ng[NW], ng8[NW];
            if constexpr (!kShort) load_rows(tb + 16, ng, ng8);
            float d[4][4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
#pragma unroll
            for (int jj = 0; jj < NW; ++jj) {
                uint32_t re02g, im02g, re13g, im13g, re02h, im02h, re13h, im13h;
                decode_word(wg[jj], re02g, im02g, re13g, im13g);
                decode_word(wg8[jj], re02h, im02h, re13h, im13h);
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    if (nt < n_tiles) {
                        if constexpr (kShort) {
                            uint32_t b0r, b0i, b1r, b1i;
                            frag_load(nt, jj, b0r, b0i, b1r, b1i);
                            mma_16816(d[nt], re02g, re02h, im02g, im02h, b0r, b0i);
                            mma_16816(d[nt], re13g, re13h, im13g, im13h, b1r, b1i);
                        } else {
                            mma_16816(d[nt], re02g, re02h, im02g, im02h, bfrag[nt][jj][0][0], bfrag[nt][jj][0][1]);
                            mma_16816(d[nt], re13g, re13h, im13g, im13h, bfrag[nt][jj][1][0], bfrag[nt][jj][1][1]);
                        }
                    }
                }
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                if (nt < n_tiles) {
                    // q == 0 / 2 hold (re_hi, im_hi) of the tile's first / second
                    // source, q == 1 / 3 the lo parts, for rows g and g + 8
                    float p[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) p[i] = __shfl_xor_sync(0xffffffffu, d[nt][i], 1);
                    const float re_g = d[nt][0] + p[0], im_g = d[nt][1] + p[1];
                    const float re_h = d[nt][2] + p[2], im_h = d[nt][3] + p[3];
                    const float pow_g = re_g * re_g + im_g * im_g;
                    const float pow_h = re_h * re_h + im_h * im_h;
                    pw[nt] += pow_g + pow_h;
                }
            }
            if constexpr (!kShort) {
#pragma unroll
                for (int jj = 0; jj < NW; ++jj) {
                    wg[jj] = ng[jj];
                    wg8[jj] = ng8[jj];
                }
            }
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            if (nt < n_tiles) {
                float acc = pw[nt];
                acc += __shfl_xor_sync(0xffffffffu, acc, 4);
                acc += __shfl_xor_sync(0xffffffffu, acc, 8);
                acc += __shfl_xor_sync(0xffffffffu, acc, 16);
                const int src = 8 * sg + 2 * nt + (q >> 1);
                if (g == 0 && (q & 1) == 0 && fvalid && src < n_src) {
                    jb.integrated[(wglob * jb.n_freq + f) * n_src + src] = acc;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(256) served_quantize_kernel(const TableHeader* table) {
    const QJob* jobs = reinterpret_cast<const QJob*>(table + 1);
    const long long n_units = table->n_units;
    const int n_jobs = table->n_jobs;
    const int lane = threadIdx.x & 31;
    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    for (long long u = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); u < n_units;
         u += warps) {
        const int j = find_job(&jobs[0].unit_begin, sizeof(QJob) / sizeof(long long), n_jobs, u);
        const QJob& jb = jobs[j];
        unsigned local = static_cast<unsigned>(u - jb.unit_begin);  // chunks of one job fit 32 bits
        const int bt = static_cast<int>(local % static_cast<unsigned>(jb.btiles));
        local /= static_cast<unsigned>(jb.btiles);
        const int ft = static_cast<int>(local % static_cast<unsigned>(jb.ftiles));
        local /= static_cast<unsigned>(jb.ftiles);
        const int w = static_cast<int>(local % static_cast<unsigned>(jb.n_win));
        const int shard = static_cast<int>(local / static_cast<unsigned>(jb.n_win));
        const int win = jb.w0 + w;
        const size_t shard_off = static_cast<size_t>(shard) * jb.n_windows * jb.n_freq * jb.n_beams;
        const size_t pidx = ((static_cast<size_t>(shard) * jb.n_windows + win) * jb.ftiles + ft) * jb.btiles + bt;
        quantize_chunk<false>(jb.integrated + shard_off, jb.codes + shard_off, jb.params, pidx, win, jb.n_freq,
                              jb.n_beams, ft, bt, lane);
    }
}

}  // namespace

bf_status launch_generate_weights(cudaStream_t stream, const float* pos, const float* freq, const float* dirs,
                                  float* out, uint64_t n_shards, uint64_t f_shard, uint64_t n_beams,
                                  uint64_t n_ant) {
    const uint64_t total = n_shards * n_beams * f_shard * n_ant;
    if (total == 0) return BF_OK;
    if (total > (1ull << 40)) return set_error(BF_ERR_OVERFLOW, "weight array exceeds the supported size");
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((total + 255) / 256, 148ull * 16));
    weights_kernel<<<blocks, 256, 0, stream>>>(pos, freq, dirs, reinterpret_cast<float2*>(out),
                                               static_cast<int>(n_shards), static_cast<int>(f_shard),
                                               static_cast<int>(n_beams), static_cast<int>(n_ant));
    return cuda_status(cudaGetLastError(), "weights_kernel launch");
}

bf_status launch_served_tracker(cudaStream_t stream, int n_ant, bool short_windows, const uint8_t* pool,
                                uint64_t pool_freq, const TableHeader* table, int grid) {
    const long long row_stride = static_cast<long long>(pool_freq) * n_ant;
    if (n_ant != 32 && n_ant != 64) return set_error(BF_ERR_UNSUPPORTED, "served trackers support n_ant 32 or 64");
    if (n_ant == 32) {
        if (short_windows) served_tracker_kernel<32, true><<<grid, 256, 0, stream>>>(pool, row_stride, table);
        else served_tracker_kernel<32, false><<<grid, 256, 0, stream>>>(pool, row_stride, table);
    } else {
        if (short_windows) served_tracker_kernel<64, true><<<grid, 256, 0, stream>>>(pool, row_stride, table);
        else served_tracker_kernel<64, false><<<grid, 256, 0, stream>>>(pool, row_stride, table);
    }
    return cuda_status(cudaGetLastError(), "served_tracker_kernel launch");
}

bf_status launch_served_quantize(cudaStream_t stream, const TableHeader* table, int grid) {
    served_quantize_kernel<<<grid, 256, 0, stream>>>(table);
    return cuda_status(cudaGetLastError(), "served_quantize_kernel launch");
}

}  // namespace bf
