// doa_scan.cu -- FP64 direction-of-arrival stages on the GPU.
//
// From the exact per-block INT32 covariances of doa_cov.cu, for each
// frequency channel f and block b in order (reference
// src/cpu_opt_beam_tracker.cpp, restated in FP64):
//   smoothing     R~[r][c] = (1/L) sum_s R[s+r][s+c] / K over the L = A-M+1
//                 sub-arrays along the linear element index (:605-657)
//   fwd-backward  R^ = (R~ + J conj(R~) J) / 2 when smoothing (:645-657)
//   loading       eps = load * tr(R^) / M, added to the diagonal (:226-237)
//   forgetting    S = lam S + (1 - lam) R^, E = lam E + (1 - lam) eps
//                 (first block: S = R^, E = eps) (:1763-1892)
//   Cholesky      L L^H = S + E I, FP64 (:398-415)
//   scan          Bartlett a^H S a (:287-302), Capon 1 / ||L^-1 a||^2
//                 (:423-437), a_i = exp(-j k_f (x_i l + y_i m)) (:96-106),
//                 summed over frequency in channel order
//   peak          argmax and the vertex of the parabola through it and its
//                 neighbours (concave case).
// FP64 is used for the phase argument before its reduction to a quadrant,
// the forgetting accumulation and the loaded Cholesky solve; the reduced
// phase goes through the FP32 Taylor sin / cos of tracker_common.cuh.
#include "bf_internal.cuh"
#include "tracker_common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

namespace bf {
namespace {

constexpr int kMaxM = 16;

struct Cd {
    double re, im;
};

// Fold of the (block, channel) cells, per cell and element:
//   smooth_warp      smoothing over the L = A - M + 1 sub-arrays and 1/K;
//   loading_eps      eps = load * tr / M of the forward-backward average;
//   fb_elems         forward-backward average R^ = (R~ + J conj(R~) J) / 2;
//   forget_step      S = lam S + (1 - lam) R^ (first block: S = R^), and the
//                    same recursion for E;
//   cholesky_warp    L L^H = S + E I by one warp;
//   inverse_column   column j of L^{-1} by forward substitution;
//   q_elem           Q = L^{-H} L^{-1} = (S + E I)^{-1}, so the scan
//                    evaluates Capon's |L^{-1} a|^2 as the quadratic form a^H Q a.
// Two schedules share them (same operations in the same order, so the same
// results): doa_fold_kernel, one CTA per channel walking its blocks in chunks
// with one warp per cell, for sequences of up to kFoldChunks chunks over at
// least one channel per SM; and three launches otherwise, where only the
// forgetting recursion is serial --
// doa_smooth_kernel and doa_factor_kernel over all cells, doa_forget_kernel
// per channel.

// Smoothing of one cell by one warp.  R~[r][c] sums R[s + r][s + c] over
// s < L: entry R[t][t + d] belongs to the elements (r, r + d) with
// r <= t < r + L, so the warp reads R's band |u - t| < M row by row (2M - 1
// contiguous entries of a row, one per lane, RB rows in flight) and
// each lane takes its elements' entries by shuffle.  The sums are of
// integers, exact in int64, so the row order does not change them.  NE is
// the count of elements per lane (at least (M^2 + 31) / 32), RB the rows
// loaded at once.
template <int NE, int RB>
__device__ __forceinline__ void smooth_warp(const int32_t* __restrict Rf, int A, int M, int K, Cd* Rt, int lane) {
    const int L = A - M + 1;
    long long ar[NE], ai[NE];
    int src[NE], r0[NE];
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        const int e = lane + 32 * k;
        const int r = e / M, c = e % M;
        ar[k] = ai[k] = 0;
        src[k] = e < M * M ? c - r + M - 1 : 0;
        r0[k] = e < M * M ? r : A;  // past every row: never adds
    }
    const int2* R2 = reinterpret_cast<const int2*>(Rf);
    const bool loads = lane < 2 * M - 1;
    for (int t0 = 0; t0 < A; t0 += RB) {
        int2 v[RB];
#pragma unroll
        for (int i = 0; i < RB; ++i) {
            const int t = t0 + i, u = t - (M - 1) + lane;
            v[i] = loads && t < A && u >= 0 && u < A ? R2[t * A + u] : make_int2(0, 0);
        }
#pragma unroll
        for (int i = 0; i < RB; ++i) {
            const int t = t0 + i;
#pragma unroll
            for (int k = 0; k < NE; ++k) {
                const int x = __shfl_sync(0xffffffffu, v[i].x, src[k]);
                const int y = __shfl_sync(0xffffffffu, v[i].y, src[k]);
                if (r0[k] <= t && t < r0[k] + L) {
                    ar[k] += x;
                    ai[k] += y;
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        const int e = lane + 32 * k;
        if (e < M * M) Rt[e] = Cd{static_cast<double>(ar[k]) / K / L, static_cast<double>(ai[k]) / K / L};
    }
}

__device__ __forceinline__ double loading_eps(const Cd* Rt, int M, int L, double load) {
    double tr = 0.0;
    for (int r = 0; r < M; ++r) {
        const Cd x = Rt[r * M + r];
        tr += L > 1 ? 0.5 * (x.re + Rt[(M - 1 - r) * M + (M - 1 - r)].re) : x.re;
    }
    return load * tr / M;
}

__device__ __forceinline__ void fb_elems(const Cd* Rt, int M, int L, Cd* out, int e0, int step) {
    for (int e = e0; e < M * M; e += step) {
        const int r = e / M, c = e % M;
        Cd x = Rt[e];
        if (L > 1) {
            const Cd y = Rt[(M - 1 - r) * M + (M - 1 - c)];
            x = Cd{0.5 * (x.re + y.re), 0.5 * (x.im - y.im)};
        }
        out[e] = x;
    }
}

__device__ __forceinline__ Cd forget_step(bool first, double lam, Cd s, Cd x) {
    return (first || lam >= 1.0) ? x : Cd{lam * s.re + (1.0 - lam) * x.re, lam * s.im + (1.0 - lam) * x.im};
}

__device__ __forceinline__ double forget_step(bool first, double lam, double acc, double eps) {
    return (first || lam >= 1.0) ? eps : lam * acc + (1.0 - lam) * eps;
}

// Right-looking Cholesky of S + E I by one warp: step j takes the square root
// of the updated diagonal, lanes i > j scale column j and update their own row
// i of the trailing lower triangle.  Returns (warp-uniformly) 1 when every
// pivot is positive.
__device__ __forceinline__ int cholesky_warp(const Cd* S, double E, int M, Cd* Lc, int lane) {
    for (int e = lane; e < M * M; e += 32) {
        const int i = e / M, j = e % M;
        Lc[e] = j <= i ? Cd{S[e].re + (i == j ? E : 0.0), S[e].im} : Cd{0.0, 0.0};
    }
    __syncwarp();
    int good = 1;
    for (int j = 0; j < M; ++j) {
        const double djj = Lc[j * M + j].re;
        if (!(djj > 1e-300)) { good = 0; break; }
        const double ljj = sqrt(djj);
        __syncwarp();
        if (lane == j) Lc[j * M + j] = Cd{ljj, 0.0};
        if (lane > j && lane < M) {
            const Cd x = Lc[lane * M + j];
            Lc[lane * M + j] = Cd{x.re / ljj, x.im / ljj};
        }
        __syncwarp();
        if (lane > j && lane < M) {
            const Cd lij = Lc[lane * M + j];
            for (int k = j + 1; k <= lane; ++k) {
                const Cd lkj = Lc[k * M + j];  // row lane -= l_ij * conj(l_kj)
                Cd& w = Lc[lane * M + k];
                w = Cd{w.re - (lij.re * lkj.re + lij.im * lkj.im), w.im - (lij.im * lkj.re - lij.re * lkj.im)};
            }
        }
        __syncwarp();
    }
    return good;
}

__device__ __forceinline__ void inverse_column(const Cd* Lc, int M, Cd* Li, int j) {
    for (int i = 0; i < j; ++i) Li[i * M + j] = Cd{0.0, 0.0};
    Li[j * M + j] = Cd{1.0 / Lc[j * M + j].re, 0.0};
    for (int i = j + 1; i < M; ++i) {
        double sr = 0.0, si = 0.0;
        for (int k = j; k < i; ++k) {
            const Cd x = Lc[i * M + k], y = Li[k * M + j];
            sr += x.re * y.re - x.im * y.im;
            si += x.re * y.im + x.im * y.re;
        }
        const double d = Lc[i * M + i].re;
        Li[i * M + j] = Cd{-sr / d, -si / d};
    }
}

__device__ __forceinline__ Cd q_elem(const Cd* Li, int M, int e) {
    const int i = e / M, j = e % M;
    double qr = 0.0, qi = 0.0;
    for (int k = i > j ? i : j; k < M; ++k) {
        const Cd x = Li[k * M + i], y = Li[k * M + j];  // conj(x) * y
        qr += x.re * y.re + x.im * y.im;
        qi += x.re * y.im - x.im * y.re;
    }
    return Cd{qr, qi};
}

// Three-launch schedule: the averaged matrix is parked in the Q slot of the
// workspace between doa_smooth_kernel and doa_forget_kernel.
__global__ void doa_smooth_kernel(const int32_t* __restrict R, int n_freq, int A, int M, int K,
                                  double load, Cd* __restrict Rhat_out, double* __restrict eps_out) {
    const int f = blockIdx.x, b = blockIdx.y;
    __shared__ Cd Rt[kMaxM * kMaxM];
    const int L = A - M + 1;
    const size_t cell = static_cast<size_t>(b) * n_freq + f;
    smooth_warp<kMaxM * kMaxM / 32, 8>(R + cell * A * A * 2, A, M, K, Rt, threadIdx.x);
    __syncwarp();
    if (threadIdx.x == 0) eps_out[cell] = loading_eps(Rt, M, L, load);
    fb_elems(Rt, M, L, Rhat_out + cell * M * M, threadIdx.x, 32);
}

__global__ void doa_forget_kernel(const Cd* __restrict Rhat, int n_blocks, int n_freq, int M, double lam,
                                  Cd* __restrict S_out, double* __restrict E) {
    const int f = blockIdx.x;
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) {
        Cd s{0.0, 0.0};
        for (int b = 0; b < n_blocks; ++b) {
            const size_t at = (static_cast<size_t>(b) * n_freq + f) * M * M + e;
            s = forget_step(b == 0, lam, s, Rhat[at]);
            S_out[at] = s;
        }
    }
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int b = 0; b < n_blocks; ++b) {
            const size_t cell = static_cast<size_t>(b) * n_freq + f;
            acc = forget_step(b == 0, lam, acc, E[cell]);
            E[cell] = acc;
        }
    }
}

__global__ void doa_factor_kernel(const Cd* __restrict S_in, const double* __restrict E_in, int n_freq, int M,
                                  Cd* __restrict Q_out, int* __restrict ok_out) {
    const int f = blockIdx.x, b = blockIdx.y;
    const size_t cell = static_cast<size_t>(b) * n_freq + f;
    const size_t base = cell * M * M;
    __shared__ Cd S[kMaxM * kMaxM];
    __shared__ Cd Lc[kMaxM * kMaxM];
    __shared__ Cd Li[kMaxM * kMaxM];
    __shared__ int ok;
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) S[e] = S_in[base + e];
    __syncthreads();
    if (threadIdx.x < 32) {
        const int good = cholesky_warp(S, E_in[cell], M, Lc, threadIdx.x);
        if (threadIdx.x == 0) {
            ok = good;
            ok_out[cell] = good;
        }
    }
    __syncthreads();
    if (ok && threadIdx.x < M) inverse_column(Lc, M, Li, threadIdx.x);
    __syncthreads();
    for (int e = threadIdx.x; e < M * M; e += blockDim.x) Q_out[base + e] = ok ? q_elem(Li, M, e) : Cd{0.0, 0.0};
}

// One-launch schedule: a CTA per channel takes its blocks fold_cells<M>() at a
// time, one warp per cell.  Per chunk: each warp smooths, averages and loads
// its cell; the CTA's threads carry the forgetting recursion (S element by
// element, E in one thread) through the chunk's blocks in order, in registers
// across chunks; each warp then factors its cell.  Chunks of 8 cells up to 11
// elements, 4 above (at most 32 KB of shared memory).
__host__ __device__ constexpr int fold_cells_for(int M) { return M <= 11 ? 8 : 4; }
template <int M>
__host__ __device__ constexpr int fold_cells() { return fold_cells_for(M); }
constexpr int kFoldChunks = 8;

template <int M>
__global__ void __launch_bounds__(32 * fold_cells<M>(), 3)
doa_fold_kernel(const int32_t* __restrict R, int n_blocks, int n_freq, int A, int K, double lam, double load,
                Cd* __restrict S_out, Cd* __restrict Q_out, double* __restrict E_out, int* __restrict ok_out) {
    constexpr int CH = fold_cells<M>(), MM = M * M, kThreads = 32 * CH;
    constexpr int kCarry = (MM + kThreads - 1) / kThreads;
    __shared__ Cd sh_a[CH][MM];  // R~, then L
    __shared__ Cd sh_b[CH][MM];  // R^, then S, then L^{-1}
    __shared__ double sh_e[CH];
    const int f = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = A - M + 1;
    Cd s_carry[kCarry];
#pragma unroll
    for (int k = 0; k < kCarry; ++k) s_carry[k] = Cd{0.0, 0.0};
    double e_carry = 0.0;
    for (int b0 = 0; b0 < n_blocks; b0 += CH) {
        const int b = b0 + warp, nb = min(CH, n_blocks - b0);
        const size_t cell = static_cast<size_t>(b) * n_freq + f;
        if (b < n_blocks) {
            smooth_warp<(MM + 31) / 32, 8>(R + cell * A * A * 2, A, M, K, sh_a[warp], lane);
            __syncwarp();
            if (lane == 0) sh_e[warp] = loading_eps(sh_a[warp], M, L, load);
            fb_elems(sh_a[warp], M, L, sh_b[warp], lane, 32);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kCarry; ++k) {
            const int e = threadIdx.x + k * kThreads;
            if (e < MM) {
                Cd s = s_carry[k];
                for (int w = 0; w < nb; ++w) {
                    s = forget_step(b0 + w == 0, lam, s, sh_b[w][e]);
                    sh_b[w][e] = s;
                    S_out[(static_cast<size_t>(b0 + w) * n_freq + f) * MM + e] = s;
                }
                s_carry[k] = s;
            }
        }
        if (threadIdx.x == kThreads - 1) {
            double acc = e_carry;
            for (int w = 0; w < nb; ++w) {
                acc = forget_step(b0 + w == 0, lam, acc, sh_e[w]);
                sh_e[w] = acc;
                E_out[static_cast<size_t>(b0 + w) * n_freq + f] = acc;
            }
            e_carry = acc;
        }
        __syncthreads();
        if (b < n_blocks) {
            const int good = cholesky_warp(sh_b[warp], sh_e[warp], M, sh_a[warp], lane);
            if (lane == 0) ok_out[cell] = good;
            __syncwarp();  // S is consumed: its slot takes L^{-1}
            if (good && lane < M) inverse_column(sh_a[warp], M, sh_b[warp], lane);
            __syncwarp();
            for (int e = lane; e < MM; e += 32) Q_out[cell * MM + e] = good ? q_elem(sh_b[warp], M, e) : Cd{0.0, 0.0};
        }
        __syncthreads();
    }
}

// A CTA of 8 warps takes 32 grid points and KB blocks (scan_blocks: 8 in the
// uniform form; 4, or 2 above 13 elements, in the general form): lane = grid
// point, warp w the channels f = 8 s + w of step s.  The steering vector of
// (channel, point) is formed once and used
// for the KB blocks.  Bartlett a^H S a and Capon 1 / (a^H Q a),
// Q = (S + eps I)^{-1}, are Hermitian quadratic forms (diagonal plus twice
// the real part of the upper triangle); the upper triangles of S and Q for
// the next step's 8 channels x KB blocks are staged into shared memory with
// cp.async while the current step computes.
// The channel steps split over the z extent of the grid, a thread-block
// cluster of up to 8 CTAs, so that the grid fills the GPU's resident CTA
// slots; each CTA adds its warps' partial sums in warp order, and cluster
// rank 0 adds the CTAs' sums in rank order through distributed shared
// memory (a fixed order: results are deterministic for a given split).
constexpr int kScanWarps = 8;
constexpr int kMaxSplit = 8;

// Blocks per CTA: each (channel, grid point) steering vector serves this many
// blocks.  The uniform form stages 4M - 2 doubles per cell and takes 8; the
// general form stages the triangles of S and Q, 4 (2 above 13 elements).
template <int M, bool kUniform>
__host__ __device__ constexpr int scan_blocks() { return kUniform ? 8 : M <= 13 ? 4 : 2; }

// Uniform sub-array form.  With p_m = p_0 + m D + e_m (D = (p_{M-1} - p_0) /
// (M - 1), e_m the residuals of the float positions) and psi = k D.d,
//   conj(a_r) a_c = exp(-i (c - r) psi) exp(i k (e_r - e_c).d)
// and to first order in theta = k (e_r - e_c).d each Hermitian quadratic
// form is
//   a^H X a = T_0 + 2 Re sum_{s=1}^{M-1} exp(-i s psi) T_s,
//   T_0 = sum_r X_rr,  T_s = sum_r X_{r,r+s} (1 + i k (e_r - e_{r+s}).d),
// with d.e = e_x l + e_y m.  T_s = A_s + l B_s per (block, channel) cell,
// so a grid point costs 2 (M - 1) products per form instead of M (M + 1) / 2
// complex ones.  The form is used when k_max max_m (|e_x,m| |l|_max +
// |e_y,m| |m|) <= 1e-4, where the neglected second-order term is below
// 5e-9 relative; any other geometry takes the general form.
constexpr double kFirstOrderBound = 1e-4;

struct ArrayInfo {
    double dx, dy;
    double ex[kMaxM], ey[kMaxM];
    int uniform;
};

// coefficient doubles per form: T_0, then (A_s.re, A_s.im, B_s.re, B_s.im)
// for s = 1 .. M - 1, padded to an even count (16-byte staging)
__host__ __device__ constexpr int coef_per_form(int M) { return 4 * M - 2; }

__global__ void doa_array_kernel(const float* __restrict pos, const double* __restrict kw, int M, int n_freq,
                                 double l_abs_max, double m_fixed, ArrayInfo* __restrict info) {
    const int lane = threadIdx.x;
    double kmax = 0.0;
    for (int f = lane; f < n_freq; f += 32) kmax = fmax(kmax, fabs(kw[f]));
    for (int o = 16; o > 0; o >>= 1) kmax = fmax(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    if (lane != 0) return;
    ArrayInfo a{};
    a.uniform = 0;
    if (M >= 2) {
        const double x0 = pos[0], y0 = pos[1];
        a.dx = (static_cast<double>(pos[3 * (M - 1)]) - x0) / (M - 1);
        a.dy = (static_cast<double>(pos[3 * (M - 1) + 1]) - y0) / (M - 1);
        double theta = 0.0;
        for (int m = 0; m < M; ++m) {
            a.ex[m] = static_cast<double>(pos[3 * m]) - x0 - m * a.dx;
            a.ey[m] = static_cast<double>(pos[3 * m + 1]) - y0 - m * a.dy;
            theta = fmax(theta, kmax * (fabs(a.ex[m]) * l_abs_max + fabs(a.ey[m]) * fabs(m_fixed)));
        }
        // differences e_r - e_c reach twice a single residual
        a.uniform = 2.0 * theta <= kFirstOrderBound ? 1 : 0;
    }
    *info = a;
}

// Per (block, channel) cell: the coefficients of the Bartlett (S) and
// Capon (Q) forms in the uniform sub-array form.
__global__ void doa_coef_kernel(const Cd* __restrict S, const Cd* __restrict Q, const double* __restrict kw,
                                int n_freq, int M, double m_fixed, const ArrayInfo* __restrict info,
                                double* __restrict coef) {
    if (!info->uniform) return;
    const int f = blockIdx.x, b = blockIdx.y;
    const size_t cell = static_cast<size_t>(b) * n_freq + f;
    const int CQ = coef_per_form(M);
    const double k = kw[f];
    double* out = coef + cell * 2 * CQ;
    const int t = threadIdx.x;
    if (t < 2 * (M - 1)) {
        const int form = t / (M - 1), sft = 1 + t % (M - 1);
        const Cd* X = (form ? Q : S) + cell * M * M;
        double dr = 0.0, di = 0.0, gxr = 0.0, gxi = 0.0, gyr = 0.0, gyi = 0.0;
        for (int r = 0; r + sft < M; ++r) {
            const Cd x = X[r * M + r + sft];
            const double ex = info->ex[r] - info->ex[r + sft], ey = info->ey[r] - info->ey[r + sft];
            dr += x.re;
            di += x.im;
            gxr += x.re * ex;
            gxi += x.im * ex;
            gyr += x.re * ey;
            gyi += x.im * ey;
        }
        // A = D + i k m Gy,  B = i k Gx
        double* o = out + form * CQ + 1 + 4 * (sft - 1);
        o[0] = dr - k * m_fixed * gyi;
        o[1] = di + k * m_fixed * gyr;
        o[2] = -k * gxi;
        o[3] = k * gxr;
    } else if (t < 2 * (M - 1) + 2) {
        const int form = t - 2 * (M - 1);
        const Cd* X = (form ? Q : S) + cell * M * M;
        double tr = 0.0;
        for (int r = 0; r < M; ++r) tr += X[r * M + r].re;
        out[form * CQ] = tr;
        out[form * CQ + CQ - 1] = 0.0;
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <int M, bool kUniform>
__global__ void __launch_bounds__(kScanWarps * 32)
doa_scan_kernel(const Cd* __restrict S, const Cd* __restrict Q, const int* __restrict ok,
                const float* __restrict pos, const double* __restrict kw, int n_blocks, int n_freq,
                double l_first, double l_step, int n, double m_fixed, double* __restrict bartlett,
                double* __restrict capon, int steps_per_split, const ArrayInfo* __restrict info,
                const double* __restrict coef) {
    // the two forms are launched together; the array decides which one runs
    if ((info->uniform != 0) != kUniform) return;
    constexpr int kScanBlocks = scan_blocks<M, kUniform>();
    constexpr int U = M * (M + 1) / 2;                 // upper triangle incl. diagonal
    constexpr int CQ = coef_per_form(M);
    // Cd staged per warp and step: upper triangles of S and Q, or the two
    // forms' coefficients (2 CQ doubles = CQ Cd)
    constexpr int kPerWarp = kUniform ? kScanBlocks * CQ : kScanBlocks * 2 * U;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * 32 + lane;
    const int b0 = blockIdx.y * kScanBlocks;
    const int nb = min(kScanBlocks, n_blocks - b0);
    extern __shared__ Cd scan_stage[];                 // [2][warps][blocks][S | Q][U]
    __shared__ int s_ok[2][kScanWarps][kScanBlocks];
    __shared__ double red_b[kScanWarps][kScanBlocks][32], red_c[kScanWarps][kScanBlocks][32];
    __shared__ double fin_b[kScanBlocks][32], fin_c[kScanBlocks][32];
    const int n_steps = (n_freq + kScanWarps - 1) / kScanWarps;
    const int st_begin = static_cast<int>(blockIdx.z) * steps_per_split;
    const int st_end = min(n_steps, st_begin + steps_per_split);

    // stage step s: thread t copies elements t, t + 256, ... of the step
    auto stage = [&](int st, int buf) {
        Cd* dst = scan_stage + static_cast<size_t>(buf) * kScanWarps * kPerWarp;
        for (int i = threadIdx.x; i < kScanWarps * kPerWarp; i += blockDim.x) {
            const int w = i / kPerWarp, rem = i % kPerWarp;
            const int f = st * kScanWarps + w;
            if constexpr (kUniform) {
                const int bi = rem / CQ, e = rem % CQ;
                if (f >= n_freq || bi >= nb) continue;
                const size_t cell = static_cast<size_t>(b0 + bi) * n_freq + f;
                cp_async16(dst + i, reinterpret_cast<const Cd*>(coef) + cell * CQ + e);
            } else {
                const int bi = rem / (2 * U), which = (rem / U) & 1, t = rem % U;
                if (f >= n_freq || bi >= nb) continue;
                int r = 0, rest = t;  // upper-triangle index -> (r, c)
                while (rest >= M - r) { rest -= M - r; ++r; }
                const int c = r + rest;
                const size_t cell = static_cast<size_t>(b0 + bi) * n_freq + f;
                cp_async16(dst + i, (which ? Q : S) + cell * M * M + r * M + c);
            }
        }
        if (threadIdx.x < kScanWarps * kScanBlocks) {
            const int w = threadIdx.x / kScanBlocks, bi = threadIdx.x % kScanBlocks;
            const int f = st * kScanWarps + w;
            s_ok[buf][w][bi] = (f < n_freq && bi < nb) ? ok[static_cast<size_t>(b0 + bi) * n_freq + f] : 0;
        }
        cp_async_commit();
    };

    const double lv = l_first + static_cast<double>(l) * l_step;
    double pb[kScanBlocks], pc[kScanBlocks];
#pragma unroll
    for (int i = 0; i < kScanBlocks; ++i) pb[i] = pc[i] = 0.0;
    double px[M], py[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        px[i] = static_cast<double>(pos[3 * i]);
        py[i] = static_cast<double>(pos[3 * i + 1]);
    }
    stage(st_begin, st_begin & 1);
    for (int st = st_begin; st < st_end; ++st) {
        if (st + 1 < st_end) stage(st + 1, (st + 1) & 1);
        else cp_async_commit();  // keep one group per step for wait_group 1
        cp_async_wait_1();
        __syncthreads();
        const int f = st * kScanWarps + warp;
        if (kUniform && f < n_freq) {
            const double* base = reinterpret_cast<const double*>(
                scan_stage + (static_cast<size_t>(st & 1) * kScanWarps + warp) * kPerWarp);
            const double k = kw[f];
            constexpr double kHalfPi = 1.5707963267948966192313216916398;
            constexpr double kTwoOverPi = 0.63661977236758134307553505349006;
            // exp(-i s psi) = (cos, -sin) of s psi, s = 1 .. M - 1
            const double psi = k * (info->dx * lv + info->dy * m_fixed);
            double zc[M], zs[M];
#pragma unroll
            for (int sft = 1; sft < M; ++sft) {
                const double ph = static_cast<double>(sft) * psi;
                int qd;
                const double q = trk::round_quadrant(ph * kTwoOverPi, qd);
                const float2 w = trk::sincos_quadrant(__double2float_rn(__fma_rn(-kHalfPi, q, ph)), qd);
                zc[sft] = static_cast<double>(w.x);
                zs[sft] = static_cast<double>(w.y);
            }
            // T_0 + 2 sum_s Re(exp(-i s psi) (A_s + l B_s))
            auto form = [&](const double* c) {
                double acc = 0.0;
#pragma unroll
                for (int sft = 1; sft < M; ++sft) {
                    const double* t = c + 1 + 4 * (sft - 1);
                    const double tre = t[0] + lv * t[2], tim = t[1] + lv * t[3];
                    acc += zc[sft] * tre + zs[sft] * tim;
                }
                return c[0] + 2.0 * acc;
            };
#pragma unroll
            for (int bi = 0; bi < kScanBlocks; ++bi) {
                if (bi < nb) {
                    pb[bi] += form(base + bi * 2 * CQ);
                    if (s_ok[st & 1][warp][bi]) {
                        const double q = form(base + bi * 2 * CQ + CQ);
                        pc[bi] += q > 0.0 ? 1.0 / q : 0.0;
                    }
                }
            }
        } else if (!kUniform && f < n_freq) {
            const Cd* base = scan_stage + (static_cast<size_t>(st & 1) * kScanWarps + warp) * kPerWarp;
            Cd a[M];
            double mag[M];
            const double k = kw[f];
#pragma unroll
            for (int i = 0; i < M; ++i) {
                constexpr double kHalfPi = 1.5707963267948966192313216916398;
                constexpr double kTwoOverPi = 0.63661977236758134307553505349006;
                const double ph = k * (px[i] * lv + py[i] * m_fixed);
                int qd;
                const double q = trk::round_quadrant(ph * kTwoOverPi, qd);
                const float2 w = trk::sincos_quadrant(__double2float_rn(__fma_rn(-kHalfPi, q, ph)), qd);
                a[i] = Cd{static_cast<double>(w.x), -static_cast<double>(w.y)};
                mag[i] = a[i].re * a[i].re + a[i].im * a[i].im;
            }
            auto quad = [&](const Cd* X) {
                double diag = 0.0, off = 0.0;
                int t = 0;
#pragma unroll
                for (int r = 0; r < M; ++r) {
                    diag += X[t].re * mag[r];
                    ++t;
                    double tr = 0.0, ti = 0.0;
#pragma unroll
                    for (int c = r + 1; c < M; ++c, ++t) {
                        const Cd x = X[t];
                        tr += x.re * a[c].re - x.im * a[c].im;
                        ti += x.re * a[c].im + x.im * a[c].re;
                    }
                    off += a[r].re * tr + a[r].im * ti;
                }
                return diag + 2.0 * off;
            };
#pragma unroll
            for (int bi = 0; bi < kScanBlocks; ++bi) {
                if (bi < nb) {
                    pb[bi] += quad(base + bi * 2 * U);
                    if (s_ok[st & 1][warp][bi]) {
                        const double q = quad(base + bi * 2 * U + U);
                        pc[bi] += q > 0.0 ? 1.0 / q : 0.0;
                    }
                }
            }
        }
        __syncthreads();  // this buffer is restaged two steps on
    }
#pragma unroll
    for (int bi = 0; bi < kScanBlocks; ++bi) {
        red_b[warp][bi][lane] = pb[bi];
        red_c[warp][bi][lane] = pc[bi];
    }
    __syncthreads();
    double sb = 0.0, sc = 0.0;
    if (warp < nb) {
        for (int w = 0; w < kScanWarps; ++w) {
            sb += red_b[w][warp][lane];
            sc += red_c[w][warp][lane];
        }
    }
    if (gridDim.z == 1) {
        if (warp < nb && l < n) {
            bartlett[static_cast<size_t>(b0 + warp) * n + l] = sb;
            capon[static_cast<size_t>(b0 + warp) * n + l] = sc;
        }
        return;
    }
    if (warp < nb) {
        fin_b[warp][lane] = sb;
        fin_c[warp][lane] = sc;
    }
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (cluster.block_rank() == 0 && warp < nb && l < n) {
        double tb = 0.0, tc = 0.0;
        for (unsigned r = 0; r < gridDim.z; ++r) {
            tb += *cluster.map_shared_rank(&fin_b[warp][lane], r);
            tc += *cluster.map_shared_rank(&fin_c[warp][lane], r);
        }
        bartlett[static_cast<size_t>(b0 + warp) * n + l] = tb;
        capon[static_cast<size_t>(b0 + warp) * n + l] = tc;
    }
    cluster.sync();  // the other CTAs keep their shared memory until rank 0 has read it
}

// Channel-step split: the smallest modelled time ceil(CTAs / slots) *
// (steps per CTA + 1/2) over splits of 1 .. kMaxSplit, where slots are the
// GPU's resident CTAs of this kernel.
int scan_split(long long base_ctas, int n_steps, long long slots) {
    int best = 1;
    double best_cost = 1e300;
    for (int s = 1; s <= std::min(kMaxSplit, n_steps); ++s) {
        const int per = (n_steps + s - 1) / s;
        const int splits = (n_steps + per - 1) / per;
        const long long waves = (base_ctas * splits + slots - 1) / slots;
        const double cost = static_cast<double>(waves) * (per + 0.5);
        if (cost < best_cost - 1e-9) { best_cost = cost; best = splits; }
    }
    return best;
}

// One form of the scan (general or uniform sub-array), split over a cluster.
template <int M, bool kUniform>
bf_status launch_scan_form(cudaStream_t stream, const Cd* S, const Cd* Q, const int* ok, const float* pos,
                           const double* kw, int B, int F, double l_first, double l_step, int n, double m_fixed,
                           double* bartlett, double* capon, const ArrayInfo* info, const double* coef) {
    constexpr int KB = scan_blocks<M, kUniform>();
    const unsigned gx = static_cast<unsigned>((n + 31) / 32), gy = static_cast<unsigned>((B + KB - 1) / KB);
    const size_t per_warp = kUniform ? static_cast<size_t>(KB) * coef_per_form(M)
                                     : static_cast<size_t>(KB) * 2 * (M * (M + 1) / 2);
    const size_t smem = 2ull * kScanWarps * per_warp * sizeof(Cd);
    auto kern = doa_scan_kernel<M, kUniform>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_status(e, "doa_scan_kernel smem attribute");
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kScanWarps * 32, smem);
    if (e != cudaSuccess) return cuda_status(e, "doa_scan_kernel occupancy");
    const int n_steps = (F + kScanWarps - 1) / kScanWarps;
    const int split = scan_split(static_cast<long long>(gx) * gy, n_steps,
                                 static_cast<long long>(std::max(per_sm, 1)) * sms);
    const int per = (n_steps + split - 1) / split;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(gx, gy, static_cast<unsigned>(split));
    cfg.blockDim = dim3(kScanWarps * 32, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = static_cast<unsigned>(split);
    cfg.attrs = attr;
    cfg.numAttrs = split > 1 ? 1 : 0;
    e = cudaLaunchKernelEx(&cfg, kern, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed, bartlett, capon, per,
                           info, coef);
    return cuda_status(e == cudaSuccess ? cudaGetLastError() : e, "doa_scan_kernel launch");
}

// Both forms go into the stream; the one the array does not select returns
// at once.
template <int M>
bf_status launch_scan_m(cudaStream_t stream, const Cd* S, const Cd* Q, const int* ok, const float* pos,
                        const double* kw, int B, int F, double l_first, double l_step, int n, double m_fixed,
                        double* bartlett, double* capon, const ArrayInfo* info, const double* coef) {
    BF_RETURN_IF((launch_scan_form<M, false>(stream, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed, bartlett,
                                             capon, info, coef)));
    if constexpr (M >= 2) {
        BF_RETURN_IF((launch_scan_form<M, true>(stream, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed,
                                                bartlett, capon, info, coef)));
    }
    return BF_OK;
}

template <int M>
bf_status dispatch_scan(int m, cudaStream_t stream, const Cd* S, const Cd* Q, const int* ok, const float* pos,
                        const double* kw, int B, int F, double l_first, double l_step, int n, double m_fixed,
                        double* bartlett, double* capon, const ArrayInfo* info, const double* coef) {
    if constexpr (M > kMaxM) {
        return set_error(BF_ERR_UNSUPPORTED, "the DOA scan supports at most 16 elements after smoothing");
    } else {
        if (m == M) {
            return launch_scan_m<M>(stream, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed, bartlett, capon,
                                    info, coef);
        }
        return dispatch_scan<M + 1>(m, stream, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed, bartlett, capon,
                                    info, coef);
    }
}

// One warp per (block, estimator): argmax plus parabolic vertex.
__global__ void doa_peak_kernel(const double* __restrict bartlett, const double* __restrict capon, int n,
                                double l_first, double l_step, double* __restrict l_est) {
    const int b = blockIdx.x, e = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* P = (e == 0 ? bartlett : capon) + static_cast<size_t>(b) * n;
    double best = -1.0;
    int bi = 0;
    for (int l = lane; l < n; l += 32) {
        if (P[l] > best) { best = P[l]; bi = l; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (lane == 0) {
        double delta = 0.0;
        if (bi > 0 && bi + 1 < n) {
            const double den = P[bi - 1] - 2.0 * P[bi] + P[bi + 1];
            if (den < 0.0) delta = fmin(0.5, fmax(-0.5, 0.5 * (P[bi - 1] - P[bi + 1]) / den));
        }
        l_est[2 * b + e] = l_first + (bi + delta) * l_step;
    }
}

}  // namespace

// Workspace: S and Q [cells][M][M] Cd, eps [cells] double, ok [cells] int,
// then (256-byte aligned) the array description and the uniform form's
// coefficients [cells][2][4M - 2] double.
uint64_t doa_coef_offset(uint64_t cells, uint64_t M) {
    const uint64_t head = cells * (2 * M * M * sizeof(Cd) + sizeof(double) + sizeof(int));
    return (head + 255) / 256 * 256;
}

uint64_t doa_workspace_bytes(uint64_t n_blocks, uint64_t n_freq, uint64_t M) {
    const uint64_t cells = n_blocks * n_freq;
    const uint64_t info = (sizeof(ArrayInfo) + 255) / 256 * 256;
    return doa_coef_offset(cells, M) + info + cells * 2 * coef_per_form(static_cast<int>(M)) * sizeof(double) + 256;
}

uint64_t doa_fold_bytes(uint64_t cells, uint64_t M) { return doa_coef_offset(cells, M); }

namespace {

template <int M>
bf_status dispatch_fold(int m, cudaStream_t stream, const int32_t* R, int B, int F, int A, int K, double lam,
                        double load, Cd* S, Cd* Q, double* E, int* ok) {
    if constexpr (M > kMaxM) {
        return set_error(BF_ERR_UNSUPPORTED, "the DOA scan supports at most 16 elements after smoothing");
    } else {
        if (m == M) {
            static_assert(2 * fold_cells<M>() * M * M * sizeof(Cd) <= 32768, "fold shared memory");
            doa_fold_kernel<M><<<F, 32 * fold_cells<M>(), 0, stream>>>(R, B, F, A, K, lam, load, S, Q, E, ok);
            return cuda_status(cudaGetLastError(), "doa_fold_kernel launch");
        }
        return dispatch_fold<M + 1>(m, stream, R, B, F, A, K, lam, load, S, Q, E, ok);
    }
}

}  // namespace

bf_status launch_doa_fold(cudaStream_t stream, const int32_t* R, const bf_dims& d, uint64_t block_len, int M,
                          double lam, double load, void* workspace) {
    const int A = static_cast<int>(d.n_ant);
    if (M > kMaxM) return set_error(BF_ERR_UNSUPPORTED, "the DOA scan supports at most 16 elements after smoothing");
    if (d.n_time / block_len > 65535) return set_error(BF_ERR_OVERFLOW, "at most 65535 covariance blocks per scan");
    const int B = static_cast<int>(d.n_time / block_len), F = static_cast<int>(d.n_freq);
    const uint64_t cells = static_cast<uint64_t>(B) * F;
    auto* S = static_cast<Cd*>(workspace);
    Cd* Lc = S + cells * M * M;  // the fold writes Q = (S + E I)^{-1} here
    auto* E = reinterpret_cast<double*>(Lc + cells * M * M);
    auto* ok = reinterpret_cast<int*>(E + cells);
    // one CTA per channel pays when the channels fill the SMs; fewer channels
    // (a channel slice of a split job) run every cell in parallel instead
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (B <= kFoldChunks * fold_cells_for(M) && F >= sms) {
        return dispatch_fold<1>(M, stream, R, B, F, A, static_cast<int>(block_len), lam, load, S, Lc, E, ok);
    }
    const dim3 cells_grid(static_cast<unsigned>(F), static_cast<unsigned>(B));
    doa_smooth_kernel<<<cells_grid, 32, 0, stream>>>(R, F, A, M, static_cast<int>(block_len), load, Lc, E);
    BF_RETURN_IF(cuda_status(cudaGetLastError(), "doa_smooth_kernel launch"));
    doa_forget_kernel<<<F, 64, 0, stream>>>(Lc, B, F, M, lam, S, E);
    BF_RETURN_IF(cuda_status(cudaGetLastError(), "doa_forget_kernel launch"));
    doa_factor_kernel<<<cells_grid, 64, 0, stream>>>(S, E, F, M, Lc, ok);
    return cuda_status(cudaGetLastError(), "doa_factor_kernel launch");
}

bf_status launch_doa_scan(cudaStream_t stream, const int32_t* R, const float* pos, const double* kw,
                          const bf_dims& d, uint64_t block_len, uint64_t subarray, double lam, double load,
                          double l_first, double l_step, uint64_t n, double m_fixed, double* bartlett,
                          double* capon, double* l_est, void* workspace) {
    const int A = static_cast<int>(d.n_ant);
    const int M = (subarray > 0 && subarray < d.n_ant) ? static_cast<int>(subarray) : A;
    BF_RETURN_IF(launch_doa_fold(stream, R, d, block_len, M, lam, load, workspace));
    const int B = static_cast<int>(d.n_time / block_len), F = static_cast<int>(d.n_freq);
    const uint64_t cells = static_cast<uint64_t>(B) * F;
    auto* S = static_cast<Cd*>(workspace);
    Cd* Lc = S + cells * M * M;
    auto* E = reinterpret_cast<double*>(Lc + cells * M * M);
    auto* ok = reinterpret_cast<int*>(E + cells);
    const dim3 cells_grid(static_cast<unsigned>(F), static_cast<unsigned>(B));
    auto* info = reinterpret_cast<ArrayInfo*>(static_cast<uint8_t*>(workspace) + doa_coef_offset(cells, M));
    auto* coef = reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(info) + (sizeof(ArrayInfo) + 255) / 256 * 256);
    const double l_abs_max = std::max(std::fabs(l_first), std::fabs(l_first + static_cast<double>(n - 1) * l_step));
    doa_array_kernel<<<1, 32, 0, stream>>>(pos, kw, M, F, l_abs_max, m_fixed, info);
    BF_RETURN_IF(cuda_status(cudaGetLastError(), "doa_array_kernel launch"));
    if (M >= 2) {
        doa_coef_kernel<<<cells_grid, 64, 0, stream>>>(S, Lc, kw, F, M, m_fixed, info, coef);
        BF_RETURN_IF(cuda_status(cudaGetLastError(), "doa_coef_kernel launch"));
    }
    BF_RETURN_IF(dispatch_scan<1>(M, stream, S, Lc, ok, pos, kw, B, F, l_first, l_step, static_cast<int>(n), m_fixed,
                                  bartlett, capon, info, coef));
    doa_peak_kernel<<<B, 64, 0, stream>>>(bartlett, capon, static_cast<int>(n), l_first, l_step, l_est);
    return cuda_status(cudaGetLastError(), "doa_peak_kernel launch");
}

bf_status launch_doa_peak(cudaStream_t stream, const double* bartlett, const double* capon, uint64_t n_blocks,
                          uint64_t n_points, double l_first, double l_step, double* l_est) {
    doa_peak_kernel<<<static_cast<unsigned>(n_blocks), 64, 0, stream>>>(bartlett, capon, static_cast<int>(n_points),
                                                                       l_first, l_step, l_est);
    return cuda_status(cudaGetLastError(), "doa_peak_kernel launch");
}

}  // namespace bf
