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
// FP64 is used for the phase argument before its reduction mod 2 pi, the
// forgetting accumulation and the loaded Cholesky solve; the reduced phase
// goes through float sincos.
#include "bf_internal.cuh"

#include <algorithm>

namespace bf {
namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr int kMaxM = 16;

struct Cd {
    double re, im;
};

// One CTA per channel walks the blocks in order (the forgetting recursion).
// Smoothing, forward-backward and forgetting run over the M x M elements;
// thread 0 factors S + E I (Cholesky, shared memory); thread j forms column j
// of L^{-1}; the threads then form Q = L^{-H} L^{-1} = (S + E I)^{-1} by
// elements, so the scan evaluates Capon's |L^{-1} a|^2 as a^H Q a.
__global__ void doa_fold_kernel(const int32_t* __restrict R, int n_blocks, int n_freq, int A, int M, int K,
                                double lam, double load, Cd* __restrict S_out, double* __restrict E_out,
                                Cd* __restrict Q_out, int* __restrict ok_out) {
    const int f = blockIdx.x;
    __shared__ Cd Rt[kMaxM * kMaxM];
    __shared__ Cd S[kMaxM * kMaxM];
    __shared__ Cd Lc[kMaxM * kMaxM];
    __shared__ Cd Li[kMaxM * kMaxM];
    __shared__ double E;
    __shared__ int ok;
    const int L = A - M + 1;
    for (int b = 0; b < n_blocks; ++b) {
        const int32_t* Rf = R + (static_cast<size_t>(b) * n_freq + f) * A * A * 2;
        for (int e = threadIdx.x; e < M * M; e += blockDim.x) {
            const int r = e / M, c = e % M;
            double sr = 0.0, si = 0.0;
            for (int s = 0; s < L; ++s) {
                sr += static_cast<double>(Rf[2 * ((s + r) * A + s + c)]);
                si += static_cast<double>(Rf[2 * ((s + r) * A + s + c) + 1]);
            }
            Rt[e] = Cd{sr / K / L, si / K / L};
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double tr = 0.0;
            for (int r = 0; r < M; ++r) {
                const Cd x = Rt[r * M + r];
                tr += L > 1 ? 0.5 * (x.re + Rt[(M - 1 - r) * M + (M - 1 - r)].re) : x.re;
            }
            const double eps = load * tr / M;
            E = (b == 0 || lam >= 1.0) ? eps : lam * E + (1.0 - lam) * eps;
        }
        for (int e = threadIdx.x; e < M * M; e += blockDim.x) {
            const int r = e / M, c = e % M;
            Cd x = Rt[e];
            if (L > 1) {
                const Cd y = Rt[(M - 1 - r) * M + (M - 1 - c)];
                x = Cd{0.5 * (x.re + y.re), 0.5 * (x.im - y.im)};
            }
            S[e] = (b == 0 || lam >= 1.0) ? x : Cd{lam * S[e].re + (1.0 - lam) * x.re, lam * S[e].im + (1.0 - lam) * x.im};
        }
        __syncthreads();
        const size_t base = (static_cast<size_t>(b) * n_freq + f) * M * M;
        for (int e = threadIdx.x; e < M * M; e += blockDim.x) S_out[base + e] = S[e];
        if (threadIdx.x == 0) {
            E_out[static_cast<size_t>(b) * n_freq + f] = E;
            // Cholesky of S + E I (lower triangular, FP64)
            int good = 1;
            for (int i = 0; i < M && good; ++i) {
                for (int j = 0; j <= i; ++j) {
                    double sr = S[i * M + j].re + (i == j ? E : 0.0), si = S[i * M + j].im;
                    for (int k = 0; k < j; ++k) {
                        const Cd x = Lc[i * M + k], y = Lc[j * M + k];  // x * conj(y)
                        sr -= x.re * y.re + x.im * y.im;
                        si -= x.im * y.re - x.re * y.im;
                    }
                    if (i == j) {
                        if (!(sr > 1e-300)) { good = 0; break; }
                        Lc[i * M + i] = Cd{sqrt(sr), 0.0};
                    } else {
                        const double d = Lc[j * M + j].re;
                        Lc[i * M + j] = Cd{sr / d, si / d};
                    }
                }
            }
            ok = good;
            ok_out[static_cast<size_t>(b) * n_freq + f] = good;
        }
        __syncthreads();
        if (ok && threadIdx.x < M) {  // column j of L^{-1} by forward substitution
            const int j = threadIdx.x;
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
        __syncthreads();
        for (int e = threadIdx.x; e < M * M; e += blockDim.x) {
            const int i = e / M, j = e % M;
            double qr = 0.0, qi = 0.0;
            if (ok) {
                for (int k = i > j ? i : j; k < M; ++k) {
                    const Cd x = Li[k * M + i], y = Li[k * M + j];  // conj(x) * y
                    qr += x.re * y.re + x.im * y.im;
                    qi += x.re * y.im - x.im * y.re;
                }
            }
            Q_out[base + e] = Cd{qr, qi};
        }
        __syncthreads();
    }
}

// A CTA of 16 warps takes 32 grid points and 8 blocks: lane = grid point,
// warp w the channels f = w, w + 16, ... in increasing order.  The steering
// vector of (channel, point) is formed once and used for all 8 blocks;
// Bartlett a^H S a and Capon 1 / (a^H Q a), Q = (S + eps I)^{-1}, are
// Hermitian quadratic forms (diagonal plus twice the real part of the upper
// triangle).  Per-warp partial sums are added in warp order at the end (a
// fixed order, so results are deterministic).
constexpr int kScanWarps = 16;
constexpr int kScanBlocks = 8;

template <int M>
__global__ void __launch_bounds__(kScanWarps * 32)
doa_scan_kernel(const Cd* __restrict S, const Cd* __restrict Q, const int* __restrict ok,
                const float* __restrict pos, const double* __restrict kw, int n_blocks, int n_freq,
                double l_first, double l_step, int n, double m_fixed, double* __restrict bartlett,
                double* __restrict capon) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * 32 + lane;
    const int b0 = blockIdx.y * kScanBlocks;
    const int nb = min(kScanBlocks, n_blocks - b0);
    extern __shared__ double scan_red[];  // [2][warps][kScanBlocks][32]
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
    for (int f = warp; f < n_freq; f += kScanWarps) {
        Cd a[M];
        double mag[M];
        const double k = kw[f];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double ph = k * (px[i] * lv + py[i] * m_fixed);
            const double rr = ph - kTwoPi * rint(ph * (1.0 / kTwoPi));
            float s, c;
            sincosf(static_cast<float>(rr), &s, &c);
            a[i] = Cd{static_cast<double>(c), -static_cast<double>(s)};
            mag[i] = a[i].re * a[i].re + a[i].im * a[i].im;
        }
        auto quad = [&](const Cd* __restrict X) {
            double diag = 0.0, off = 0.0;
#pragma unroll
            for (int r = 0; r < M; ++r) {
                diag += X[r * M + r].re * mag[r];
                double tr = 0.0, ti = 0.0;
#pragma unroll
                for (int c = r + 1; c < M; ++c) {
                    const Cd x = X[r * M + c];
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
                const size_t cell = static_cast<size_t>(b0 + bi) * n_freq + f;
                pb[bi] += quad(S + cell * M * M);
                if (ok[cell]) {
                    const double q = quad(Q + cell * M * M);
                    pc[bi] += q > 0.0 ? 1.0 / q : 0.0;
                }
            }
        }
    }
#pragma unroll
    for (int bi = 0; bi < kScanBlocks; ++bi) {
        scan_red[((0 * kScanWarps + warp) * kScanBlocks + bi) * 32 + lane] = pb[bi];
        scan_red[((1 * kScanWarps + warp) * kScanBlocks + bi) * 32 + lane] = pc[bi];
    }
    __syncthreads();
    if (warp < nb && l < n) {
        double sb = 0.0, sc = 0.0;
        for (int w = 0; w < kScanWarps; ++w) {
            sb += scan_red[((0 * kScanWarps + w) * kScanBlocks + warp) * 32 + lane];
            sc += scan_red[((1 * kScanWarps + w) * kScanBlocks + warp) * 32 + lane];
        }
        bartlett[static_cast<size_t>(b0 + warp) * n + l] = sb;
        capon[static_cast<size_t>(b0 + warp) * n + l] = sc;
    }
}

template <int M>
bf_status launch_scan_m(cudaStream_t stream, const Cd* S, const Cd* Q, const int* ok, const float* pos,
                        const double* kw, int B, int F, double l_first, double l_step, int n, double m_fixed,
                        double* bartlett, double* capon) {
    const dim3 grid(static_cast<unsigned>((n + 31) / 32), static_cast<unsigned>((B + kScanBlocks - 1) / kScanBlocks));
    const size_t smem = 2ull * kScanWarps * kScanBlocks * 32 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(doa_scan_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_status(e, "doa_scan_kernel smem attribute");
    doa_scan_kernel<M><<<grid, kScanWarps * 32, smem, stream>>>(S, Q, ok, pos, kw, B, F, l_first, l_step, n,
                                                               m_fixed, bartlett, capon);
    return cuda_status(cudaGetLastError(), "doa_scan_kernel launch");
}

template <int M>
bf_status dispatch_scan(int m, cudaStream_t stream, const Cd* S, const Cd* Q, const int* ok, const float* pos,
                        const double* kw, int B, int F, double l_first, double l_step, int n, double m_fixed,
                        double* bartlett, double* capon) {
    if constexpr (M > kMaxM) {
        return set_error(BF_ERR_UNSUPPORTED, "the DOA scan supports at most 16 elements after smoothing");
    } else {
        if (m == M) return launch_scan_m<M>(stream, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed, bartlett, capon);
        return dispatch_scan<M + 1>(m, stream, S, Q, ok, pos, kw, B, F, l_first, l_step, n, m_fixed, bartlett, capon);
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

uint64_t doa_workspace_bytes(uint64_t n_blocks, uint64_t n_freq, uint64_t M) {
    const uint64_t cells = n_blocks * n_freq;
    return cells * (2 * M * M * sizeof(Cd) + sizeof(double) + sizeof(int)) + 256;
}

bf_status launch_doa_scan(cudaStream_t stream, const int32_t* R, const float* pos, const double* kw,
                          const bf_dims& d, uint64_t block_len, uint64_t subarray, double lam, double load,
                          double l_first, double l_step, uint64_t n, double m_fixed, double* bartlett,
                          double* capon, double* l_est, void* workspace) {
    const int A = static_cast<int>(d.n_ant);
    const int M = (subarray > 0 && subarray < d.n_ant) ? static_cast<int>(subarray) : A;
    if (M > kMaxM) return set_error(BF_ERR_UNSUPPORTED, "the DOA scan supports at most 16 elements after smoothing");
    const int B = static_cast<int>(d.n_time / block_len), F = static_cast<int>(d.n_freq);
    const uint64_t cells = static_cast<uint64_t>(B) * F;
    auto* S = static_cast<Cd*>(workspace);
    Cd* Lc = S + cells * M * M;  // the fold writes Q = (S + E I)^{-1} here
    auto* E = reinterpret_cast<double*>(Lc + cells * M * M);
    auto* ok = reinterpret_cast<int*>(E + cells);
    doa_fold_kernel<<<F, 64, 0, stream>>>(R, B, F, A, M, static_cast<int>(block_len), lam, load, S, E, Lc, ok);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "doa_fold_kernel launch");
    BF_RETURN_IF(dispatch_scan<1>(M, stream, S, Lc, ok, pos, kw, B, F, l_first, l_step, static_cast<int>(n), m_fixed,
                                  bartlett, capon));
    doa_peak_kernel<<<B, 64, 0, stream>>>(bartlett, capon, static_cast<int>(n), l_first, l_step, l_est);
    return cuda_status(cudaGetLastError(), "doa_peak_kernel launch");
}

}  // namespace bf
