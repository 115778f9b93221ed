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

// One block of threads per channel; thread 0 walks the blocks in order.
__global__ void doa_fold_kernel(const int32_t* __restrict R, int n_blocks, int n_freq, int A, int M, int K,
                                double lam, double load, Cd* __restrict S_out, double* __restrict E_out,
                                Cd* __restrict L_out, int* __restrict ok_out) {
    const int f = blockIdx.x;
    __shared__ Cd Rt[kMaxM * kMaxM];
    __shared__ Cd S[kMaxM * kMaxM];
    __shared__ double E;
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
            Cd Lc[kMaxM * kMaxM];
            int ok = 1;
            for (int i = 0; i < M && ok; ++i) {
                for (int j = 0; j <= i; ++j) {
                    double sr = S[i * M + j].re + (i == j ? E : 0.0), si = S[i * M + j].im;
                    for (int k = 0; k < j; ++k) {
                        const Cd x = Lc[i * M + k], y = Lc[j * M + k];  // x * conj(y)
                        sr -= x.re * y.re + x.im * y.im;
                        si -= x.im * y.re - x.re * y.im;
                    }
                    if (i == j) {
                        if (!(sr > 1e-300)) { ok = 0; break; }
                        Lc[i * M + i] = Cd{sqrt(sr), 0.0};
                    } else {
                        const double d = Lc[j * M + j].re;
                        Lc[i * M + j] = Cd{sr / d, si / d};
                    }
                }
            }
            for (int e = 0; e < M * M; ++e) L_out[base + e] = ok ? Lc[e] : Cd{0.0, 0.0};
            ok_out[static_cast<size_t>(b) * n_freq + f] = ok;
        }
        __syncthreads();
    }
}

// A CTA of 8 warps takes 32 grid points of one block: lane = grid point,
// warp w sums the channels f = w, w + 8, ... in increasing order, and the
// eight partial sums are added in warp order at the end (a fixed order, so
// results are deterministic).
constexpr int kScanWarps = 8;

__global__ void __launch_bounds__(kScanWarps * 32)
doa_scan_kernel(const Cd* __restrict S, const Cd* __restrict Lf, const int* __restrict ok,
                const float* __restrict pos, const double* __restrict kw, int n_freq, int M,
                double l_first, double l_step, int n, double m_fixed, double* __restrict bartlett,
                double* __restrict capon) {
    const int b = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * 32 + lane;
    extern __shared__ Cd scan_smem[];              // [warp][S | L][M * M]
    Cd* sSw = scan_smem + static_cast<size_t>(warp) * 2 * M * M;
    Cd* sLw = sSw + M * M;
    __shared__ double red_b[kScanWarps][32], red_c[kScanWarps][32];
    const double lv = l_first + static_cast<double>(l) * l_step;
    double pb = 0.0, pc = 0.0;
    for (int f = warp; f < n_freq; f += kScanWarps) {
        const size_t base = (static_cast<size_t>(b) * n_freq + f) * M * M;
        __syncwarp();
        for (int e = lane; e < M * M; e += 32) {
            sSw[e] = S[base + e];
            sLw[e] = Lf[base + e];
        }
        const int fok = ok[static_cast<size_t>(b) * n_freq + f];
        __syncwarp();
        Cd a[kMaxM];
        for (int i = 0; i < M; ++i) {
            const double ph = kw[f] * (static_cast<double>(pos[3 * i]) * lv + static_cast<double>(pos[3 * i + 1]) * m_fixed);
            const double rr = ph - kTwoPi * rint(ph * (1.0 / kTwoPi));
            float s, c;
            sincosf(static_cast<float>(rr), &s, &c);
            a[i] = Cd{static_cast<double>(c), -static_cast<double>(s)};
        }
        double acc = 0.0;
        for (int r = 0; r < M; ++r) {
            double tr = 0.0, ti = 0.0;
            for (int c = 0; c < M; ++c) {
                const Cd x = sSw[r * M + c];
                tr += x.re * a[c].re - x.im * a[c].im;
                ti += x.re * a[c].im + x.im * a[c].re;
            }
            acc += a[r].re * tr + a[r].im * ti;
        }
        pb += acc;
        if (fok) {
            Cd v[kMaxM];
            double nrm = 0.0;
            for (int i = 0; i < M; ++i) {
                double sr = a[i].re, si = a[i].im;
                for (int k = 0; k < i; ++k) {
                    const Cd x = sLw[i * M + k];
                    sr -= x.re * v[k].re - x.im * v[k].im;
                    si -= x.re * v[k].im + x.im * v[k].re;
                }
                const double d = sLw[i * M + i].re;
                v[i] = Cd{sr / d, si / d};
                nrm += v[i].re * v[i].re + v[i].im * v[i].im;
            }
            pc += nrm > 0.0 ? 1.0 / nrm : 0.0;
        }
    }
    red_b[warp][lane] = pb;
    red_c[warp][lane] = pc;
    __syncthreads();
    if (warp == 0 && l < n) {
        double sb = 0.0, sc = 0.0;
        for (int w = 0; w < kScanWarps; ++w) {
            sb += red_b[w][lane];
            sc += red_c[w][lane];
        }
        bartlett[static_cast<size_t>(b) * n + l] = sb;
        capon[static_cast<size_t>(b) * n + l] = sc;
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
    Cd* Lc = S + cells * M * M;
    auto* E = reinterpret_cast<double*>(Lc + cells * M * M);
    auto* ok = reinterpret_cast<int*>(E + cells);
    doa_fold_kernel<<<F, 64, 0, stream>>>(R, B, F, A, M, static_cast<int>(block_len), lam, load, S, E, Lc, ok);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "doa_fold_kernel launch");
    const dim3 grid(static_cast<unsigned>((n + 31) / 32), static_cast<unsigned>(B));
    const size_t smem = static_cast<size_t>(kScanWarps) * 2 * M * M * sizeof(Cd);
    e = cudaFuncSetAttribute(doa_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_status(e, "doa_scan_kernel smem attribute");
    doa_scan_kernel<<<grid, kScanWarps * 32, smem, stream>>>(S, Lc, ok, pos, kw, F, M, l_first, l_step,
                                                             static_cast<int>(n), m_fixed, bartlett, capon);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "doa_scan_kernel launch");
    doa_peak_kernel<<<B, 64, 0, stream>>>(bartlett, capon, static_cast<int>(n), l_first, l_step, l_est);
    return cuda_status(cudaGetLastError(), "doa_peak_kernel launch");
}

}  // namespace bf
