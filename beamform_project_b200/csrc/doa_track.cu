// doa_track.cu -- the reference's adaptive tracker on the GPU: per window a
// coarse-to-fine direction search over (l, m), then the beam along the
// estimated direction.
//
// Reference: CpuOptBeamTracker::run_into (src/cpu_opt_beam_tracker.cpp:
// 1619-2454).  Per window (block of K spectra), after the covariance fold
// (doa_cov.cu + launch_doa_fold: smoothing, forward-backward, loading,
// forgetting, loaded Cholesky):
//   level 0   a G x G grid centred on the previous window's estimate (the
//             seeded prior for the first), pitch 2 fov / (G - 1), cells off
//             the unit disk pulled in to r^2 = 0.999 (:806-828); power summed
//             over channels (Bartlett a^H R a, Capon 1 / (a^H (R + eps I)^-1 a),
//             non-finite powers count 0) and its first argmax (:2138-2147);
//   levels    3 x 3 candidates around the running centre at half the previous
//             half-pitch (fov / G halved per level), argmax, then the 3-point
//             quadratic interpolation of the reference on the candidates'
//             centre row and column, applied to the new centre (:2149-2381);
//             with no refinement the interpolation runs on the coarse grid;
//   emission  the window's per-spectrum beam power along the estimate, in the
//             reference's float32 order (the tracker of tracker.cu, mode 0).
// The steering phase is FP64 (k (x l + y m + z n)) reduced to a quadrant, with
// the FP32 Taylor sin / cos of tracker_common.cuh, and powers are FP64 (the
// reference: FP32), so the search follows the reference's geometry and
// decisions and differs only where two candidates' powers tie to float
// precision.  Grid construction, clamping and interpolation are float32 with
// the reference's operation order.
//
// Launches per window: (level kernel, select kernel) per level.  The level
// kernel evaluates its points x channels (lane = point, warp = channel) and
// writes one partial sum per (point, 64-channel group); the select kernel
// (one CTA) adds the groups in order, takes the argmax and writes the next
// level's points, or the window's direction and the next window's grid.
#include "bf_internal.cuh"
#include "tracker_common.cuh"

#include <algorithm>
#include <cmath>

namespace bf {
namespace {

constexpr int kMaxM = 16;
constexpr int kMaxGrid = 64;                     // G <= 64: at most 4096 coarse points
constexpr int kMaxPoints = kMaxGrid * kMaxGrid;
constexpr int kChanGroup = 64;                   // channels per partial sum

struct Cd {
    double re, im;
};

// Search state between launches (device memory).
struct SearchState {
    float cl, cm;          // running centre (l, m)
    float half_l, half_m;  // refinement half-pitch of the current level
    int n_points;          // points of the current level
    int pad;
};

struct TrackParams {
    const Cd* S;           // folded covariance [cells][M][M]
    const Cd* Q;           // (S + E I)^-1 [cells][M][M]
    const int* ok;         // [cells]
    const float* pos;      // [A][3]
    const double* kw;      // [F]
    int n_freq, M;
    int capon;
};

__device__ __forceinline__ float2 clamp_disk(float l, float m) {
    const float r2 = __fadd_rn(__fmul_rn(l, l), __fmul_rn(m, m));
    if (r2 > 0.999f) {
        const float s = __fsqrt_rn(__fdiv_rn(0.999f, r2));
        l = __fmul_rn(l, s);
        m = __fmul_rn(m, s);
    }
    return make_float2(l, m);
}

// Bartlett or Capon power of window `b` at the points, summed over each
// 64-channel group: partial[group][point].
template <int M>
__global__ void __launch_bounds__(256) doa_level_kernel(TrackParams p, int b, const float2* __restrict points,
                                                        const SearchState* __restrict state,
                                                        double* __restrict partial) {
    const int n_points = state->n_points;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int pt = blockIdx.x * 32 + lane;
    const int group = blockIdx.y;
    __shared__ double red[8][32];
    double acc = 0.0;
    if (pt < n_points) {
        const float2 lm = points[pt];
        const double l = lm.x, m = lm.y;
        // n as direction_from_lm forms it (float), for arrays with z != 0
        const float nf = __fsqrt_rn(__fsub_rn(1.0f, __fadd_rn(__fmul_rn(lm.x, lm.x), __fmul_rn(lm.y, lm.y))));
        const double n = nf;
        for (int f = group * kChanGroup + warp; f < min(p.n_freq, (group + 1) * kChanGroup); f += 8) {
            const size_t cell = static_cast<size_t>(b) * p.n_freq + f;
            const double k = p.kw[f];
            Cd a[M];
            double mag[M];
#pragma unroll
            for (int i = 0; i < M; ++i) {
                const double delay = trk::steering_delay(p.pos, i, l, m, n);
                const float2 w = trk::steering_from_delay(k, delay);
                a[i] = Cd{static_cast<double>(w.x), -static_cast<double>(w.y)};  // exp(-i phase)
                mag[i] = a[i].re * a[i].re + a[i].im * a[i].im;
            }
            const Cd* X = (p.capon ? p.Q : p.S) + cell * M * M;
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
                off += a[r].re * tr + a[r].im * ti;  // Re(conj(a_r) * (X a)_r upper part)
            }
            double pw = diag + 2.0 * off;
            if (p.capon) pw = (p.ok[cell] && pw > 0.0) ? 1.0 / pw : 0.0;
            if (!isfinite(pw)) pw = 0.0;
            acc += pw;
        }
    }
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && pt < n_points) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += red[w][lane];
        partial[static_cast<size_t>(group) * kMaxPoints + pt] = s;
    }
}

// The reference's 3-point interpolation (src/cpu_opt_beam_tracker.cpp:
// 830-850): an offset only where denom > 0, clamped to [-0.5, 0.5].
__device__ __forceinline__ float interp_offset(float pc, float p_up, float p_down) {
    const float denom = __fadd_rn(__fsub_rn(p_down, __fmul_rn(2.0f, pc)), p_up);
    if (!(denom > 0.0f)) return 0.0f;
    const float d = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(p_up, p_down)), denom);
    return fminf(0.5f, fmaxf(-0.5f, d));
}

__device__ __forceinline__ void coarse_grid(SearchState* st, float2* points, float cl, float cm, int G, float fov_l,
                                            float fov_m) {
    const float step_l = G == 1 ? 0.0f : __fdiv_rn(__fmul_rn(2.0f, fov_l), static_cast<float>(G - 1));
    const float step_m = G == 1 ? 0.0f : __fdiv_rn(__fmul_rn(2.0f, fov_m), static_cast<float>(G - 1));
    const float start_l = __fsub_rn(cl, fov_l), start_m = __fsub_rn(cm, fov_m);
    for (int i = 0; i < G * G; ++i) {
        const int u = i % G, v = i / G;
        points[i] = clamp_disk(__fadd_rn(start_l, __fmul_rn(static_cast<float>(u), step_l)),
                               __fadd_rn(start_m, __fmul_rn(static_cast<float>(v), step_m)));
    }
    st->n_points = G * G;
}

__device__ __forceinline__ void refine_grid(SearchState* st, float2* points) {
    for (int dv = -1; dv <= 1; ++dv) {
        for (int du = -1; du <= 1; ++du) {
            points[(dv + 1) * 3 + (du + 1)] =
                clamp_disk(__fadd_rn(st->cl, __fmul_rn(static_cast<float>(du), st->half_l)),
                           __fadd_rn(st->cm, __fmul_rn(static_cast<float>(dv), st->half_m)));
        }
    }
    st->n_points = 9;
}

// One CTA: the level's powers, argmax and the next level or window.
__global__ void __launch_bounds__(256) doa_select_kernel(const double* __restrict partial, int n_groups,
                                                         float2* __restrict points, SearchState* __restrict st,
                                                         int level, int levels, int G, float fov_l, float fov_m,
                                                         int interp, float* __restrict dir_out, int last_window) {
    __shared__ float pw[kMaxPoints];
    __shared__ float best_v[256];
    __shared__ int best_i[256];
    const int n = st->n_points;
    // powers in float, as the reference compares and interpolates them
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int g = 0; g < n_groups; ++g) s += partial[static_cast<size_t>(g) * kMaxPoints + i];
        pw[i] = static_cast<float>(s);
    }
    __syncthreads();
    // first maximum: strict > over increasing index
    float bv = -INFINITY;
    int bi = n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (pw[i] > bv) { bv = pw[i]; bi = i; }
    }
    best_v[threadIdx.x] = bv;
    best_i[threadIdx.x] = bi;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int t = 1; t < blockDim.x; ++t) {
        if (best_v[t] > bv || (best_v[t] == bv && best_i[t] < bi)) { bv = best_v[t]; bi = best_i[t]; }
    }
    if (bi >= n) bi = 0;  // every power NaN-free and -inf: the first cell, as the reference
    const float2 best = points[bi];
    float cl = best.x, cm = best.y;
    if (level == 0) {
        if (levels == 0 && interp) {
            const int u = bi % G, v = bi / G;
            auto at = [&](int du, int dv) -> float {
                const int uu = u + du, vv = v + dv;
                return (uu < 0 || uu >= G || vv < 0 || vv >= G) ? 0.0f : pw[vv * G + uu];
            };
            const float pc = pw[bi];
            const float du = interp_offset(pc, at(1, 0), at(-1, 0));
            const float dv = interp_offset(pc, at(0, 1), at(0, -1));
            const float step_l = G == 1 ? 0.0f : __fdiv_rn(__fmul_rn(2.0f, fov_l), static_cast<float>(G - 1));
            const float step_m = G == 1 ? 0.0f : __fdiv_rn(__fmul_rn(2.0f, fov_m), static_cast<float>(G - 1));
            const float2 c = clamp_disk(__fadd_rn(cl, __fmul_rn(du, step_l)), __fadd_rn(cm, __fmul_rn(dv, step_m)));
            cl = c.x;
            cm = c.y;
        }
        st->half_l = __fdiv_rn(fov_l, static_cast<float>(G));
        st->half_m = __fdiv_rn(fov_m, static_cast<float>(G));
    } else {
        if (interp) {
            // the candidates' centre row and column, whichever candidate won
            const float du = interp_offset(pw[4], pw[5], pw[3]);
            const float dv = interp_offset(pw[4], pw[7], pw[1]);
            const float2 c = clamp_disk(__fadd_rn(cl, __fmul_rn(du, st->half_l)),
                                        __fadd_rn(cm, __fmul_rn(dv, st->half_m)));
            cl = c.x;
            cm = c.y;
        }
    }
    st->cl = cl;
    st->cm = cm;
    if (level < levels) {
        st->half_l = __fmul_rn(st->half_l, 0.5f);
        st->half_m = __fmul_rn(st->half_m, 0.5f);
        refine_grid(st, points);
        return;
    }
    // the window's direction (direction_from_lm) and the next window's grid
    dir_out[0] = cl;
    dir_out[1] = cm;
    dir_out[2] = __fsqrt_rn(__fsub_rn(1.0f, __fadd_rn(__fmul_rn(cl, cl), __fmul_rn(cm, cm))));
    if (!last_window) coarse_grid(st, points, cl, cm, G, fov_l, fov_m);
}

__global__ void doa_track_init_kernel(SearchState* st, float2* points, float l0, float m0, int G, float fov_l,
                                      float fov_m) {
    if (threadIdx.x == 0 && blockIdx.x == 0) coarse_grid(st, points, l0, m0, G, fov_l, fov_m);
}

template <int M>
bf_status launch_level(cudaStream_t stream, const TrackParams& p, int b, const float2* points, const SearchState* st,
                       double* partial, int n_points_max, int n_groups) {
    const dim3 grid(static_cast<unsigned>((n_points_max + 31) / 32), static_cast<unsigned>(n_groups));
    doa_level_kernel<M><<<grid, 256, 0, stream>>>(p, b, points, st, partial);
    return cuda_status(cudaGetLastError(), "doa_level_kernel launch");
}

template <int M>
bf_status dispatch_level(int m, cudaStream_t stream, const TrackParams& p, int b, const float2* points,
                         const SearchState* st, double* partial, int n_points_max, int n_groups) {
    if constexpr (M > kMaxM) {
        return set_error(BF_ERR_UNSUPPORTED, "the DOA search supports at most 16 elements after smoothing");
    } else {
        if (m == M) return launch_level<M>(stream, p, b, points, st, partial, n_points_max, n_groups);
        return dispatch_level<M + 1>(m, stream, p, b, points, st, partial, n_points_max, n_groups);
    }
}

uint64_t align256(uint64_t x) { return (x + 255) / 256 * 256; }

}  // namespace

uint64_t doa_track_workspace_bytes(const bf_dims& d, uint64_t block_len, uint64_t subarray) {
    const uint64_t B = d.n_time / block_len, F = d.n_freq, A = d.n_ant;
    const uint64_t M = (subarray > 0 && subarray < A) ? subarray : A;
    const uint64_t groups = (F + kChanGroup - 1) / kChanGroup;
    return align256(B * F * A * A * 2 * sizeof(int32_t)) + align256(doa_fold_bytes(B * F, M)) +
           align256(kMaxPoints * sizeof(float2)) + align256(groups * kMaxPoints * sizeof(double)) +
           align256(sizeof(SearchState));
}

bf_status launch_doa_track(cudaStream_t stream, const uint8_t* v, const float* pos, const double* kw,
                           const bf_dims& d, const bf_doa_track_config& c, float* dirs, float* intensity,
                           void* workspace) {
    const uint64_t A = d.n_ant, F = d.n_freq, K = c.block_len;
    const int B = static_cast<int>(d.n_time / K);
    const int M = static_cast<int>((c.subarray > 0 && c.subarray < A) ? c.subarray : A);
    if (M > kMaxM) return set_error(BF_ERR_UNSUPPORTED, "the DOA search supports at most 16 elements after smoothing");
    const uint64_t groups = (F + kChanGroup - 1) / kChanGroup;
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    auto* R = reinterpret_cast<int32_t*>(ws);
    ws += align256(static_cast<uint64_t>(B) * F * A * A * 2 * sizeof(int32_t));
    void* fold = ws;
    ws += align256(doa_fold_bytes(static_cast<uint64_t>(B) * F, M));
    auto* points = reinterpret_cast<float2*>(ws);
    ws += align256(kMaxPoints * sizeof(float2));
    auto* partial = reinterpret_cast<double*>(ws);
    ws += align256(groups * kMaxPoints * sizeof(double));
    auto* st = reinterpret_cast<SearchState*>(ws);

    BF_RETURN_IF(launch_doa_covariance(stream, v, R, d, K));
    BF_RETURN_IF(launch_doa_fold(stream, R, d, K, M, c.forgetting, c.diag_load, fold));
    const uint64_t cells = static_cast<uint64_t>(B) * F;
    TrackParams p{};
    p.S = static_cast<const Cd*>(fold);
    p.Q = p.S + cells * M * M;
    p.ok = reinterpret_cast<const int*>(reinterpret_cast<const double*>(p.Q + cells * M * M) + cells);
    p.pos = pos;
    p.kw = kw;
    p.n_freq = static_cast<int>(F);
    p.M = M;
    p.capon = c.estimator != 0;
    const int G = static_cast<int>(c.grid), L = static_cast<int>(c.levels);
    doa_track_init_kernel<<<1, 32, 0, stream>>>(st, points, c.prior_l, c.prior_m, G, c.fov_l, c.fov_m);
    BF_RETURN_IF(cuda_status(cudaGetLastError(), "doa_track_init_kernel launch"));
    for (int b = 0; b < B; ++b) {
        for (int level = 0; level <= L; ++level) {
            const int n_max = level == 0 ? G * G : 9;
            BF_RETURN_IF(dispatch_level<1>(M, stream, p, b, points, st, partial, n_max, static_cast<int>(groups)));
            doa_select_kernel<<<1, 256, 0, stream>>>(partial, static_cast<int>(groups), points, st, level, L, G,
                                                     c.fov_l, c.fov_m, c.interp != 0, dirs + 3 * b, b + 1 == B);
            BF_RETURN_IF(cuda_status(cudaGetLastError(), "doa_select_kernel launch"));
        }
    }
    if (intensity == nullptr) return BF_OK;
    // emission: the reference-order tracker along each window's estimate
    return launch_tracker(stream, 0, v, pos, kw, dirs, intensity, nullptr, d, K);
}

}  // namespace bf
