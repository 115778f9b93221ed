/*
 * bf_oracle.c -- CPU restatement of the reference beamformer hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py may load it.  The product library (libbf_b200.so) never links,
 * loads or calls anything in this directory and has no CPU fallback.
 *
 * Every function restates one reference function in plain C, with the same
 * float32 operation order (compile with -ffp-contract=off so no FMA is
 * formed), and cites the reference file:line it follows.  Parity of this
 * restatement is pinned against the reference's own known-answer tests and
 * against the reference CPU core compiled from its sources (oracle/_ref).
 *
 * Layouts (all row-major, little endian):
 *   voltage    u8   [T][F][A]   one packed complex int4 byte per sample
 *   weights    f32  [B][F][A][2] (re, im) canonical layout
 *   intensity  f32  [T][F][B]
 *   integrated f32  [W][F][B],  W = ceil(T / S)
 *   codes      i8   [W][F][B]
 *   params     f32  [W][ceil(F/16)][ceil(B/16)][2] (offset, scale)
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_API __attribute__((visibility("default")))

static const double ORC_C = 299792458.0;                       /* physics.hpp */
static const double ORC_TWO_PI = 6.283185307179586476925286766559;

/* ------------------------------------------------------------------------ */
/* int4 contract: include/beamformer/int4.hpp:19-30                          */
/* ------------------------------------------------------------------------ */
static inline int orc_nibble(unsigned v) {
    v &= 0xFu;
    return v < 8u ? (int)v : (int)v - 16;
}

ORC_API void orc_unpack(const uint8_t* packed, size_t n, int8_t* re, int8_t* im) {
    for (size_t i = 0; i < n; ++i) {
        re[i] = (int8_t)orc_nibble(packed[i]);
        im[i] = (int8_t)orc_nibble((unsigned)packed[i] >> 4);
    }
}

/* pack_complex_int4: include/beamformer/int4.hpp:32-39 (returns -1 on range error) */
ORC_API int orc_pack(int re, int im) {
    if (re < -8 || re > 7 || im < -8 || im > 7) return -1;
    return (int)(((unsigned)re & 0xFu) | (((unsigned)im & 0xFu) << 4));
}

/* ------------------------------------------------------------------------ */
/* Steering weights: src/weights.cpp:42-55 (FP64 phase, float cos/sin)      */
/* pos [A][3], freq [F], dirs [B][3]  ->  w [B][F][A][2]                      */
/* ------------------------------------------------------------------------ */
ORC_API void orc_generate_weights(size_t A, size_t F, size_t B, const float* pos,
                                  const float* freq, const float* dirs, float* w) {
    for (size_t b = 0; b < B; ++b) {
        const float* d = dirs + 3 * b;
        for (size_t f = 0; f < F; ++f) {
            const double k = ORC_TWO_PI * (double)freq[f] / ORC_C;
            for (size_t a = 0; a < A; ++a) {
                const float* p = pos + 3 * a;
                const double delay = (double)p[0] * d[0] + (double)p[1] * d[1]
                                     + (double)p[2] * d[2];
                const double phase = k * delay;
                float* o = w + 2 * ((b * F + f) * A + a);
                o[0] = (float)cos(phase);
                o[1] = (float)sin(phase);
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Packed beamformer: src/cpu_beamformer.cpp:56-78                           */
/* sum_re += w.re*x.re - w.im*x.im ; sum_im += w.re*x.im + w.im*x.re          */
/* (weights used as stored, no conjugate), power = re*re + im*im.            */
/* ------------------------------------------------------------------------ */
static inline float orc_beam_power(const uint8_t* vrow, const float* wrow, size_t A) {
    float sr = 0.0f, si = 0.0f;
    for (size_t a = 0; a < A; ++a) {
        const float xr = (float)orc_nibble(vrow[a]);
        const float xi = (float)orc_nibble((unsigned)vrow[a] >> 4);
        const float wr = wrow[2 * a], wi = wrow[2 * a + 1];
        const float p0 = wr * xr;
        const float p1 = wi * xi;
        const float d0 = p0 - p1;
        sr = sr + d0;
        const float q0 = wr * xi;
        const float q1 = wi * xr;
        const float d1 = q0 + q1;
        si = si + d1;
    }
    const float a2 = sr * sr;
    const float b2 = si * si;
    return a2 + b2;
}

ORC_API void orc_beamform_packed_intensity(const uint8_t* v, const float* w, size_t T,
                                           size_t F, size_t A, size_t B, float* out) {
    for (size_t t = 0; t < T; ++t)
        for (size_t f = 0; f < F; ++f)
            for (size_t b = 0; b < B; ++b)
                out[(t * F + f) * B + b] =
                    orc_beam_power(v + (t * F + f) * A, w + 2 * ((b * F + f) * A), A);
}

/* Window count: src/temporal_integration.cpp:16-26 */
ORC_API size_t orc_window_count(size_t T, size_t S) {
    return S == 0 ? 0 : T / S + (T % S == 0 ? 0 : 1);
}

/* Temporal integration: src/temporal_integration.cpp:95-109 (increasing-t sum) */
ORC_API void orc_integrate(const float* I, size_t T, size_t F, size_t B, size_t S,
                           float* out) {
    const size_t W = orc_window_count(T, S);
    for (size_t win = 0; win < W; ++win) {
        const size_t t0 = win * S;
        const size_t t1 = t0 + S < T ? t0 + S : T;
        for (size_t f = 0; f < F; ++f)
            for (size_t b = 0; b < B; ++b) {
                float s = 0.0f;
                for (size_t t = t0; t < t1; ++t) s = s + I[(t * F + f) * B + b];
                out[(win * F + f) * B + b] = s;
            }
    }
}

/* Fused beamform + integrate for a window subset, identical values to
 * orc_integrate(orc_beamform_packed_intensity(...)) without the [T][F][B]
 * intermediate.  windows == NULL means all windows.  Output layout is the
 * full [W][F][B]; only the listed windows are written. */
ORC_API void orc_beamform_integrated(const uint8_t* v, const float* w, size_t T, size_t F,
                                     size_t A, size_t B, size_t S, const int64_t* windows,
                                     size_t n_windows, float* out) {
    const size_t W = orc_window_count(T, S);
    const size_t nw = windows ? n_windows : W;
    for (size_t i = 0; i < nw; ++i) {
        const size_t win = windows ? (size_t)windows[i] : i;
        if (win >= W) continue;
        const size_t t0 = win * S;
        const size_t t1 = t0 + S < T ? t0 + S : T;
        for (size_t f = 0; f < F; ++f)
            for (size_t b = 0; b < B; ++b) {
                float s = 0.0f;
                for (size_t t = t0; t < t1; ++t)
                    s = s + orc_beam_power(v + (t * F + f) * A, w + 2 * ((b * F + f) * A), A);
                out[(win * F + f) * B + b] = s;
            }
    }
}

/* FP64 version of the fused product, used to state the error of every float
 * output against an exact-arithmetic reference (sum over antennas and over
 * time in double; the weights are the float32 array as given). */
ORC_API void orc_beamform_integrated_f64(const uint8_t* v, const float* w, size_t T,
                                         size_t F, size_t A, size_t B, size_t S,
                                         const int64_t* windows, size_t n_windows,
                                         double* out) {
    const size_t W = orc_window_count(T, S);
    const size_t nw = windows ? n_windows : W;
    for (size_t i = 0; i < nw; ++i) {
        const size_t win = windows ? (size_t)windows[i] : i;
        if (win >= W) continue;
        const size_t t0 = win * S;
        const size_t t1 = t0 + S < T ? t0 + S : T;
        for (size_t f = 0; f < F; ++f)
            for (size_t b = 0; b < B; ++b) {
                double s = 0.0;
                for (size_t t = t0; t < t1; ++t) {
                    const uint8_t* vr = v + (t * F + f) * A;
                    const float* wr = w + 2 * ((b * F + f) * A);
                    double sr = 0.0, si = 0.0;
                    for (size_t a = 0; a < A; ++a) {
                        const double xr = orc_nibble(vr[a]);
                        const double xi = orc_nibble((unsigned)vr[a] >> 4);
                        sr += (double)wr[2 * a] * xr - (double)wr[2 * a + 1] * xi;
                        si += (double)wr[2 * a] * xi + (double)wr[2 * a + 1] * xr;
                    }
                    s += sr * sr + si * si;
                }
                out[(win * F + f) * B + b] = s;
            }
    }
}

/* ------------------------------------------------------------------------ */
/* int8 chunk quantizer: src/quantization.cpp:20-30, 61-161                  */
/* one (offset, scale) per 1x16x16 (window x freq x beam) chunk; codes in     */
/* [-127,127] via lrint (round half even), -128 marks a non-finite value.    */
/* ------------------------------------------------------------------------ */
ORC_API void orc_quantize(const float* I, size_t W, size_t F, size_t B, int8_t* codes,
                          float* params) {
    const size_t ft = (F + 15) / 16, bt = (B + 15) / 16;
    const float out_min = -127.0f - 0.5f, out_max = 127.0f + 0.5f;
    const float out_range = out_max - out_min;
    for (size_t w = 0; w < W; ++w)
        for (size_t fi = 0; fi < ft; ++fi)
            for (size_t bi = 0; bi < bt; ++bi) {
                float mn = INFINITY, mx = -INFINITY;
                int nonfinite = 0;
                for (size_t f = fi * 16; f < fi * 16 + 16 && f < F; ++f)
                    for (size_t b = bi * 16; b < bi * 16 + 16 && b < B; ++b) {
                        const float x = I[(w * F + f) * B + b];
                        if (!isfinite(x)) nonfinite = 1;
                        else {
                            mn = x < mn ? x : mn;
                            mx = x > mx ? x : mx;
                        }
                    }
                float offset = 0.0f, scale = 0.0f;
                if (!nonfinite && isfinite(mn) && isfinite(mx)) {
                    scale = (mx - mn) / out_range;
                    const float t = out_min * scale;
                    offset = mn - t;
                    if (!isfinite(offset) || !isfinite(scale)) offset = scale = 0.0f;
                }
                float* p = params + 2 * ((w * ft + fi) * bt + bi);
                p[0] = offset;
                p[1] = scale;
                for (size_t f = fi * 16; f < fi * 16 + 16 && f < F; ++f)
                    for (size_t b = bi * 16; b < bi * 16 + 16 && b < B; ++b) {
                        const size_t idx = (w * F + f) * B + b;
                        const float x = I[idx];
                        int code;
                        if (!isfinite(x)) code = -128;
                        else if (scale == 0.0f) code = 0;
                        else {
                            const float num = x - offset;
                            const float q = num / scale;
                            long r = lrintf(q);
                            code = (int)(r < -127 ? -127 : (r > 127 ? 127 : r));
                        }
                        codes[idx] = (int8_t)code;
                    }
            }
}

/* ------------------------------------------------------------------------ */
/* Tracker: src/beam_tracker.cpp:44-76 (window directions) and :115-145      */
/* (one weight set per window, per-spectrum |sum w x|^2, n_beams == 1).       */
/* ------------------------------------------------------------------------ */

/* direction_from_lm: src/geometry.cpp:97-106. returns 0 on success. */
ORC_API int orc_direction_from_lm(float l, float m, float* out3) {
    if (!isfinite(l) || !isfinite(m)) return -1;
    const float a = l * l;
    const float b = m * m;
    const float tr = a + b;
    if (tr > 1.0f) return -1;
    out3[0] = l;
    out3[1] = m;
    out3[2] = sqrtf(1.0f - tr);
    return 0;
}

/* tracker_window_direction: src/beam_tracker.cpp:52-76, one per window:
 * l = l0 + (float)(w*S) * rate_l, m likewise, then direction_from_lm. */
ORC_API int orc_tracker_window_directions(float l0, float m0, float rate_l, float rate_m,
                                          size_t T, size_t S, float* dirs /*[W][3]*/) {
    const size_t W = orc_window_count(T, S);
    for (size_t w = 0; w < W; ++w) {
        const float tf = (float)(w * S);
        const float dl = tf * rate_l;
        const float dm = tf * rate_m;
        const float l = l0 + dl;
        const float m = m0 + dm;
        if (orc_direction_from_lm(l, m, dirs + 3 * w) != 0) return -1;
    }
    return 0;
}

/* Per-window weights [W][F][A][2] from positions, frequencies and the window
 * directions (src/beam_tracker.cpp:130-134 -> src/weights.cpp:42-55). */
ORC_API void orc_tracker_weights(size_t W, size_t F, size_t A, const float* pos,
                                 const float* freq, const float* dirs, float* w) {
    for (size_t win = 0; win < W; ++win)
        orc_generate_weights(A, F, 1, pos, freq, dirs + 3 * win, w + (size_t)2 * win * F * A);
}

/* Per-spectrum tracker intensity [T][F] (src/beam_tracker.cpp:136-145). */
ORC_API void orc_tracker(const uint8_t* v, const float* window_weights, size_t T, size_t F,
                         size_t A, size_t S, float* out) {
    for (size_t t = 0; t < T; ++t) {
        const float* ww = window_weights + (size_t)2 * (t / S) * F * A;
        for (size_t f = 0; f < F; ++f)
            out[t * F + f] = orc_beam_power(v + (t * F + f) * A, ww + 2 * f * A, A);
    }
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic voltages.  Not a reference function: the reference's     */
/* make_noise (src/synthetic_data.cpp:107-119) draws uniform [-7,7] from     */
/* std::mt19937.  This generator draws an approximately Gaussian component   */
/* (sum of eight 16-bit uniforms, Irwin-Hall), scales it by sigma, adds the  */
/* source term mu, rounds half-to-even and clips to [-8, 7].  It uses only   */
/* integer hashing and correctly rounded float32 mul/add, so the CUDA        */
/* generator produces identical bytes.                                       */
/* ------------------------------------------------------------------------ */
static inline uint64_t orc_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline int orc_irwin_hall8(uint64_t seed, uint64_t counter) {
    const uint64_t h0 = orc_mix64(seed ^ orc_mix64(2 * counter));
    const uint64_t h1 = orc_mix64(seed ^ orc_mix64(2 * counter + 1));
    int s = 0;
    for (int i = 0; i < 4; ++i) {
        s += (int)((h0 >> (16 * i)) & 0xFFFFu);
        s += (int)((h1 >> (16 * i)) & 0xFFFFu);
    }
    /* 2*sum - 8*65535: zero mean, odd integer, |.| < 2^20 (exact in float) */
    return 2 * s - 8 * 65535;
}

static inline int orc_round_clip(float x) {
    const float r = nearbyintf(x); /* default rounding mode: half to even */
    int i = (int)r;
    return i < -8 ? -8 : (i > 7 ? 7 : i);
}

/* scale = sigma / std(2*sum - 8*65535) rounded to float by the caller.
 * mu (optional) is [U][F][A][2] (re, im) float, epoch u = t / epoch_len.  */
ORC_API void orc_generate_voltage(uint64_t seed, uint64_t sample_offset, size_t T, size_t F,
                                  size_t A, float scale, const float* mu, size_t epoch_len,
                                  uint8_t* out) {
    for (size_t t = 0; t < T; ++t)
        for (size_t f = 0; f < F; ++f)
            for (size_t a = 0; a < A; ++a) {
                const size_t i = (t * F + f) * A + a;
                float mr = 0.0f, mi = 0.0f;
                if (mu) {
                    const float* m = mu + 2 * (((t / epoch_len) * F + f) * A + a);
                    mr = m[0];
                    mi = m[1];
                }
                const uint64_t c = sample_offset + (uint64_t)i;
                const float gr = (float)orc_irwin_hall8(seed, 2 * c);
                const float gi = (float)orc_irwin_hall8(seed, 2 * c + 1);
                const float xr = gr * scale;
                const float xi = gi * scale;
                const float yr = xr + mr;
                const float yi = xi + mi;
                const int re = orc_round_clip(yr), im = orc_round_clip(yi);
                out[i] = (uint8_t)(((unsigned)re & 0xFu) | (((unsigned)im & 0xFu) << 4));
            }
}

/* ------------------------------------------------------------------------ */
/* DOA scan in FP64 (restates src/cpu_opt_beam_tracker.cpp in double):       */
/*  smoothing over sub-arrays along the linear element index and             */
/*  forward-backward averaging (:605-657), diagonal loading                  */
/*  eps = load * tr(R) / M applied to each block before forgetting           */
/*  (:226-237, :1866-1880), forgetting R = lam R + (1 - lam) R_blk           */
/*  (:1763-1892), Cholesky (:398-415), Capon 1 / ||L^-1 a||^2 (:423-437),    */
/*  Bartlett a^H R a (:287-302), steering a_i = exp(-j k (x_i l + y_i m))    */
/*  (:96-106), powers summed over frequency.  The peak is refined by the      */
/*  vertex of the parabola through the argmax and its neighbours (the        */
/*  reference's quadratic_interp, :830-850, only accepts convex triples and   */
/*  so never moves a maximum; here the concave vertex is used).              */
/* Inputs: R [B][F][A][A][2] int64 block sums of x x^H over K spectra.       */
/* Outputs: bartlett, capon [B][n]; l_est [B][2] (bartlett, capon).          */
/* ------------------------------------------------------------------------ */
ORC_API void orc_doa_scan(const int64_t* R, size_t B, size_t F, size_t A, size_t K,
                          size_t subarray, double lam, double load, const float* pos,
                          const double* kw, double l_first, double l_step, size_t n,
                          double m_fixed, double* bartlett, double* capon, double* l_est) {
    const size_t M = (subarray > 0 && subarray < A) ? subarray : A;
    const size_t L = A - M + 1;
    double* S = (double*)calloc(2 * F * M * M, sizeof(double)); /* folded state */
    double* E = (double*)calloc(F, sizeof(double));
    double* Rb = (double*)malloc(sizeof(double) * 2 * M * M);
    double* Rt = (double*)malloc(sizeof(double) * 2 * M * M);
    double* Lc = (double*)malloc(sizeof(double) * 2 * M * M);
    double* ar = (double*)malloc(sizeof(double) * M);
    double* ai = (double*)malloc(sizeof(double) * M);
    double* vr = (double*)malloc(sizeof(double) * M);
    double* vi = (double*)malloc(sizeof(double) * M);
    for (size_t b = 0; b < B; ++b) {
        for (size_t l = 0; l < n; ++l) bartlett[b * n + l] = capon[b * n + l] = 0.0;
        for (size_t f = 0; f < F; ++f) {
            const int64_t* Rf = R + 2 * (b * F + f) * A * A;
            /* smoothing: mean over sub-arrays of the 1/K covariance */
            for (size_t r = 0; r < M; ++r)
                for (size_t c = 0; c < M; ++c) {
                    double sr = 0.0, si = 0.0;
                    for (size_t s = 0; s < L; ++s) {
                        sr += (double)Rf[2 * ((s + r) * A + s + c)];
                        si += (double)Rf[2 * ((s + r) * A + s + c) + 1];
                    }
                    Rt[2 * (r * M + c)] = sr / (double)K / (double)L;
                    Rt[2 * (r * M + c) + 1] = si / (double)K / (double)L;
                }
            /* forward-backward: 1/2 (R + J conj(R) J) when smoothing */
            for (size_t r = 0; r < M; ++r)
                for (size_t c = 0; c < M; ++c) {
                    double re = Rt[2 * (r * M + c)], im = Rt[2 * (r * M + c) + 1];
                    if (L > 1) {
                        const size_t pr = M - 1 - r, pc = M - 1 - c;
                        re = 0.5 * (re + Rt[2 * (pr * M + pc)]);
                        im = 0.5 * (im - Rt[2 * (pr * M + pc) + 1]);
                    }
                    Rb[2 * (r * M + c)] = re;
                    Rb[2 * (r * M + c) + 1] = im;
                }
            double tr = 0.0;
            for (size_t r = 0; r < M; ++r) tr += Rb[2 * (r * M + r)];
            const double eps = load * tr / (double)M;
            double* Sf = S + 2 * f * M * M;
            if (b == 0 || lam >= 1.0) {
                for (size_t i = 0; i < 2 * M * M; ++i) Sf[i] = Rb[i];
                E[f] = eps;
            } else {
                for (size_t i = 0; i < 2 * M * M; ++i) Sf[i] = lam * Sf[i] + (1.0 - lam) * Rb[i];
                E[f] = lam * E[f] + (1.0 - lam) * eps;
            }
            /* Cholesky of S + E I (lower, FP64) */
            int ok = 1;
            for (size_t i = 0; i < M && ok; ++i)
                for (size_t j = 0; j <= i; ++j) {
                    double sr = Sf[2 * (i * M + j)] + (i == j ? E[f] : 0.0);
                    double si = Sf[2 * (i * M + j) + 1];
                    for (size_t k = 0; k < j; ++k) {
                        const double xr = Lc[2 * (i * M + k)], xi = Lc[2 * (i * M + k) + 1];
                        const double yr = Lc[2 * (j * M + k)], yi = -Lc[2 * (j * M + k) + 1];
                        sr -= xr * yr - xi * yi;
                        si -= xr * yi + xi * yr;
                    }
                    if (i == j) {
                        if (sr <= 1e-300) { ok = 0; break; }
                        Lc[2 * (i * M + i)] = sqrt(sr);
                        Lc[2 * (i * M + i) + 1] = 0.0;
                    } else {
                        const double d = Lc[2 * (j * M + j)];
                        Lc[2 * (i * M + j)] = sr / d;
                        Lc[2 * (i * M + j) + 1] = si / d;
                    }
                }
            for (size_t l = 0; l < n; ++l) {
                const double lv = l_first + (double)l * l_step;
                for (size_t i = 0; i < M; ++i) {
                    const double ph = kw[f] * ((double)pos[3 * i] * lv + (double)pos[3 * i + 1] * m_fixed);
                    const double rr = ph - 6.283185307179586476925286766559 *
                                               nearbyint(ph * (1.0 / 6.283185307179586476925286766559));
                    const float rf = (float)rr;
                    ar[i] = (double)cosf(rf);
                    ai[i] = -(double)sinf(rf);
                }
                /* Bartlett: sum_rc conj(a_r) S_rc a_c */
                double pb = 0.0;
                for (size_t r = 0; r < M; ++r) {
                    double tr2 = 0.0, ti2 = 0.0;
                    for (size_t c = 0; c < M; ++c) {
                        const double sr = Sf[2 * (r * M + c)], si = Sf[2 * (r * M + c) + 1];
                        tr2 += sr * ar[c] - si * ai[c];
                        ti2 += sr * ai[c] + si * ar[c];
                    }
                    pb += ar[r] * tr2 + ai[r] * ti2; /* Re(conj(a_r) * t) */
                }
                bartlett[b * n + l] += pb;
                if (ok) {
                    double nrm = 0.0;
                    for (size_t i = 0; i < M; ++i) {
                        double sr = ar[i], si = ai[i];
                        for (size_t k = 0; k < i; ++k) {
                            const double xr = Lc[2 * (i * M + k)], xi = Lc[2 * (i * M + k) + 1];
                            sr -= xr * vr[k] - xi * vi[k];
                            si -= xr * vi[k] + xi * vr[k];
                        }
                        const double d = Lc[2 * (i * M + i)];
                        vr[i] = sr / d;
                        vi[i] = si / d;
                        nrm += vr[i] * vr[i] + vi[i] * vi[i];
                    }
                    capon[b * n + l] += nrm > 0.0 ? 1.0 / nrm : 0.0;
                }
            }
        }
        for (int e = 0; e < 2; ++e) {
            const double* P = (e == 0 ? bartlett : capon) + b * n;
            size_t best = 0;
            for (size_t l = 1; l < n; ++l)
                if (P[l] > P[best]) best = l;
            double delta = 0.0;
            if (best > 0 && best + 1 < n) {
                const double den = P[best - 1] - 2.0 * P[best] + P[best + 1];
                if (den < 0.0) {
                    delta = 0.5 * (P[best - 1] - P[best + 1]) / den;
                    if (delta > 0.5) delta = 0.5;
                    if (delta < -0.5) delta = -0.5;
                }
            }
            l_est[2 * b + e] = l_first + ((double)best + delta) * l_step;
        }
    }
    free(S); free(E); free(Rb); free(Rt); free(Lc); free(ar); free(ai); free(vr); free(vi);
}

/* ------------------------------------------------------------------------ */
/* DOA covariance.  Reference: src/cpu_opt_beam_tracker.cpp:559-602 forms     */
/* R[f] = (1/K) sum_k x_k x_k^H in std::complex<float> per frequency.  The   */
/* integer restatement below returns the exact per-block sum in int64       */
/* (re, im), from which the float32 reference value is sum * (1/K) exactly   */
/* when K is a power of two and every partial sum stays below 2^24.          */
/* R layout: [F][A][A][2] (row i, column j) = sum_t x_i * conj(x_j).          */
/* ------------------------------------------------------------------------ */
ORC_API void orc_covariance_block_i64(const uint8_t* v, size_t T, size_t F, size_t A,
                                      int64_t* R) {
    memset(R, 0, sizeof(int64_t) * 2 * F * A * A);
    for (size_t t = 0; t < T; ++t)
        for (size_t f = 0; f < F; ++f) {
            const uint8_t* row = v + (t * F + f) * A;
            int64_t* Rf = R + 2 * f * A * A;
            for (size_t i = 0; i < A; ++i) {
                const int xr = orc_nibble(row[i]), xi = orc_nibble((unsigned)row[i] >> 4);
                for (size_t j = 0; j < A; ++j) {
                    const int yr = orc_nibble(row[j]), yi = orc_nibble((unsigned)row[j] >> 4);
                    /* x_i * conj(x_j) */
                    Rf[2 * (i * A + j)] += xr * yr + xi * yi;
                    Rf[2 * (i * A + j) + 1] += xi * yr - xr * yi;
                }
            }
        }
}
