// ref_shim.cpp -- extern "C" entry points into the reference CPU core.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build.py compiles this file together
// with the reference's own CPU sources (read where they lie in the reference
// checkout, never copied) into oracle/_ref/libbfref.so.  Tests use it to pin
// the C restatement (bf_oracle.c) and the CUDA kernels to the reference's
// actual outputs; bench.py's reference arm times it on the host cores.
// Every function returns 0 on success or a nonzero code with the exception
// text available from ref_last_error().
#include <beamformer/beam_tracker.hpp>
#include <beamformer/beam_tracker_opt_v2.hpp>
#include <beamformer/cpu_opt_beam_tracker.hpp>
#include <beamformer/cpu_beamformer.hpp>
#include <beamformer/geometry.hpp>
#include <beamformer/io.hpp>
#include <beamformer/quantization.hpp>
#include <beamformer/synthetic_data.hpp>
#include <beamformer/temporal_integration.hpp>
#include <beamformer/weights.hpp>

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

using namespace beamformer;

namespace {
thread_local std::string g_err;

template <class Fn>
int guarded(Fn&& fn) {
    try {
        fn();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return 1;
    } catch (const std::logic_error& e) {
        g_err = e.what();
        return 2;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 3;
    }
}

Dimensions dims_of(uint64_t t, uint64_t f, uint64_t a, uint64_t b) {
    return Dimensions{t, f, a, b};
}

std::vector<Vec3> vec3s(const float* p, size_t n) {
    std::vector<Vec3> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    return out;
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_max_threads() { return omp_get_max_threads(); }

// src/cpu_beamformer.cpp:40-79
int ref_cpu_beamform_packed_intensity(const uint8_t* v, const float* w, uint64_t T, uint64_t F,
                                      uint64_t A, uint64_t B, float* out) {
    return guarded([&] {
        const Dimensions d = dims_of(T, F, A, B);
        PackedVoltage pv(v, v + T * F * A);
        Weights wv(B * F * A);
        std::memcpy(wv.data(), w, wv.size() * sizeof(ComplexFloat));
        Intensities I(T * F * B);
        cpu_beamform_packed_intensity_into(pv, wv, d, I);
        std::memcpy(out, I.data(), I.size() * sizeof(float));
    });
}

// src/temporal_integration.cpp:79-110
int ref_cpu_integrate(const float* I, uint64_t T, uint64_t F, uint64_t A, uint64_t B,
                      uint64_t S, float* out) {
    return guarded([&] {
        const Dimensions d = dims_of(T, F, A, B);
        Intensities in(I, I + T * F * B);
        IntegratedIntensities o(integrated_intensity_count(d, S));
        cpu_integrate_intensity_into(in, d, S, o);
        std::memcpy(out, o.data(), o.size() * sizeof(float));
    });
}

// src/quantization.cpp:61-161 (integrated dims: n_time = windows)
int ref_cpu_quantize(const float* I, uint64_t W, uint64_t F, uint64_t A, uint64_t B,
                     int8_t* codes, float* params) {
    return guarded([&] {
        const Dimensions d = dims_of(W, F, A, B);
        IntegratedIntensities in(I, I + W * F * B);
        const auto q = cpu_quantize_integrated_intensity(in, d);
        std::memcpy(codes, q.codes.data(), q.codes.size());
        std::memcpy(params, q.parameters.data(), q.parameters.size() * 2 * sizeof(float));
    });
}

// src/weights.cpp:11-60
int ref_generate_weights(uint64_t A, uint64_t F, uint64_t B, const float* pos,
                         const float* freq, const float* dirs, float* out) {
    return guarded([&] {
        const Dimensions d = dims_of(1, F, A, B);
        const auto w = generate_weights(d, vec3s(pos, A), std::vector<float>(freq, freq + F),
                                        vec3s(dirs, B));
        std::memcpy(out, w.data(), w.size() * sizeof(ComplexFloat));
    });
}

// src/weights.cpp:63-122
int ref_generate_tiled_weights(uint64_t A, uint64_t F, uint64_t B, const float* pos,
                               const float* freq, const float* dirs, float* out) {
    return guarded([&] {
        const Dimensions d = dims_of(1, F, A, B);
        const auto w = generate_tiled_weights(d, vec3s(pos, A),
                                              std::vector<float>(freq, freq + F), vec3s(dirs, B));
        std::memcpy(out, w.data(), w.size() * sizeof(ComplexFloat));
    });
}

// src/geometry.cpp:53-67, :79-95
int ref_default_positions(uint64_t A, float* out) {
    return guarded([&] {
        const auto p = default_positions(A);
        for (size_t i = 0; i < p.size(); ++i)
            for (int c = 0; c < 3; ++c) out[3 * i + c] = p[i][c];
    });
}

int ref_channelized_frequencies(uint64_t F, float* out) {
    return guarded([&] {
        const auto f = channelized_frequencies(F);
        std::memcpy(out, f.data(), f.size() * sizeof(float));
    });
}

// src/beam_tracker.cpp:67-76
int ref_tracker_window_direction(float l0, float m0, float rl, float rm, uint64_t window,
                                 uint64_t S, float* out3) {
    return guarded([&] {
        TrackerTrajectoryConfig tr;
        tr.direction_start = direction_from_lm(l0, m0);
        tr.direction_rate_per_sample = {rl, rm};
        const auto d = tracker_window_direction(tr, window, S);
        out3[0] = d[0];
        out3[1] = d[1];
        out3[2] = d[2];
    });
}

static TrackerConfig tracker_config(float l0, float m0, float rl, float rm, uint64_t S) {
    TrackerConfig cfg;
    cfg.trajectory.direction_start = direction_from_lm(l0, m0);
    cfg.trajectory.direction_rate_per_sample = {rl, rm};
    cfg.integration_spectra = S;
    return cfg;
}

// src/beam_tracker.cpp:90-146 (naive) and src/beam_tracker_opt_v2.cpp:143-311 (OpenMP)
int ref_beam_tracker(int variant, const uint8_t* v, uint64_t T, uint64_t F, uint64_t A,
                     float l0, float m0, float rl, float rm, uint64_t S, float* out) {
    return guarded([&] {
        const Dimensions d = dims_of(T, F, A, 1);
        PackedVoltage pv(v, v + T * F * A);
        Intensities I(T * F);
        const TrackerConfig cfg = tracker_config(l0, m0, rl, rm, S);
        if (variant == 0) {
            beam_tracker_cpu_packed_intensity_into(pv, d, cfg, I);
        } else {
            beam_tracker_opt_v2_cpu_packed_intensity_into(pv, d, cfg, I);
        }
        std::memcpy(out, I.data(), I.size() * sizeof(float));
    });
}

// src/synthetic_data.cpp:50-119
int ref_make_noise(uint64_t T, uint64_t F, uint64_t A, uint32_t seed, uint8_t* out) {
    return guarded([&] {
        const auto v = make_noise(dims_of(T, F, A, 1), seed);
        std::memcpy(out, v.data(), v.size());
    });
}

int ref_make_one_hot(uint64_t T, uint64_t F, uint64_t A, uint64_t t, uint64_t f, uint64_t a,
                     int re, int im, uint8_t* out) {
    return guarded([&] {
        const auto v = make_one_hot(dims_of(T, F, A, 1), t, f, a,
                                    ComplexInt4{static_cast<int8_t>(re), static_cast<int8_t>(im)});
        std::memcpy(out, v.data(), v.size());
    });
}

int ref_make_point_source(uint64_t T, uint64_t F, uint64_t A, const float* pos,
                          const float* freq, const float* dir, float amplitude, uint8_t* out) {
    return guarded([&] {
        const auto v = make_point_source(dims_of(T, F, A, 1), vec3s(pos, A),
                                         std::vector<float>(freq, freq + F),
                                         Vec3{dir[0], dir[1], dir[2]}, amplitude);
        std::memcpy(out, v.data(), v.size());
    });
}

// src/beam_tracker.cpp:148-192
int ref_make_moving_point_source(uint64_t T, uint64_t F, uint64_t A, const float* pos,
                                 const float* freq, float l0, float m0, float rl, float rm,
                                 float amplitude, uint8_t* out) {
    return guarded([&] {
        TrackerTrajectoryConfig tr;
        tr.direction_start = direction_from_lm(l0, m0);
        tr.direction_rate_per_sample = {rl, rm};
        const auto v = beam_tracker_make_moving_point_source(
            dims_of(T, F, A, 1), vec3s(pos, A), std::vector<float>(freq, freq + F), tr, amplitude);
        std::memcpy(out, v.data(), v.size());
    });
}

// CpuOptBeamTracker (include/beamformer/cpu_opt_beam_tracker.hpp:91-169):
// run the DOA search over all windows and return each window's direction
// and, when intensity is given, the emitted [T][F] beam power.
int ref_doa_directions(const uint8_t* v, uint64_t T, uint64_t F, uint64_t A, const float* pos,
                       const float* freq, int capon, uint64_t G, uint64_t levels, float fov_l,
                       float fov_m, uint64_t subarray, float lam, float load, uint64_t K, float l0,
                       float m0, float* dirs, float* intensity) {
    return guarded([&] {
        const Dimensions d = dims_of(T, F, A, 1);
        CpuOptTrackerConfig cfg;
        cfg.estimator = capon ? TrackerEstimator::Capon : TrackerEstimator::Bartlett;
        cfg.coarse_grid_resolution = G;
        cfg.refinement_levels = levels;
        cfg.search_fov_l = fov_l;
        cfg.search_fov_m = fov_m;
        cfg.spatial_smoothing_subarray_size = subarray;
        cfg.forgetting_factor = lam;
        cfg.diagonal_load = load;
        cfg.integration_spectra = K;
        CpuOptBeamTracker tracker(vec3s(pos, A), std::vector<float>(freq, freq + F), d, cfg);
        TrackerTrajectoryConfig prior;
        prior.direction_start = direction_from_lm(l0, m0);
        tracker.seed_trajectory(prior);
        PackedVoltage pv(v, v + T * F * A);
        Intensities I(T * F);
        tracker.run_into(pv, I);
        if (intensity != nullptr) std::memcpy(intensity, I.data(), I.size() * sizeof(float));
        const std::size_t W = tracker_window_count(T, K);
        for (std::size_t w = 0; w < W; ++w) {
            const Vec3 dd = tracker.window_direction(w);
            dirs[3 * w] = dd[0];
            dirs[3 * w + 1] = dd[1];
            dirs[3 * w + 2] = dd[2];
        }
    });
}

// src/io.cpp:60-344: every file format, written by the reference into dir
// (voltage.bin, weights.bin, tiled.bin, intensity.bin, codes.bin,
// params.bin, int8_meta.txt, shard_payload.bin, shard_meta.txt,
// shard_loss.bin).  Dimensions T x F x A x B; the int8 files hold
// W = ceil(T / S) windows; the shard descriptor is the default one of
// shard_id with the given timestamps and loss-mask id.
int ref_io_write(const char* dir, const uint8_t* volt, const float* w, const float* tw, const float* inten,
                 const int8_t* codes, const float* params, const uint8_t* loss, uint64_t T, uint64_t F,
                 uint64_t A, uint64_t B, uint64_t S, uint64_t shard_id, uint64_t ts_start, uint64_t ts_step,
                 uint64_t loss_id) {
    return guarded([&] {
        const std::string base(dir);
        const Dimensions d = dims_of(T, F, A, B);
        const std::size_t W = integrated_time_count(T, TemporalIntegrationConfig{S});
        const Dimensions wd = dims_of(W, F, A, B);
        write_packed_voltage(base + "/voltage.bin", PackedVoltage(volt, volt + T * F * A), d);
        Weights wv(B * F * A);
        std::memcpy(wv.data(), w, wv.size() * sizeof(ComplexFloat));
        write_weights(base + "/weights.bin", wv, d);
        TiledWeights tv(tiled_weight_count(d));
        std::memcpy(tv.data(), tw, tv.size() * sizeof(ComplexFloat));
        write_tiled_weights(base + "/tiled.bin", tv, d);
        write_intensities(base + "/intensity.bin", Intensities(inten, inten + T * F * B), d);
        write_quantized_intensities(base + "/codes.bin", QuantizedIntensities(codes, codes + W * F * B), wd);
        std::vector<Int8QuantizationParameters> pv(quantization_parameter_count(wd));
        std::memcpy(pv.data(), params, pv.size() * sizeof(Int8QuantizationParameters));
        write_quantization_parameters(base + "/params.bin", pv, wd);
        ShardDescriptor sd = default_shard_descriptors()[shard_id];
        sd.timestamp_start = ts_start;
        sd.timestamp_step = ts_step;
        sd.loss_mask_id = loss_id;
        write_quantized_output_metadata(base + "/int8_meta.txt",
                                        QuantizedOutputMetadata{wd, T, TemporalIntegrationConfig{S}, sd, "params.bin"});
        PackedShard shard{sd, PackedVoltage(volt, volt + T * F * A), LossMask(loss, loss + T * F)};
        write_packed_shard(base + "/shard_payload.bin", base + "/shard_meta.txt", base + "/shard_loss.bin", shard, d);
    });
}

// Reads every file of ref_io_write's set from dir with the reference's
// readers; returns 0 when all contents equal the given arrays and fields.
int ref_io_read_check(const char* dir, const uint8_t* volt, const float* w, const float* tw, const int8_t* codes,
                      const float* params, const uint8_t* loss, uint64_t T, uint64_t F, uint64_t A, uint64_t B,
                      uint64_t S, uint64_t shard_id, uint64_t ts_start, uint64_t ts_step, uint64_t loss_id) {
    return guarded([&] {
        const std::string base(dir);
        const Dimensions d = dims_of(T, F, A, B);
        const std::size_t W = integrated_time_count(T, TemporalIntegrationConfig{S});
        const Dimensions wd = dims_of(W, F, A, B);
        auto same = [](const void* a, const void* b, std::size_t n, const char* what) {
            if (std::memcmp(a, b, n) != 0) throw std::runtime_error(std::string("content differs: ") + what);
        };
        const auto v = read_packed_voltage(base + "/voltage.bin", d);
        same(v.data(), volt, v.size(), "voltage");
        const auto wv = read_weights(base + "/weights.bin", d);
        same(wv.data(), w, wv.size() * sizeof(ComplexFloat), "weights");
        const auto tv = read_tiled_weights(base + "/tiled.bin", d);
        same(tv.data(), tw, tv.size() * sizeof(ComplexFloat), "tiled weights");
        const auto cv = read_quantized_intensities(base + "/codes.bin", wd);
        same(cv.data(), codes, cv.size(), "codes");
        const auto pv = read_quantization_parameters(base + "/params.bin", wd);
        same(pv.data(), params, pv.size() * sizeof(Int8QuantizationParameters), "parameters");
        const auto md = read_quantized_output_metadata(base + "/int8_meta.txt");
        if (md.output_dims.n_time != W || md.input_n_time != T || md.temporal_integration.integration_spectra != S ||
            md.shard.shard_id != shard_id || md.shard.timestamp_start != ts_start ||
            md.shard.timestamp_step != ts_step || md.shard.loss_mask_id != loss_id ||
            md.parameters_file != "params.bin") {
            throw std::runtime_error("int8 metadata fields differ");
        }
        const auto sh = read_packed_shard(base + "/shard_payload.bin", base + "/shard_meta.txt",
                                          base + "/shard_loss.bin", d);
        same(sh.payload.data(), volt, sh.payload.size(), "shard payload");
        same(sh.loss_mask.data(), loss, sh.loss_mask.size(), "shard loss mask");
        if (sh.descriptor.shard_id != shard_id || sh.descriptor.timestamp_start != ts_start ||
            sh.descriptor.loss_mask_id != loss_id) {
            throw std::runtime_error("shard descriptor fields differ");
        }
    });
}

}  // extern "C"
