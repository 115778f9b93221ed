// test_cxx_api.cpp -- the C++ drop-in API (include/beamformer/) exercised the
// way the reference's own CUDA tests exercise theirs (tests/cuda/*.cpp in
// the reference): exception types, known answers, workspace reuse, device
// frames, the quantized pipeline, the TensorSplit kernel and the tracker.
// Plain executable: prints one line per check, exits 0 when all pass.
#include "beamformer/beam_tracker.hpp"
#include "beamformer/cuda_beam_tracker_v5.hpp"
#include "beamformer/cuda_beamformer.hpp"
#include "beamformer/geometry.hpp"
#include "beamformer/served.hpp"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

using namespace beamformer;

namespace {

int failures = 0;

void expect(bool ok, const std::string& what) {
    std::printf("%s %s\n", ok ? "ok  " : "FAIL", what.c_str());
    if (!ok) ++failures;
}

template <class E>
bool throws(const std::function<void()>& fn) {
    try {
        fn();
    } catch (const E&) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

// Reference float32 order (src/cpu_beamformer.cpp:56-78), for small checks.
float cpu_power(const PackedVoltage& v, const Weights& w, const Dimensions& d, std::size_t t, std::size_t f,
                std::size_t b) {
    volatile float sr = 0.f, si = 0.f;
    for (std::size_t a = 0; a < d.n_ant; ++a) {
        const auto x = unpack_complex_int4(v[voltage_index(t, f, a, d)]);
        const float xr = x.real, xi = x.imag;
        const auto& wv = w[weight_index(b, f, a, d)];
        volatile float p0 = wv.real * xr, p1 = wv.imag * xi, q0 = wv.real * xi, q1 = wv.imag * xr;
        volatile float d0 = p0 - p1, d1 = q0 + q1;
        sr = sr + d0;
        si = si + d1;
    }
    volatile float a2 = sr * sr, b2 = si * si;
    return a2 + b2;
}

Weights weights_for(const Dimensions& d, const std::vector<Vec3>& dirs) {
    const auto pos = default_positions(d.n_ant);
    const auto freq = channelized_frequencies(d.n_freq);
    Weights w(d.n_beams * d.n_freq * d.n_ant);
    for (std::size_t b = 0; b < d.n_beams; ++b)
        for (std::size_t f = 0; f < d.n_freq; ++f) {
            const double k = 6.283185307179586476925286766559 * freq[f] / 299792458.0;
            for (std::size_t a = 0; a < d.n_ant; ++a) {
                const double delay = static_cast<double>(pos[a][0]) * dirs[b][0] +
                                     static_cast<double>(pos[a][1]) * dirs[b][1] +
                                     static_cast<double>(pos[a][2]) * dirs[b][2];
                w[weight_index(b, f, a, d)] = {static_cast<float>(std::cos(k * delay)),
                                               static_cast<float>(std::sin(k * delay))};
            }
        }
    return w;
}

TiledWeights tile(const Weights& w, const Dimensions& d) {
    TiledWeights t(tiled_weight_count(d), ComplexFloat{0.f, 0.f});
    for (std::size_t b = 0; b < d.n_beams; ++b)
        for (std::size_t f = 0; f < d.n_freq; ++f)
            for (std::size_t a = 0; a < d.n_ant; ++a)
                t[tiled_weight_index(f, b / 32, a, b % 32, d)] = w[weight_index(b, f, a, d)];
    return t;
}

PackedVoltage random_voltage(const Dimensions& d, unsigned seed) {
    std::mt19937 rng(seed);
    PackedVoltage v(voltage_sample_count(d));
    for (auto& x : v) x = static_cast<std::uint8_t>(rng() & 0xFF);
    return v;
}

}  // namespace

int main() {
    // ---- dimension and selector rules (config.hpp:81-94, cuda_beamformer.cu:418-433)
    expect(throws<std::invalid_argument>([] { validate_dimensions(Dimensions{0, 336, 32, 1}); }), "n_time 0 rejected");
    expect(throws<std::invalid_argument>([] { CudaBeamformerWorkspace ws(Dimensions{8, 336, 32, 4}, CudaBeamformerKernel::Direct, TemporalIntegrationConfig{10}); }),
           "Direct kernel rejects 10-spectrum integration");
    expect(throws<std::invalid_argument>([] { CudaBeamformerWorkspace ws(Dimensions{8, 336, 32, 4}, CudaBeamformerKernel::Tiled, std::nullopt, CudaBeamformerOutput::QuantizedInt8); }),
           "int8 output needs integration");
    {
        CudaBeamformerWorkspace ws(Dimensions{8, 336, 32, 4});
        expect(throws<std::logic_error>([&] { ws.run_kernel(Dimensions{8, 336, 32, 4}); }), "run before upload is a logic_error");
        expect(throws<std::invalid_argument>([&] { ws.upload_packed_voltage(PackedVoltage(16, 0), Dimensions{16, 336, 32, 4}); }),
               "capacity exceeded");
    }
    const auto info = cuda_device_info();
    expect(info.compute_major >= 10, "device is sm_100 class: " + info.name);

    // ---- one-hot {3,-2} -> 13 on its channel (tests/cpu/test_cpu_beamformer.cpp:112-124)
    {
        const Dimensions d{1, 336, 32, 5};
        std::vector<Vec3> dirs;
        for (int b = 0; b < 5; ++b) dirs.push_back(direction_from_lm(static_cast<float>(b - 2) * 0.02F, 0.F));
        const auto w = weights_for(d, dirs);
        PackedVoltage v(voltage_sample_count(d), pack_complex_int4(0, 0));
        v[voltage_index(0, 17, 7, d)] = pack_complex_int4(3, -2);
        const auto I = cuda_beamform_packed_intensity(v, w, d);
        bool ok = true;
        for (std::size_t f = 0; f < 336; ++f)
            for (std::size_t b = 0; b < 5; ++b) ok &= std::abs(I[intensity_index(0, f, b, d)] - (f == 17 ? 13.F : 0.F)) < 1e-5F;
        expect(ok, "one-hot power 13");
        const auto It = cuda_beamform_packed_intensity(v, tile(w, d), d, nullptr, CudaBeamformerKernel::Tiled);
        expect(It == I, "Tiled equals Direct bit for bit");
    }

    // ---- random data: bit-exact against the reference float32 order
    {
        const Dimensions d{21, 336, 64, 40};
        std::vector<Vec3> dirs;
        for (int b = 0; b < 40; ++b) dirs.push_back(direction_from_lm(-0.4F + 0.02F * b, 0.1F));
        const auto w = weights_for(d, dirs);
        const auto v = random_voltage(d, 7);
        CudaBeamformerTimings t;
        const auto I = cuda_beamform_packed_intensity(v, w, d, &t);
        bool ok = true;
        for (std::size_t tt : {std::size_t{0}, std::size_t{20}})
            for (std::size_t f : {std::size_t{0}, std::size_t{200}, std::size_t{335}})
                for (std::size_t b = 0; b < 40; ++b) ok &= I[intensity_index(tt, f, b, d)] == cpu_power(v, w, d, tt, f, b);
        expect(ok && t.kernel_ms > 0.0, "per-spectrum output bit-exact vs reference order");

        // integrated 320 with a partial window (T = 700 -> 3 windows)
        const Dimensions di{700, 336, 64, 40};
        const auto vi = random_voltage(di, 8);
        const auto wi = weights_for(di, dirs);
        const auto integ = cuda_beamform_packed_integrated_intensity(vi, tile(wi, di), di, integration_direct);
        bool ok2 = integ.size() == 3 * 336 * 40;
        for (std::size_t b = 0; b < 40 && ok2; ++b) {
            volatile float s = 0.f;
            for (std::size_t tt = 640; tt < 700; ++tt) s = s + cpu_power(vi, wi, di, tt, 5, b);
            ok2 &= integ[(2 * 336 + 5) * 40 + b] == s;
        }
        expect(ok2, "integrated partial window bit-exact");

        // quantized pipeline equals quantizing the integrated output
        const auto q = cuda_beamform_packed_quantized_integrated_intensity(vi, tile(wi, di), di, integration_direct);
        expect(q.codes.size() == integ.size() && q.parameters.size() == 3 * 21 * 3, "quantized layout 3 x 21 x 3");

        // TensorSplit workspace: within 1e-3 + 1e-5|x| of the reference-order kernel
        CudaBeamformerWorkspace ws(di, CudaBeamformerKernel::TensorSplit, integration_direct);
        ws.upload_weights(wi, di);
        IntegratedIntensities out(integ.size());
        ws.run_integrated_pipeline(vi, out, di);
        bool ok3 = true;
        for (std::size_t i = 0; i < out.size(); ++i) ok3 &= std::abs(out[i] - integ[i]) <= 1e-3F + 1e-5F * std::abs(integ[i]);
        expect(ok3, "TensorSplit workspace within tolerance");
        expect(throws<std::invalid_argument>([&] { CudaBeamformerWorkspace x(di, CudaBeamformerKernel::TensorSplit, TemporalIntegrationConfig{40}); }),
               "TensorSplit rejects 40-spectrum integration");
        {
            // per-spectrum output on the tensor path (workspace without integration)
            CudaBeamformerWorkspace wps(di, CudaBeamformerKernel::TensorSplit);
            wps.upload_weights(wi, di);
            Intensities ps(di.n_time * di.n_freq * di.n_beams);
            wps.run_pipeline(vi, ps, di);
            bool okp = true;
            for (std::size_t tt : {std::size_t{0}, std::size_t{333}, std::size_t{699}})
                for (std::size_t f : {std::size_t{0}, std::size_t{111}, std::size_t{335}})
                    for (std::size_t b = 0; b < 40; ++b) {
                        const float r = cpu_power(vi, wi, di, tt, f, b);
                        okp &= std::abs(ps[intensity_index(tt, f, b, di)] - r) <= 1e-3F + 1e-5F * std::abs(r);
                    }
            expect(okp, "TensorSplit per-spectrum output within tolerance");
        }
        {
            // 10-spectrum windows (integration_after_upchan) on the tensor path
            const auto integ10 = cuda_beamform_packed_integrated_intensity(vi, tile(wi, di), di, integration_after_upchan);
            CudaBeamformerWorkspace w10(di, CudaBeamformerKernel::TensorSplit, integration_after_upchan);
            w10.upload_weights(wi, di);
            IntegratedIntensities o10(integ10.size());
            w10.run_integrated_pipeline(vi, o10, di);
            bool ok10 = o10.size() == 70 * 336 * 40;
            for (std::size_t i = 0; i < o10.size() && ok10; ++i) {
                ok10 &= std::abs(o10[i] - integ10[i]) <= 1e-3F + 1e-5F * std::abs(integ10[i]);
            }
            expect(ok10, "TensorSplit 10-spectrum integration within tolerance");
        }
        {
            // covariance form: same window sums, within the split kernel's bar
            CudaBeamformerWorkspace wc(di, CudaBeamformerKernel::TensorCovariance, integration_direct);
            wc.upload_weights(wi, di);
            IntegratedIntensities oc(integ.size());
            wc.run_integrated_pipeline(vi, oc, di);
            bool okc = true;
            for (std::size_t i = 0; i < oc.size(); ++i) okc &= std::abs(oc[i] - integ[i]) <= 1e-3F + 1e-5F * std::abs(integ[i]);
            expect(okc, "TensorCovariance workspace within tolerance");
            expect(throws<std::invalid_argument>([&] { CudaBeamformerWorkspace x(di, CudaBeamformerKernel::TensorCovariance); }),
                   "TensorCovariance needs integration");
            expect(throws<std::invalid_argument>([&] { CudaBeamformerWorkspace x(di, CudaBeamformerKernel::TensorCovariance, integration_after_upchan); }),
                   "TensorCovariance rejects 10-spectrum integration");
        }
        {
            // checked form: the covariance form with split-kernel recomputation, and
            // the split kernel alone for 10-spectrum windows
            CudaBeamformerWorkspace wk(di, CudaBeamformerKernel::TensorChecked, integration_direct);
            wk.upload_weights(wi, di);
            IntegratedIntensities ok_(integ.size());
            wk.run_integrated_pipeline(vi, ok_, di);
            bool okk = true;
            for (std::size_t i = 0; i < ok_.size(); ++i) okk &= std::abs(ok_[i] - integ[i]) <= 1e-3F + 1e-5F * std::abs(integ[i]);
            expect(okk, "TensorChecked workspace within tolerance");
            CudaBeamformerWorkspace wk10(di, CudaBeamformerKernel::TensorChecked, integration_after_upchan);
            wk10.upload_weights(wi, di);
            const auto integ10 = cuda_beamform_packed_integrated_intensity(vi, tile(wi, di), di, integration_after_upchan);
            IntegratedIntensities o10(integ10.size());
            wk10.run_integrated_pipeline(vi, o10, di);
            bool ok10 = true;
            for (std::size_t i = 0; i < o10.size(); ++i) ok10 &= std::abs(o10[i] - integ10[i]) <= 1e-3F + 1e-5F * std::abs(integ10[i]);
            expect(ok10, "TensorChecked 10-spectrum integration within tolerance");
            expect(throws<std::invalid_argument>([&] { CudaBeamformerWorkspace x(di, CudaBeamformerKernel::TensorChecked); }),
                   "TensorChecked needs integration");
            expect(throws<std::invalid_argument>([&] {
                       launch_packed_integrated_beamformer(CudaBeamformerKernel::TensorChecked, nullptr, nullptr, nullptr,
                                                           nullptr, di, integration_direct);
                   }),
                   "TensorChecked stage call needs its workspace entry point");
        }
        {
            // chunked host pipeline: bit-identical to the one-launch TensorSplit workspace
            CudaBeamformerWorkspace wq(di, CudaBeamformerKernel::TensorSplit, integration_direct,
                                       CudaBeamformerOutput::QuantizedInt8);
            wq.upload_weights(wi, di);
            QuantizedIntegratedOutput qw{QuantizedIntensities(integ.size()),
                                         std::vector<Int8QuantizationParameters>(3 * 21 * 3)};
            wq.run_quantized_integrated_pipeline(vi, qw, di);
            CudaChunkedGridPipeline pipe(di, integration_direct, 1, 640);
            expect(pipe.chunk_spectra() == 640, "chunked pipeline keeps a 640-spectrum chunk");
            expect(throws<std::logic_error>([&] { IntegratedIntensities x; pipe.run(vi, &x, nullptr); }),
                   "chunked pipeline before weights is a logic_error");
            pipe.upload_weights(wi);
            IntegratedIntensities pi;
            QuantizedIntegratedOutput pq;
            const double ms = pipe.run(vi, &pi, &pq);
            bool same_p = pq.parameters.size() == qw.parameters.size();
            for (std::size_t i = 0; i < pq.parameters.size() && same_p; ++i) {
                same_p &= pq.parameters[i].offset == qw.parameters[i].offset &&
                          pq.parameters[i].scale == qw.parameters[i].scale;
            }
            expect(ms > 0.0 && pi == out && pq.codes == qw.codes && same_p,
                   "chunked pipeline equals one TensorSplit launch bit for bit");
            expect(throws<std::invalid_argument>([&] { CudaChunkedGridPipeline x(di, integration_direct, 1, 600); }),
                   "chunked pipeline rejects a chunk off the 640-spectrum grid");
        }

        // device frame path: voltage and weights already on the device
        std::uint8_t* dv = nullptr;
        ComplexFloat* dw = nullptr;
        float* dout = nullptr;
        cudaMalloc(&dv, vi.size());
        cudaMalloc(&dw, tiled_weight_bytes(di));
        cudaMalloc(&dout, integ.size() * 4);
        cudaMemcpy(dv, vi.data(), vi.size(), cudaMemcpyHostToDevice);
        const auto tw = tile(wi, di);
        cudaMemcpy(dw, tw.data(), tiled_weight_bytes(di), cudaMemcpyHostToDevice);
        const auto shard = default_shard_descriptors()[1];
        CudaBeamformerWorkspace wf(di, CudaBeamformerKernel::Tiled, integration_direct);
        auto vf = make_packed_voltage_frame_view(dv, di, 42, shard);
        auto wfv = make_tiled_weights_frame_view(dw, di, 42, shard);
        const Dimensions od{3, 336, 64, 40};
        auto of = make_intensity_frame_view(dout, od, 42, shard);
        wf.run_device_frame(vf, wfv, of);
        std::vector<float> back(integ.size());
        cudaMemcpy(back.data(), dout, back.size() * 4, cudaMemcpyDeviceToHost);
        expect(back == integ, "device frame output equals host pipeline");
        auto bad = make_intensity_frame_view(dout, od, 43, shard);
        expect(throws<std::invalid_argument>([&] { wf.run_device_frame(vf, wfv, bad); }), "frame id mismatch rejected");
        cudaFree(dv);
        cudaFree(dw);
        cudaFree(dout);
    }

    // ---- tracker: constant trajectory equals the one-beam grid (tests/cpu/test_beam_tracker.cpp:121-139)
    {
        const Dimensions d{96, 336, 64, 1};
        TrackerConfig cfg;
        cfg.trajectory.direction_start = direction_from_lm(0.05F, -0.02F);
        cfg.integration_spectra = 32;
        const auto v = random_voltage(d, 11);
        const auto I = cuda_beam_tracker_v5(v, d, cfg);
        const auto w = weights_for(d, {cfg.trajectory.direction_start});
        bool ok = I.size() == 96 * 336;
        for (std::size_t t = 0; t < 96 && ok; t += 7)
            for (std::size_t f = 0; f < 336; f += 5) {
                const float r = cpu_power(v, w, d, t, f, 0);
                ok &= std::abs(I[t * 336 + f] - r) <= 1e-3F + 1e-5F * std::abs(r);
            }
        expect(ok, "tracker (stationary) within tolerance of the one-beam grid");
        expect(throws<std::invalid_argument>([&] { cuda_beam_tracker_v5(v, Dimensions{96, 336, 64, 2}, cfg); }),
               "tracker requires n_beams == 1");

        // batched stream, CUDA graph on, two batches
        V5ExecutionConfig vc;
        vc.enable_cuda_graph = true;
        const Dimensions wdim{32, 336, 64, 1};
        BatchedTrackerStreamV5 s(wdim, cfg, 3, vc);
        std::vector<float> out(s.batch_output_floats());
        s.process_batch(0, v.data(), out.data());
        expect(out == I && s.last_kernel_time_ms() > 0.f, "batched stream equals one-shot tracker");
        s.process_batch(0, v.data(), out.data());
        expect(out == I, "graph replay repeats the result");
    }

    {
        // served mode: one grid and one tracker job give the same bytes alone and in a mix
        ServedConfig sc;
        sc.hbm_budget_bytes = 2'000'000'000ULL;
        sc.pool_spectra = 320 * 8;
        std::vector<float> freq(2 * 336);
        for (std::size_t f = 0; f < freq.size(); ++f) freq[f] = 400e6F + static_cast<float>(f) * (400e6F / 671.F);
        std::vector<Vec3> pos(64);
        for (std::size_t a = 0; a < 64; ++a) pos[a] = {static_cast<float>(a % 32) * 0.1875F, static_cast<float>(a / 32) * 0.1875F, 0.F};
        ServedJob g;
        g.kind = ServedJobKind::Grid;
        g.n_ant = 64;
        g.n_shards = 2;
        g.n_beams = 8;
        g.n_spectra = 640;
        g.integration_spectra = 10;
        g.pool_offset = 320;
        g.positions = pos;
        g.frequencies_hz = freq;
        for (std::size_t b = 0; b < 8; ++b) g.directions.push_back(direction_from_lm(0.03F * static_cast<float>(b), 0.F));
        ServedJob t = g;
        t.kind = ServedJobKind::Tracker;
        t.n_beams = 3;
        t.integration_spectra = 320;
        t.directions.clear();
        t.trajectories = {{0.1F, 0.F, 1e-6F, 0.F}, {-0.1F, 0.05F, 0.F, 0.F}, {0.F, 0.F, 0.F, -1e-6F}};
        auto run = [&](std::vector<ServedJob> jobs, std::size_t pick) {
            ServedBeamformer srv(sc);
            std::vector<std::uint64_t> ids;
            for (const auto& j : jobs) ids.push_back(srv.submit(j));
            while (srv.step() > 0) {
            }
            srv.synchronize();
            const ServedResult r = srv.result(ids[pick]);
            const ServedJob& j = jobs[pick];
            const std::size_t n = j.kind == ServedJobKind::Grid ? j.n_shards * r.n_windows * 336 * j.n_beams
                                                                : r.n_windows * j.n_shards * 336 * j.n_beams;
            std::vector<float> host(n);
            cudaMemcpy(host.data(), r.integrated, n * sizeof(float), cudaMemcpyDeviceToHost);
            return host;
        };
        const auto ga = run({g}, 0);
        const auto ta = run({t}, 0);
        const auto gm = run({t, g, t}, 1);
        const auto tm = run({g, t}, 1);
        bool positive = !ga.empty();
        for (float x : ga) positive &= std::isfinite(x) && x > 0.F;
        expect(positive && ga.size() == 2 * 64 * 336 * 8, "served grid job produces finite powers");
        expect(ga == gm && ta == tm, "served jobs are bit-identical alone and in a mix");
        ServedBeamformer srv(sc);
        const auto pool64 = srv.pool(64);
        expect(pool64.data != nullptr && pool64.spectra == sc.pool_spectra &&
                   pool64.channels == static_cast<std::uint64_t>(sc.shard_channels) * sc.max_shards,
               "served pool geometry");
        expect(throws<std::invalid_argument>([&] { srv.pool(48); }), "served pool needs 32 or 64 antennas");
        ServedJob big = g;
        big.n_spectra = 320 * 100000;
        expect(throws<std::length_error>([&] { srv.submit(big); }), "oversize served job is a length_error");
        ServedJob bad = g;
        bad.n_spectra = 100;
        expect(throws<std::invalid_argument>([&] { srv.submit(bad); }), "served job length must be whole windows");
    }

    std::printf("%s (%d failures)\n", failures == 0 ? "ALL OK" : "FAILED", failures);
    return failures == 0 ? 0 : 1;
}
