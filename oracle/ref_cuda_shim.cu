// ref_cuda_shim.cu -- extern "C" entry points into the reference's own CUDA
// kernels, for timing them beside the B200 kernels on the same GPU.
//
// TEST / MEASUREMENT INFRASTRUCTURE ONLY.  oracle/build.py compiles this file
// with nvcc (sm_100a) together with the reference's CUDA sources
// (src/cuda_beamformer.cu, src/cuda_quantize_int8.cu,
// src/cuda_beam_tracker_v5.cu) and its CPU sources, read where they lie in
// the reference checkout, into oracle/_ref/libbfref_cuda.so.  bench.py loads it
// for its "reference_gpu" lines; nothing in the product links it.  Every
// function returns 0 on success or a nonzero code with the exception text
// available from refgpu_last_error().
#include <beamformer/beam_tracker.hpp>
#include <beamformer/cuda_beam_tracker_v5.hpp>
#include <beamformer/cuda_stage_api.hpp>
#include <beamformer/geometry.hpp>

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

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
}  // namespace

extern "C" {

const char* refgpu_last_error() { return g_err.c_str(); }

// launch_packed_integrated_beamformer (src/cuda_beamformer.cu:488-543):
// kernel 0 = Direct, 1 = Tiled; weights canonical [B][F][A] (Direct) or tiled
// [F][ceil(B/32)][A][32] (Tiled) complex64, all device pointers.
int refgpu_grid_integrated(int kernel, void* stream, const uint8_t* v, const void* w, float* out,
                           uint64_t T, uint64_t F, uint64_t A, uint64_t B, uint64_t S) {
    return guarded([&] {
        const Dimensions d{T, F, A, B};
        TemporalIntegrationConfig ti;
        ti.integration_spectra = S;
        launch_packed_integrated_beamformer(kernel == 0 ? CudaBeamformerKernel::Direct : CudaBeamformerKernel::Tiled,
                                            static_cast<cudaStream_t>(stream), v,
                                            static_cast<const ComplexFloat*>(w), out, d, ti);
    });
}

// launch_quantize_integrated_intensity (src/cuda_quantize_int8.cu:132-147) on
// integrated [W][F][B]; params as {offset, scale} pairs.
int refgpu_quantize(void* stream, const float* in, int8_t* codes, void* params, uint64_t W, uint64_t F,
                    uint64_t A, uint64_t B) {
    return guarded([&] {
        const Dimensions d{W, F, A, B};
        launch_quantize_integrated_intensity(static_cast<cudaStream_t>(stream), in, codes,
                                             static_cast<Int8QuantizationParameters*>(params), d);
    });
}

// cuda_beam_tracker_v5_device_resident (src/cuda_beam_tracker_v5.cu:383-420):
// per-spectrum [T][F][1] float32 output on the reference's default geometry.
int refgpu_tracker_v5(const uint8_t* v, float* out, uint64_t T, uint64_t F, uint64_t A, float l0, float m0,
                      float rl, float rm, uint64_t S, uint64_t chunk, uint64_t unroll, void* stream) {
    return guarded([&] {
        const Dimensions d{T, F, A, 1};
        TrackerConfig cfg;
        cfg.trajectory.direction_start = direction_from_lm(l0, m0);
        cfg.trajectory.direction_rate_per_sample = {rl, rm};
        cfg.integration_spectra = S;
        V5ExecutionConfig ex;
        ex.time_chunk_size = chunk;
        ex.time_unroll = unroll;
        cuda_beam_tracker_v5_device_resident(v, out, d, cfg, ex, stream);
    });
}

}  // extern "C"
