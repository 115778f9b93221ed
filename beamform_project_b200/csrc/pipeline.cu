// pipeline.cu -- the tensor-core grid beamformer fed from host memory.
//
// The reference's host pipeline (CudaBeamformerWorkspace::
// run_quantized_integrated_pipeline, src/cuda_beamformer.cu) copies the
// whole voltage block to the device, runs the kernels, and copies the
// products back, one phase after the other.  On a B200 the kernels of a
// full-band block take a tenth of its host-to-device copy over PCIe, so this
// pipeline cuts the block into time chunks of whole integration windows and
// overlaps three streams:
//
//   copy-in   chunk c + 1 host -> device    (waits until chunk c - 1's kernels
//                                            have finished reading its slot)
//   compute   chunk c: tensor-core grid + int8 chunk quantizer
//                                           (waits for its voltage, and until
//                                            chunk c - 2's products have left
//                                            its output slot)
//   copy-out  chunk c - 1 device -> host    (waits for its kernels)
//
// Two voltage slots and two product slots, so the device holds
// 2 x (chunk voltage + chunk products) whatever the block length.  A chunk is a
// multiple of lcm(128, S) spectra, so its tiles and windows start where
// they would in a single launch and the products are bit-identical to
// bf_grid_tensor_integrated over the whole block.  Copies from pinned host
// memory run at PCIe rate while the kernels run; pageable memory works but
// the driver stages it.
#include "bf_internal.cuh"

#include <algorithm>
#include <cstdint>
#include <string>

namespace {

using namespace bf;

constexpr uint64_t kTileSpectra = 128;           // one tensor-core tile of spectra
constexpr uint64_t kAutoChunkBytes = 64ull << 20;  // voltage per chunk when chunk_spectra is 0

uint64_t gcd_u64(uint64_t a, uint64_t b) {
    while (b != 0) {
        const uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

uint64_t chunk_unit(uint64_t spectra) { return spectra / gcd_u64(spectra, kTileSpectra) * kTileSpectra; }

uint64_t quant_pairs_per_window(const bf_dims& d) { return ((d.n_freq + 15) / 16) * ((d.n_beams + 15) / 16); }

}  // namespace

struct bf_grid_pipeline {
    int device = 0;
    bf_dims dims{};            // the whole block of one shard
    uint64_t spectra = 0;      // integration length
    uint64_t n_shards = 0;
    uint64_t chunk = 0;        // spectra per chunk (multiple of lcm(128, spectra))
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    cudaEvent_t h2d_done[2] = {}, comp_done[2] = {}, d2h_done[2] = {};
    cudaEvent_t start = nullptr, end = nullptr;
    uint8_t* volt[2] = {};
    float* integ[2] = {};
    int8_t* codes[2] = {};
    float* params[2] = {};
    void* split = nullptr;     // split operand, or the checked form's (covariance image + split image)
    bool checked = false;      // run the checked covariance form instead of the split kernel
    void* workspace = nullptr; // the checked form's fallback list
    bool weights_ready = false;

    bf_status init() {
        BF_RETURN_IF(cuda_status(cudaGetDevice(&device), "cudaGetDevice"));
        BF_RETURN_IF(cuda_status(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking), "cudaStreamCreate"));
        BF_RETURN_IF(cuda_status(cudaStreamCreateWithFlags(&comp, cudaStreamNonBlocking), "cudaStreamCreate"));
        BF_RETURN_IF(cuda_status(cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking), "cudaStreamCreate"));
        for (int i = 0; i < 2; ++i) {
            BF_RETURN_IF(cuda_status(cudaEventCreateWithFlags(&h2d_done[i], cudaEventDisableTiming), "cudaEventCreate"));
            BF_RETURN_IF(cuda_status(cudaEventCreateWithFlags(&comp_done[i], cudaEventDisableTiming), "cudaEventCreate"));
            BF_RETURN_IF(cuda_status(cudaEventCreateWithFlags(&d2h_done[i], cudaEventDisableTiming), "cudaEventCreate"));
        }
        BF_RETURN_IF(cuda_status(cudaEventCreate(&start), "cudaEventCreate"));
        BF_RETURN_IF(cuda_status(cudaEventCreate(&end), "cudaEventCreate"));
        const uint64_t t = std::min(chunk, dims.n_time);
        const uint64_t w = window_count(t, spectra);
        const uint64_t vbytes = n_shards * t * dims.n_freq * dims.n_ant;
        const uint64_t n_out = n_shards * w * dims.n_freq * dims.n_beams;
        const uint64_t n_par = 2 * n_shards * w * quant_pairs_per_window(dims);
        for (int i = 0; i < 2; ++i) {
            BF_RETURN_IF(cuda_status(cudaMalloc(&volt[i], vbytes), "cudaMalloc chunk voltage"));
            BF_RETURN_IF(cuda_status(cudaMalloc(&integ[i], n_out * sizeof(float)), "cudaMalloc chunk output"));
            BF_RETURN_IF(cuda_status(cudaMalloc(&codes[i], n_out), "cudaMalloc chunk codes"));
            BF_RETURN_IF(cuda_status(cudaMalloc(&params[i], n_par * sizeof(float)), "cudaMalloc chunk parameters"));
        }
        if (checked) {
            const bf_dims dc{t, dims.n_freq, dims.n_ant, dims.n_beams};
            const uint64_t ws = auto_workspace_bytes(dc, spectra, n_shards);
            if (ws > 0) BF_RETURN_IF(cuda_status(cudaMalloc(&workspace, ws), "cudaMalloc fallback list"));
            return cuda_status(cudaMalloc(&split, auto_weight_bytes(dims, n_shards)), "cudaMalloc weights");
        }
        return cuda_status(cudaMalloc(&split, split_weight_bytes(dims, n_shards)), "cudaMalloc split weights");
    }

    // Waits for everything issued on the three streams (a run that failed part
    // way may have copies in flight).
    void drain() {
        if (in) cudaStreamSynchronize(in);
        if (comp) cudaStreamSynchronize(comp);
        if (out) cudaStreamSynchronize(out);
    }

    ~bf_grid_pipeline() {
        drain();
        for (int i = 0; i < 2; ++i) {
            cudaFree(volt[i]);
            cudaFree(integ[i]);
            cudaFree(codes[i]);
            cudaFree(params[i]);
            if (h2d_done[i]) cudaEventDestroy(h2d_done[i]);
            if (comp_done[i]) cudaEventDestroy(comp_done[i]);
            if (d2h_done[i]) cudaEventDestroy(d2h_done[i]);
        }
        cudaFree(split);
        cudaFree(workspace);
        if (start) cudaEventDestroy(start);
        if (end) cudaEventDestroy(end);
        if (in) cudaStreamDestroy(in);
        if (comp) cudaStreamDestroy(comp);
        if (out) cudaStreamDestroy(out);
    }

    // Issues every chunk on the three streams; returns after the last copy-out.
    bf_status run(const uint8_t* host_v, float* host_i, int8_t* host_c, float* host_p, float* elapsed_ms) {
        const uint64_t F = dims.n_freq, A = dims.n_ant, B = dims.n_beams;
        const uint64_t T = dims.n_time, W = window_count(T, spectra);
        const uint64_t qpw = quant_pairs_per_window(dims);
        const uint64_t n_chunks = (T + chunk - 1) / chunk;
        const bool quantize = host_c != nullptr;
        BF_RETURN_IF(cuda_status(cudaEventRecord(start, in), "cudaEventRecord"));
        BF_RETURN_IF(cuda_status(cudaStreamWaitEvent(comp, start, 0), "cudaStreamWaitEvent"));
        BF_RETURN_IF(cuda_status(cudaStreamWaitEvent(out, start, 0), "cudaStreamWaitEvent"));
        for (uint64_t c = 0; c < n_chunks; ++c) {
            const int s = static_cast<int>(c & 1);
            const uint64_t t0 = c * chunk, tc = std::min(chunk, T - t0);
            const uint64_t w0 = t0 / spectra, wc = window_count(tc, spectra);
            // copy-in: this slot was last read by chunk c - 2's kernels
            if (c >= 2) BF_RETURN_IF(cuda_status(cudaStreamWaitEvent(in, comp_done[s], 0), "cudaStreamWaitEvent"));
            for (uint64_t sh = 0; sh < n_shards; ++sh) {
                BF_RETURN_IF(cuda_status(cudaMemcpyAsync(volt[s] + sh * tc * F * A, host_v + (sh * T + t0) * F * A,
                                                         tc * F * A, cudaMemcpyHostToDevice, in),
                                         "cudaMemcpyAsync voltage chunk"));
            }
            BF_RETURN_IF(cuda_status(cudaEventRecord(h2d_done[s], in), "cudaEventRecord"));
            // compute: voltage present, and chunk c - 2's products copied out of this slot
            BF_RETURN_IF(cuda_status(cudaStreamWaitEvent(comp, h2d_done[s], 0), "cudaStreamWaitEvent"));
            if (c >= 2) BF_RETURN_IF(cuda_status(cudaStreamWaitEvent(comp, d2h_done[s], 0), "cudaStreamWaitEvent"));
            const bf_dims dc{tc, F, A, B};
            if (checked) {
                BF_RETURN_IF(launch_grid_auto(comp, volt[s], split, integ[s], quantize ? codes[s] : nullptr,
                                              quantize ? params[s] : nullptr, workspace, dc, spectra, n_shards));
            } else {
                BF_RETURN_IF(launch_grid_tensor(comp, volt[s], split, integ[s], quantize ? codes[s] : nullptr,
                                                quantize ? params[s] : nullptr, dc, spectra, n_shards, nullptr));
            }
            BF_RETURN_IF(cuda_status(cudaEventRecord(comp_done[s], comp), "cudaEventRecord"));
            // copy-out: [shard][window] rows of this chunk into the block's place
            BF_RETURN_IF(cuda_status(cudaStreamWaitEvent(out, comp_done[s], 0), "cudaStreamWaitEvent"));
            for (uint64_t sh = 0; sh < n_shards; ++sh) {
                const uint64_t src = sh * wc * F * B, dst = (sh * W + w0) * F * B;
                if (host_i != nullptr) {
                    BF_RETURN_IF(cuda_status(cudaMemcpyAsync(host_i + dst, integ[s] + src, wc * F * B * sizeof(float),
                                                             cudaMemcpyDeviceToHost, out),
                                             "cudaMemcpyAsync integrated chunk"));
                }
                if (quantize) {
                    BF_RETURN_IF(cuda_status(cudaMemcpyAsync(host_c + dst, codes[s] + src, wc * F * B,
                                                             cudaMemcpyDeviceToHost, out),
                                             "cudaMemcpyAsync code chunk"));
                    BF_RETURN_IF(cuda_status(
                        cudaMemcpyAsync(host_p + 2 * (sh * W + w0) * qpw, params[s] + 2 * sh * wc * qpw,
                                        2 * wc * qpw * sizeof(float), cudaMemcpyDeviceToHost, out),
                        "cudaMemcpyAsync parameter chunk"));
                }
            }
            BF_RETURN_IF(cuda_status(cudaEventRecord(d2h_done[s], out), "cudaEventRecord"));
        }
        BF_RETURN_IF(cuda_status(cudaEventRecord(end, out), "cudaEventRecord"));
        BF_RETURN_IF(cuda_status(cudaEventSynchronize(end), "cudaEventSynchronize"));
        uint32_t code = 0;
        BF_RETURN_IF(take_tc_error(&code));
        if (code != 0) {
            return set_error(BF_ERR_TIMEOUT, "a bounded wait of the tensor-core grid kernel ran out (code " +
                                                 std::to_string(code) + ")");
        }
        if (elapsed_ms != nullptr) {
            BF_RETURN_IF(cuda_status(cudaEventElapsedTime(elapsed_ms, start, end), "cudaEventElapsedTime"));
        }
        return BF_OK;
    }
};

namespace {

bf_status check_request(const bf_dims* dims, uint64_t spectra, uint64_t n_shards, uint64_t chunk_spectra) {
    BF_RETURN_IF(validate_dims(dims));
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (spectra == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    if (spectra > 32 && spectra % 32 != 0) {
        return set_error(BF_ERR_UNSUPPORTED,
                         "the tensor-core kernel needs integration_spectra below 32 or a multiple of 32");
    }
    if (dims->n_time >= (1ull << 31) || n_shards > 1024 || spectra >= (1ull << 30)) {
        return set_error(BF_ERR_OVERFLOW, "CUDA tensor-core grid exceeds the supported size");
    }
    const uint64_t unit = chunk_unit(spectra);
    if (chunk_spectra % unit != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "chunk_spectra must be a multiple of lcm(128, integration_spectra) = " +
                                                      std::to_string(unit));
    }
    return BF_OK;
}

uint64_t pick_chunk(const bf_dims& d, uint64_t spectra, uint64_t n_shards, uint64_t chunk_spectra) {
    const uint64_t unit = chunk_unit(spectra);
    uint64_t chunk = chunk_spectra;
    if (chunk == 0) {
        const uint64_t per_spectrum = n_shards * d.n_freq * d.n_ant;
        chunk = std::max<uint64_t>(unit, kAutoChunkBytes / per_spectrum / unit * unit);
    }
    // never more than the block, rounded up to the unit
    return std::min(chunk, (d.n_time + unit - 1) / unit * unit);
}

}  // namespace

extern "C" {

BF_API uint64_t bf_grid_pipeline_chunk_spectra(const bf_dims* dims, uint64_t integration_spectra,
                                               uint64_t n_shards, uint64_t chunk_spectra) {
    if (check_request(dims, integration_spectra, n_shards, chunk_spectra) != BF_OK) return 0;
    return pick_chunk(*dims, integration_spectra, n_shards, chunk_spectra);
}

static bf_status create_pipeline(const bf_dims* dims, uint64_t integration_spectra, uint64_t n_shards,
                                 uint64_t chunk_spectra, bool checked, bf_grid_pipeline** pipeline) {
    clear_error();
    if (pipeline == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "pipeline must not be null");
    *pipeline = nullptr;
    BF_RETURN_IF(check_request(dims, integration_spectra, n_shards, chunk_spectra));
    auto* p = new bf_grid_pipeline();
    p->checked = checked;
    p->dims = *dims;
    p->spectra = integration_spectra;
    p->n_shards = n_shards;
    p->chunk = pick_chunk(*dims, integration_spectra, n_shards, chunk_spectra);
    const bf_status st = p->init();
    if (st != BF_OK) {
        delete p;
        return st;
    }
    *pipeline = p;
    return BF_OK;
}

BF_API bf_status bf_grid_pipeline_create(const bf_dims* dims, uint64_t integration_spectra, uint64_t n_shards,
                                         uint64_t chunk_spectra, bf_grid_pipeline** pipeline) {
    return create_pipeline(dims, integration_spectra, n_shards, chunk_spectra, false, pipeline);
}

BF_API bf_status bf_grid_pipeline_create_checked(const bf_dims* dims, uint64_t integration_spectra,
                                                 uint64_t n_shards, uint64_t chunk_spectra,
                                                 bf_grid_pipeline** pipeline) {
    return create_pipeline(dims, integration_spectra, n_shards, chunk_spectra, true, pipeline);
}

BF_API bf_status bf_grid_pipeline_upload_weights(bf_grid_pipeline* p, const float* host_weights) {
    clear_error();
    if (p == nullptr || host_weights == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "pipeline and host_weights must not be null");
    }
    const uint64_t n = p->n_shards * p->dims.n_beams * p->dims.n_freq * p->dims.n_ant * 2;
    float* canon = nullptr;
    BF_RETURN_IF(cuda_status(cudaMalloc(&canon, n * sizeof(float)), "cudaMalloc weights"));
    bf_status st = cuda_status(cudaMemcpyAsync(canon, host_weights, n * sizeof(float), cudaMemcpyHostToDevice, p->comp),
                               "cudaMemcpyAsync weights");
    if (st == BF_OK) {
        st = p->checked ? launch_prepare_auto(p->comp, canon, p->split, p->dims, p->n_shards)
                        : launch_prepare_split(p->comp, canon, p->split, p->dims, p->n_shards);
    }
    const bf_status sync = cuda_status(cudaStreamSynchronize(p->comp), "cudaStreamSynchronize");
    cudaFree(canon);
    if (st == BF_OK) st = sync;
    p->weights_ready = st == BF_OK;
    return st;
}

BF_API bf_status bf_grid_pipeline_run(bf_grid_pipeline* p, const uint8_t* host_voltage, float* host_integrated,
                                      int8_t* host_codes, float* host_params, float* elapsed_ms) {
    clear_error();
    if (p == nullptr || host_voltage == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "pipeline and host_voltage must not be null");
    }
    if ((host_codes == nullptr) != (host_params == nullptr)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "host_codes and host_params must both be given or both be null");
    }
    if (host_integrated == nullptr && host_codes == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "no output requested");
    }
    if (!p->weights_ready) return set_error(BF_ERR_LOGIC, "weights have not been uploaded for these dimensions");
    int dev = 0;
    BF_RETURN_IF(cuda_status(cudaGetDevice(&dev), "cudaGetDevice"));
    if (dev != p->device) return set_error(BF_ERR_LOGIC, "the pipeline belongs to another device");
    const bf_status st = p->run(host_voltage, host_integrated, host_codes, host_params, elapsed_ms);
    if (st != BF_OK) p->drain();  // no copy may touch the caller's buffers after an error return
    return st;
}

BF_API bf_status bf_grid_pipeline_destroy(bf_grid_pipeline* p) {
    clear_error();
    delete p;
    return BF_OK;
}

}  // extern "C"
