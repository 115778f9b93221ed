// served.hpp -- served, continuously batched beamforming and tracking.
//
// No reference counterpart: the reference runs one job per call.  A
// ServedBeamformer admits grid and tracker jobs as they arrive against an
// HBM budget (and optionally a bound on the device time of a window), keeps
// their state on the device, and runs one 320-spectrum window of every live
// job per step as one CUDA-graph replay (bf_serve_* in bf_b200.h).  Jobs
// give the same results alone and in a mix.  Errors throw the same exception
// types as the rest of this API; a job that can never fit the budget throws
// std::length_error.
#pragma once

#include "beamformer/geometry.hpp"

#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

struct bf_server;

namespace beamformer {

struct ServedConfig {
    std::size_t hbm_budget_bytes = 120'000'000'000ULL;
    std::uint32_t max_jobs = 512;
    std::uint32_t window_spectra = 320;
    std::size_t pool_spectra = 20480;     // device voltage pool rows per antenna count
    std::uint32_t shard_channels = 336;
    std::uint32_t max_shards = 4;
    std::uint64_t pool_seed = 1;
    float pool_sigma = 2.0F;              // Gaussian-like int4 noise of the pools
    float window_budget_us = 0.0F;        // 0: admission by memory and slots only
    std::uint32_t windows_per_step = 1;   // windows per job per step (throughput setting)
};

enum class ServedJobKind { Grid = 0, Tracker = 1 };
enum class ServedJobState { Queued = 0, Live = 1, Running = 2, Done = 3, Cancelled = 4, Unknown = 5 };

struct ServedJob {
    ServedJobKind kind = ServedJobKind::Grid;
    std::size_t n_ant = 64;
    std::size_t n_shards = 1;
    std::size_t n_beams = 1;              // grid beams or tracker sources
    std::size_t n_spectra = 320;          // a multiple of the window
    std::size_t integration_spectra = 320;
    std::size_t pool_offset = 0;
    std::vector<Vec3> positions;          // [n_ant] metres
    std::vector<float> frequencies_hz;    // [n_shards * shard_channels]
    std::vector<Vec3> directions;         // grid: [n_beams] unit vectors
    std::vector<std::array<float, 4>> trajectories;  // tracker: [n_beams] l0, m0, dl, dm per spectrum
    bool quantize = true;                 // grid: int8 chunk codes as well
};

// Device pointers of a finished job, valid until release().
struct ServedResult {
    const float* integrated = nullptr;    // grid [shard][W][F][B]; tracker [W][F_total][sources]
    const std::int8_t* codes = nullptr;   // grid, quantized: [shard][W][F][B]
    const float* params = nullptr;        // [shard][W][ceil(F/16)][ceil(B/16)][2]
    std::size_t n_windows = 0;
};

struct ServedStats {
    std::uint64_t steps = 0, job_windows = 0, jobs_done = 0, live_jobs = 0, queued_jobs = 0;
    std::uint64_t arena_bytes_peak = 0, graph_captures = 0;
    double beam_samples = 0.0, window_ms_p50 = 0.0, window_ms_p99 = 0.0;
};

class ServedBeamformer {
public:
    explicit ServedBeamformer(const ServedConfig& config = ServedConfig{});
    ~ServedBeamformer();
    ServedBeamformer(const ServedBeamformer&) = delete;
    ServedBeamformer& operator=(const ServedBeamformer&) = delete;

    std::uint64_t submit(const ServedJob& job);
    std::size_t step();                   // returns the number of live jobs it ran
    ServedJobState state(std::uint64_t job_id);
    std::vector<std::uint64_t> take_done();
    ServedResult result(std::uint64_t job_id);
    void cancel(std::uint64_t job_id);
    void release(std::uint64_t job_id);
    // Self-contained image of a job (description, windows served, their
    // results); waits for the job's launched windows.  restore() queues it in
    // a server with the same window, shard and pool settings, where it
    // resumes at its next window with results equal to an uninterrupted run.
    std::vector<std::uint8_t> checkpoint(std::uint64_t job_id);
    std::uint64_t restore(const std::vector<std::uint8_t>& image);
    void synchronize();
    ServedStats stats();
    std::vector<float> window_times_ms();
    void* stream();                       // cudaStream_t of the server
    // Ingest hook: the device pool that jobs of n_ant antennas read,
    // [spectra][channels][n_ant] packed bytes.  A capture stage writes rows
    // there in stream order on stream() before the step that reads them.
    struct Pool {
        std::uint8_t* data = nullptr;
        std::uint64_t spectra = 0, channels = 0;
    };
    Pool pool(std::uint64_t n_ant);

private:
    bf_server* server_ = nullptr;
};

}  // namespace beamformer
