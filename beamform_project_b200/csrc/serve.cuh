// serve.cuh -- device job tables of the served batch (serve.cpp drives them;
// serve_kernels.cu and grid_tc.cu execute them).
//
// A served launch processes one window of every live job of one kernel class.
// Its table sits in device memory at a fixed address captured in the window's
// CUDA graph: a header (unit count, job count) and the job entries sorted by
// their first unit.  The host rewrites the table (one stream-ordered copy)
// before each replay, so the graph never changes while the live set does.
#pragma once

#include "bf_internal.cuh"

namespace bf {

struct TableHeader {
    long long n_units;
    int n_jobs;
    int pad;
};

// Streaming tracker job: windows of `spectra` samples, one steering vector
// per (window, source) from a linear (l, m) trajectory evaluated at the
// window's first sample.
struct TrJob {
    const float* pos;        // [A][3] metres
    const double* kw;        // [F] wave numbers (rad/m)
    const float* traj;       // [n_src][4]: l0, m0, dl, dm per spectrum
    float* integrated;       // [n_windows][F][n_src]
    long long unit_begin;
    long long t0;            // pool row of this launch's first spectrum
    int n_freq, n_src, spectra;
    int w0;                  // global index of this launch's first window
    int n_win;               // windows in this launch
    int src_groups;          // ceil(n_src / 8): sources per unit are 8
    int fgroups;             // ceil(n_freq / 8): channels per unit are 8
    int pad;
};

// int8 chunk quantization of the windows a grid launch just wrote.
struct QJob {
    const float* integrated;  // [shard][n_windows][F][B]
    int8_t* codes;            // same layout
    float2* params;           // [shard][n_windows][ftiles][btiles]
    long long unit_begin;
    int n_freq, n_beams, n_windows, w0, n_win, ftiles, btiles, n_shards;
};

// Device generate_weights (reference src/weights.cpp:11-60): canonical
// complex64 weights [shard][B][F_shard][A] for channels shard * F_shard + f.
bf_status launch_generate_weights(cudaStream_t stream, const float* pos, const float* freq, const float* dirs,
                                  float* out, uint64_t n_shards, uint64_t f_shard, uint64_t n_beams,
                                  uint64_t n_ant);

// One persistent launch (grid CTAs of 256 threads) over a tracker table;
// voltage rows come from `pool` ([rows][pool_freq][A] bytes).  A table with
// short_windows set holds only jobs of at most 16 spectra per window.
bf_status launch_served_tracker(cudaStream_t stream, int n_ant, bool short_windows, const uint8_t* pool,
                                uint64_t pool_freq, const TableHeader* table, int grid);

// One persistent launch (grid CTAs of 256 threads, a warp per chunk).
bf_status launch_served_quantize(cudaStream_t stream, const TableHeader* table, int grid);

}  // namespace bf
