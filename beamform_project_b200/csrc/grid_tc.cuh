// grid_tc.cuh -- job descriptors of the tcgen05 grid kernel, shared by the
// plain entry points and the served batch (serve.cu).
#pragma once

#include <cuda.h>

#include "bf_internal.cuh"
#include "serve.cuh"

namespace bf {

// One job as a launch sees it (a plain launch has one; a served launch reads
// a table of them).  Spectra are mapped to tile rows in 32-row TMEM lane
// quadrants: quadrant q of tile k holds spectra k*4R + q*R .. + R - 1 in its
// first R rows (R = rows_q).  R = 32 packs the tile densely; for windows of
// S < 32 spectra R is the largest multiple of S up to 32, so that every
// window lies inside one quadrant (the spare rows are zero).
struct TcJob {
    const uint8_t* split;       // prepared weights, [shard][F][hi|lo][K/64][N][128 B]
    float* integrated;          // [shard][n_windows][F][B]
    long long unit_begin;       // first unit of this job within the launch
    int n_time;                 // spectra this launch covers
    int t0;                     // tensor-map row of the launch's first spectrum
    int n_freq, n_beams, spectra;
    int beam_stride;            // beams per integrated row (n_beams, or all beam groups' beams)
    int n_windows;              // windows of the integrated array
    int w0;                     // integrated-array window of the launch's first window
    int rows_q;                 // R
    int tiles_per_channel, group_tiles, groups_per_channel;
    int n_shards;
};

// Table of a served launch in device memory: the header, then n_jobs TcJob
// entries sorted by unit_begin.  All jobs of one table share the tensor map
// (so its box, i.e. rows_q), the padded beam count, and the window kind
// (all S < 32 or all S >= 32).
using TcTableHeader = TableHeader;

__host__ __device__ inline int small_window_rows(int spectra) {
    return spectra >= 32 ? 32 : (32 / spectra) * spectra;
}

// Fills the tiling fields of `job` (rows_q, tiles, groups) for `n_time`
// spectra of windows of `spectra`; returns the job's unit count.
// group_mult > 1 makes each unit group_mult times the smallest unit (whole
// windows either way).
long long tc_job_tiling(TcJob& job, int n_time, int spectra, int n_freq, int n_shards, int group_mult = 1);

// 4-D map {antenna, channel, spectrum row, shard} over packed bytes with the
// given row and shard strides (bytes); the box is one channel of 128 rows,
// or of rows_q rows when rows_q < 32.
bf_status encode_voltage_map(CUtensorMap* map, const uint8_t* base, uint64_t n_ant, uint64_t n_freq,
                             uint64_t n_rows, uint64_t n_shards, uint64_t row_stride, uint64_t shard_stride,
                             int rows_q);

int tc_padded_beams(uint64_t b);

// One persistent launch (grid CTAs) over a device-resident job table.
// grid == 0 only sets the kernel's shared-memory attribute (call it once
// before capturing launches in a graph).
bf_status launch_grid_tensor_served(cudaStream_t stream, const CUtensorMap& map, int n_ant, int nb_pad,
                                    const TcTableHeader* table, int grid);

}  // namespace bf
