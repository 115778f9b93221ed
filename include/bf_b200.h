/*
 * bf_b200.h -- C ABI of the B200 (sm_100a) voltage-beamformer hot path.
 *
 * Plain pointers, sizes and a CUDA stream passed as `void*`: no C++ or torch
 * types cross this boundary, so any FFI (ctypes, cgo, JNI, N-API) can bind it.
 * The C++ API in include/beamformer/ (same names and exception types as the
 * reference's include/beamformer) is a thin layer over these calls.
 *
 * Conventions
 *  - Every call returns bf_status; BF_OK == 0.  On failure the message is kept
 *    per host thread and read with bf_last_error().  Nothing throws.
 *  - Device-stage calls ("bf_launch_*", "bf_grid_*", "bf_tracker*",
 *    "bf_doa_*") take device pointers and a stream, are stream-ordered,
 *    allocate no memory, take no lock and never synchronise the stream.
 *    Launch errors are reported as BF_ERR_CUDA; errors raised while the
 *    kernel runs surface at the caller's next synchronisation.
 *  - Layouts (little endian, row-major):
 *      voltage      u8  [T][F][A]  packed complex int4: low nibble = real,
 *                                  high nibble = imaginary, two's complement
 *      weights      f32 [B][F][A][2]           canonical (re, im)
 *      tiled weights f32 [F][ceil(B/32)][A][32][2]  (zero-padded last tile)
 *      intensity    f32 [T][F][B]
 *      integrated   f32 [W][F][B], W = ceil(T / S)
 *      codes        i8  [W][F][B]
 *      params       f32 [W][ceil(F/16)][ceil(B/16)][2]  (offset, scale)
 *    Calls that take n_shards process that many independent frequency
 *    shards stored back to back ([shard][...] for every array).
 */
#ifndef BF_B200_H
#define BF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define BF_API __declspec(dllexport)
#else
#define BF_API __attribute__((visibility("default")))
#endif

/* Status codes.  The C++ layer maps them back onto the reference's exception
 * types (src/cuda_beamformer.cu:22-27, include/beamformer/config.hpp:43-94). */
typedef enum bf_status {
    BF_OK = 0,
    BF_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    BF_ERR_LOGIC = 2,            /* std::logic_error      */
    BF_ERR_CUDA = 3,             /* std::runtime_error    */
    BF_ERR_OVERFLOW = 4,         /* std::overflow_error   */
    BF_ERR_OUT_OF_RANGE = 5,     /* std::out_of_range     */
    BF_ERR_TIMEOUT = 6,          /* a bounded device wait ran out */
    BF_ERR_UNSUPPORTED = 7,      /* valid request outside what the kernels support */
    BF_ERR_RESOURCE = 8          /* a served job can never fit the HBM budget */
} bf_status;

/* Dimensions: include/beamformer/config.hpp:74-79 (n_time, n_freq, n_ant,
 * n_beams).  Validation follows validate_dimensions (config.hpp:81-94). */
typedef struct bf_dims {
    uint64_t n_time;
    uint64_t n_freq;
    uint64_t n_ant;
    uint64_t n_beams;
} bf_dims;

/* Kernel selector: include/beamformer/cuda_stage_api.hpp:14-17 (Direct,
 * Tiled) plus the split-precision tcgen05 tensor-core kernel. */
typedef enum bf_kernel {
    BF_KERNEL_DIRECT = 0, /* canonical weights, reference float32 order   */
    BF_KERNEL_TILED = 1,  /* tiled weights,     reference float32 order   */
    BF_KERNEL_TENSOR = 2  /* split fp16 weights (bf_prepare_split_weights) */
} bf_kernel;

/* Library version string. */
BF_API const char* bf_version(void);

/* Copies the calling thread's last error message into buf (NUL-terminated,
 * truncated to n) and returns its full length. */
BF_API size_t bf_last_error(char* buf, size_t n);

/* validate_dimensions: include/beamformer/config.hpp:81-94. */
BF_API bf_status bf_validate_dimensions(const bf_dims* dims);

/* cuda_device_info: include/beamformer/cuda_beamformer.hpp:42.
 * name is NUL-terminated into name_buf (name_len bytes). */
BF_API bf_status bf_device_info(char* name_buf, size_t name_len, int* compute_major,
                                int* compute_minor, uint64_t* global_memory_bytes,
                                int* driver_version, int* runtime_version);

/* ------------------------------------------------------------------------ */
/* Device-stage API: include/beamformer/cuda_stage_api.hpp:21-42            */
/* ------------------------------------------------------------------------ */

/* launch_packed_beamformer (cuda_stage_api.hpp:21-25): per-spectrum power
 * [T][F][B].  kernel DIRECT reads canonical weights, TILED reads tiled
 * weights; both reproduce the reference float32 operation order exactly. */
BF_API bf_status bf_launch_packed_beamformer(int kernel, void* stream,
                                             const uint8_t* packed_voltage,
                                             const float* weights, float* intensity,
                                             const bf_dims* dims);

/* launch_packed_integrated_beamformer (cuda_stage_api.hpp:27-35): fused
 * beamform + increasing-time float32 integration over integration_spectra,
 * writing [W][F][B] with a partial last window.  Any integration length >= 1
 * is accepted here (the C++ layer keeps the reference's 10/320 rule). */
BF_API bf_status bf_launch_packed_integrated_beamformer(
    int kernel, void* stream, const uint8_t* packed_voltage, const float* weights,
    float* integrated_intensity, const bf_dims* dims, uint64_t integration_spectra);

/* launch_quantize_integrated_intensity (cuda_stage_api.hpp:37-42): one
 * (offset, scale) pair per 1x16x16 chunk; codes identical to
 * cpu_quantize_integrated_intensity (src/quantization.cpp:61-161). */
BF_API bf_status bf_launch_quantize_integrated_intensity(void* stream,
                                                         const float* integrated_intensity,
                                                         int8_t* codes, float* params,
                                                         const bf_dims* integrated_dims);

/* ------------------------------------------------------------------------ */
/* Split-precision tensor-core grid (tcgen05, sm_100a)                      */
/* No reference counterpart: the reference grid kernels are scalar float32  */
/* (src/cuda_beamformer.cu:108-354).  Same inputs, same output layouts.      */
/* ------------------------------------------------------------------------ */

/* Bytes of the prepared operand for n_shards shards of dims. */
BF_API uint64_t bf_split_weight_bytes(const bf_dims* dims, uint64_t n_shards);

/* Converts canonical complex64 weights ([shard][B][F][A][2], device) into the
 * tensor-core operand: each weight as an fp16 hi + lo pair (w = hi + lo to
 * about 2^-22 relative), in the kernel's swizzled shared-memory image. */
BF_API bf_status bf_prepare_split_weights(void* stream, const float* weights,
                                          void* split_weights, const bf_dims* dims,
                                          uint64_t n_shards);

/* Fused grid beamformer on tcgen05 tensor cores: |X.W|^2, integration over
 * integration_spectra (below 32, or a multiple of 32) and, when codes and params
 * are non-NULL, the int8 chunk quantizer.  Any n_ant the reference takes
 * (32, 64, 128, 256) and n_beams <= 128.  At 128 and 256 antennas the
 * voltage operand is held in tensor memory and the beams run in groups of 64
 * (32 at 256 antennas), one launch per group over the same voltage (one
 * channel's weight image for more beams does not fit in shared memory), and
 * the quantizer runs as a second kernel.
 * integrated may not be NULL (it is also the quantizer's input). */
BF_API bf_status bf_grid_tensor_integrated(void* stream, const uint8_t* packed_voltage,
                                           const void* split_weights, float* integrated,
                                           int8_t* codes, float* params, const bf_dims* dims,
                                           uint64_t integration_spectra, uint64_t n_shards);

/* Bytes of scratch bf_grid_tensor_quantized needs (one 32-bit arrival counter
 * per window and 16-channel group of every shard). */
BF_API uint64_t bf_grid_tensor_workspace_bytes(const bf_dims* dims, uint64_t integration_spectra,
                                               uint64_t n_shards);

/* bf_grid_tensor_integrated with the int8 chunk quantizer fused into the
 * kernel's epilogue: a chunk spans 16 channels owned by different CTAs, so
 * the CTA that finishes the last channel of a (window, 16-channel group)
 * quantizes that group's chunks.  `workspace` (bf_grid_tensor_workspace_bytes,
 * device memory owned by the caller) holds the arrival counters; the call
 * clears it on the stream before the kernel runs.  Codes and parameters are
 * identical to launch_quantize_integrated_intensity on the same integrated
 * output (src/quantization.cpp:61-161). */
BF_API bf_status bf_grid_tensor_quantized(void* stream, const uint8_t* packed_voltage,
                                          const void* split_weights, float* integrated,
                                          int8_t* codes, float* params, void* workspace,
                                          const bf_dims* dims, uint64_t integration_spectra,
                                          uint64_t n_shards);

/* bf_grid_tensor_quantized for callers that cannot allocate device memory
 * (device memory fixed at start-up, or an FFI caller holding only a stream
 * and its data buffers).  No counterpart in the reference.
 * The scratch is a fixed array inside this library (64 KiB on every GPU that
 * uses it, held until the process exits).  It holds the counters of the
 * quantizer fused into long windows, so with integration_spectra >= 32 the
 * request may need at most 16384 counters: n_shards * ceil(n_time /
 * integration_spectra) * ceil(n_freq / 16) <= 16384; larger requests fail
 * with BF_ERR_INVALID_ARGUMENT.  Shorter windows quantize in a second kernel
 * and use no counters, so they have no such limit.  The call allocates
 * nothing: it clears the counters it uses on the stream, then launches.
 * Each call made outside stream capture looks up the array's address on the
 * current device again (a cudaDeviceReset reloads the library's device code,
 * possibly elsewhere); a call made while the stream captures reuses the
 * address found by the last call on that device, so make the first call on a
 * device, and the first after a cudaDeviceReset, before any capture.  All
 * calls share the one array, which keeps the last call's counts: calls whose
 * kernels overlap on the GPU (different streams, or different host threads
 * on one device) race on it and must be serialised by the caller. */
BF_API bf_status bf_grid_tensor_quantized_static(void* stream, const uint8_t* packed_voltage,
                                                 const void* split_weights, float* integrated,
                                                 int8_t* codes, float* params, const bf_dims* dims,
                                                 uint64_t integration_spectra, uint64_t n_shards);

/* Covariance-form grid beamformer for long integration windows.  No
 * reference counterpart (the reference integrates spectrum by spectrum,
 * src/cuda_beamformer.cu:108-354); same outputs and layouts as
 * bf_grid_tensor_integrated.  Each window's integrated power is the quadratic
 * form v^T E v of its array covariance E = sum_t y(t) y(t)^T (exact INT32 on
 * int8 tensor cores), with v the beam weights split into fp16 hi + lo.
 * n_ant 64, integration_spectra a multiple of 64 up to 16384, n_freq even,
 * n_beams <= 128. */
BF_API uint64_t bf_cov_weight_bytes(const bf_dims* dims, uint64_t n_shards);

/* Canonical complex64 weights ([shard][B][F][A][2], device) -> the operand of
 * bf_grid_cov_integrated (128 KiB per channel). */
BF_API bf_status bf_prepare_cov_weights(void* stream, const float* weights, void* cov_weights,
                                        const bf_dims* dims, uint64_t n_shards);

/* Integrated power [shard][W][F][B] (and, when codes and params are non-NULL,
 * the int8 chunk codes and parameters of launch_quantize_integrated_intensity). */
BF_API bf_status bf_grid_cov_integrated(void* stream, const uint8_t* packed_voltage,
                                        const void* cov_weights, float* integrated, int8_t* codes,
                                        float* params, const bf_dims* dims,
                                        uint64_t integration_spectra, uint64_t n_shards);

/* bf_grid_cov_integrated that also writes, per value, the estimate
 * est = 2^-23 |v_b|^2 tr(E) / I of its relative error ([shard][W][F][B]
 * float, device): the fp32 sums of the quadratic form carry terms up to
 * |v_b|^2 tr(E), so est is large where a beam holds little of the window's
 * power (deep sidelobes of a strong source). */
BF_API bf_status bf_grid_cov_estimate(void* stream, const uint8_t* packed_voltage, const void* cov_weights,
                                      float* integrated, float* estimate, const bf_dims* dims,
                                      uint64_t integration_spectra, uint64_t n_shards);

/* Checked grid beamformer: the fastest tensor-core path that keeps every
 * value within 1e-5 relative of FP64.  No reference counterpart (same
 * outputs and layouts as launch_packed_integrated_beamformer plus
 * launch_quantize_integrated_intensity, cuda_stage_api.hpp:27-42).  Where the
 * covariance form applies (n_ant 64, even n_freq, integration_spectra a
 * multiple of 64 up to 16384) it runs that form with per-value error
 * estimates, then the split-precision kernel recomputes every (shard,
 * channel, window group) holding a value whose estimate exceeds the limit
 * calibrated against FP64; otherwise it runs the split-precision kernel.
 * The operand (bf_auto_weight_bytes) holds the covariance image (n_ant 64,
 * even n_freq) followed by the split image, both from canonical complex64
 * weights.  workspace (bf_grid_auto_workspace_bytes, 256-byte aligned,
 * device, zero bytes when the covariance form does not apply): its first
 * 32-bit word holds, after the call, how many split-kernel units were
 * recomputed. */
BF_API uint64_t bf_auto_weight_bytes(const bf_dims* dims, uint64_t n_shards);
BF_API bf_status bf_prepare_auto_weights(void* stream, const float* weights, void* auto_weights,
                                         const bf_dims* dims, uint64_t n_shards);
BF_API uint64_t bf_grid_auto_workspace_bytes(const bf_dims* dims, uint64_t integration_spectra,
                                             uint64_t n_shards);
BF_API bf_status bf_grid_auto_integrated(void* stream, const uint8_t* packed_voltage, const void* auto_weights,
                                         float* integrated, int8_t* codes, float* params, void* workspace,
                                         const bf_dims* dims, uint64_t integration_spectra, uint64_t n_shards);

/* ------------------------------------------------------------------------ */
/* Autotuner of the grid path.  No reference counterpart: the reference's    */
/* launch knobs are set by hand (V5ExecutionConfig,                          */
/* include/beamformer/cuda_beam_tracker_v5.hpp:45-49) or fixed at compile     */
/* time (src/cuda_beamformer.cu:140-143).                                     */
/* ------------------------------------------------------------------------ */

/* One launch choice of the grid path: form (bf_grid_auto_integrated: 0 the
 * split-precision kernel, 1 the checked covariance form), group_mult (split
 * kernel: time units of 1, 2 or 4 times the smallest whole-window unit),
 * paired (split kernel: CTA pairs walk channel pairs). */
typedef struct bf_grid_config {
    int32_t form;
    int32_t group_mult;
    int32_t paired;
    int32_t reserved;
} bf_grid_config;

/* Times every candidate choice for the class of (dims, integration_spectra)
 * -- n_ant, padded beams, integration length -- on seeded synthetic data of
 * that shape (at most 8192 spectra), keeps only candidates whose products
 * agree with the default's (bit for bit for the split kernel's choices,
 * within 1e-3 + 1e-5 |x| for the covariance form), and records the fastest
 * (it must beat the default by 2 %) in the tuning table, which untuned calls
 * of bf_grid_tensor_integrated, bf_grid_tensor_quantized(_static),
 * bf_grid_auto_integrated and the host pipeline then use.  Setup-time call:
 * it allocates and synchronises the stream.  Candidates (at most capacity;
 * 8 is enough), their best of three times (ms) and pass flags are written
 * out; *best is the index chosen (0 = the default). */
BF_API bf_status bf_autotune_grid(void* stream, const bf_dims* dims, uint64_t integration_spectra,
                                  uint64_t n_shards, bf_grid_config* candidates, float* candidate_ms,
                                  uint8_t* candidate_ok, uint32_t capacity, uint32_t* n_candidates,
                                  uint32_t* best);
/* bf_grid_auto_integrated with an explicit choice (tests, the tuner). */
BF_API bf_status bf_grid_auto_integrated_with(void* stream, const uint8_t* packed_voltage, const void* auto_weights,
                                              float* integrated, int8_t* codes, float* params, void* workspace,
                                              const bf_dims* dims, uint64_t integration_spectra,
                                              uint64_t n_shards, const bf_grid_config* config);
/* The tuning table: keyed by (device name, n_ant, padded beams,
 * integration_spectra); device NULL means the current device.  It is read
 * at first use from the cache file (beside this library, or $BF_TUNE_CACHE;
 * "off" reads and writes nothing) and written by bf_tune_save.  found is 0
 * (and *config the default) for a class never tuned. */
BF_API bf_status bf_tune_get(const char* device, int n_ant, int nb_pad, uint64_t integration_spectra,
                             bf_grid_config* config, int32_t* found);
BF_API bf_status bf_tune_set(const char* device, int n_ant, int nb_pad, uint64_t integration_spectra,
                             const bf_grid_config* config, float ms);
BF_API bf_status bf_tune_clear(void);
BF_API bf_status bf_tune_load(const char* path);  /* NULL: the cache file */
BF_API bf_status bf_tune_save(const char* path);  /* NULL: the cache file */
BF_API size_t bf_tune_cache_path(char* buf, size_t n);
/* The selection rule on its own: the fastest candidate with ok set, unless
 * it beats candidate 0 (the default) by less than min_gain (a fraction). */
BF_API bf_status bf_tune_pick(uint32_t n, const double* ms, const uint8_t* ok, double min_gain, uint32_t* best);

/* Host-buffer grid pipeline.  Counterpart of the reference's
 * CudaBeamformerWorkspace::run_quantized_integrated_pipeline
 * (include/beamformer/cuda_beamformer.hpp:66-76: weights resident, voltage
 * uploaded and products downloaded per call), with the block cut into time
 * chunks whose host->device copy, kernels and device->host copy overlap on
 * three streams.  Products are bit-identical to bf_grid_tensor_integrated over
 * the whole block.  Host layouts: voltage [shard][T][F][A] bytes, integrated
 * [shard][W][F][B] float, codes [shard][W][F][B] int8, params
 * [shard][W][F/16][B/16][offset, scale] float.  Pin the host buffers
 * (cudaHostAlloc / cudaHostRegister) for copies at PCIe rate alongside the
 * kernels.  A pipeline belongs to the device current at creation and to one
 * host thread at a time. */
typedef struct bf_grid_pipeline bf_grid_pipeline;

/* Spectra per chunk the pipeline would use: chunk_spectra itself (a multiple
 * of lcm(128, integration_spectra)) or, for 0, about 64 MiB of voltage;
 * never more than the block rounded up to that multiple.  0 for an invalid
 * request. */
BF_API uint64_t bf_grid_pipeline_chunk_spectra(const bf_dims* dims, uint64_t integration_spectra,
                                               uint64_t n_shards, uint64_t chunk_spectra);

/* Allocates two chunk slots of voltage and products and the prepared-weight
 * operand for n_shards shards of dims (dims.n_time is the block length).
 * Same limits as bf_grid_tensor_integrated. */
BF_API bf_status bf_grid_pipeline_create(const bf_dims* dims, uint64_t integration_spectra,
                                         uint64_t n_shards, uint64_t chunk_spectra,
                                         bf_grid_pipeline** pipeline);
/* bf_grid_pipeline_create for the checked grid beamformer
 * (bf_grid_auto_integrated): same buffers, chunks and products layout; the
 * uploaded weights become the checked form's operand. */
BF_API bf_status bf_grid_pipeline_create_checked(const bf_dims* dims, uint64_t integration_spectra,
                                                 uint64_t n_shards, uint64_t chunk_spectra,
                                                 bf_grid_pipeline** pipeline);

/* Canonical complex64 weights [shard][B][F][A][2] from host memory, prepared
 * into the resident split operand.  Synchronous. */
BF_API bf_status bf_grid_pipeline_upload_weights(bf_grid_pipeline* pipeline, const float* host_weights);

/* One block: host voltage in, host products out (integrated may be NULL when
 * codes and params are given; codes and params both or neither).  Returns
 * after the last product has reached host memory; *elapsed_ms (optional) is
 * the device time from the first copy-in to the last copy-out.
 * BF_ERR_TIMEOUT when a bounded device wait ran out. */
BF_API bf_status bf_grid_pipeline_run(bf_grid_pipeline* pipeline, const uint8_t* host_voltage,
                                      float* host_integrated, int8_t* host_codes, float* host_params,
                                      float* elapsed_ms);

BF_API bf_status bf_grid_pipeline_destroy(bf_grid_pipeline* pipeline);

/* Reads and clears the device-side error word of the tensor-core kernels
 * (0 = no error).  Every wait inside those kernels is bounded; a wait that
 * runs out sets a bit here (and the kernel returns) instead of hanging.
 * Synchronous: call after the stream has been synchronised.  No reference
 * counterpart (the reference kernels have no device-side waits). */
BF_API bf_status bf_take_device_error(uint32_t* code);

/* ------------------------------------------------------------------------ */
/* Tracker: include/beamformer/beam_tracker.hpp:91-100 (per-spectrum         */
/* [T][F][1]) and cuda_beam_tracker_v5.hpp:69-125 (device resident).         */
/* ------------------------------------------------------------------------ */

/* One steering direction per window (window_directions [W][3] float,
 * device), antenna positions [A][3] float (device) and per-channel wave
 * numbers 2*pi*f/c [F] double (device).  Weights are generated on the GPU
 * in registers: FP64 phase, reduced mod 2*pi in FP64, float sin/cos.
 *   mode 0: reference float32 order (matches beam_tracker_cpu bit-exactly up
 *           to the last bit of the sin/cos of the phase)
 *   mode 1: streaming tensor-core kernel (fp16 hi+lo weights, fp32 sums)
 * intensity ([T][F], may be NULL) receives per-spectrum power; integrated
 * ([W][F], may be NULL) receives the per-window sum. */
BF_API bf_status bf_tracker(void* stream, int mode, const uint8_t* packed_voltage,
                            const float* positions, const double* wave_numbers,
                            const float* window_directions, float* intensity,
                            float* integrated, const bf_dims* dims,
                            uint64_t integration_spectra);

/* ------------------------------------------------------------------------ */
/* DOA: covariance and Bartlett / Capon scan.  Reference: CpuOptBeamTracker */
/* (include/beamformer/cpu_opt_beam_tracker.hpp:91-169, src/cpu_opt_beam_   */
/* tracker.cpp:226-850, 1619-2454).  dims: n_time = blocks * block_len,     */
/* n_beams = 1.                                                             */
/* ------------------------------------------------------------------------ */

/* Exact per-block covariance on int8 tensor cores (tcgen05 kind::i8):
 * covariance[b][f][i][j] = sum over the block's spectra of x_i * conj(x_j),
 * (re, im) int32, full A x A Hermitian (A = 32 or 64; block_len a multiple
 * of 128 dividing n_time).  Replaces the float sums of
 * spatial_smoothed_covariance_into (src/cpu_opt_beam_tracker.cpp:559-602),
 * which equal these sums times 1/K. */
BF_API bf_status bf_doa_covariance_i32(void* stream, const uint8_t* packed_voltage,
                                       int32_t* covariance, const bf_dims* dims,
                                       uint64_t block_len);

/* Scratch bytes bf_doa_scan needs. */
BF_API uint64_t bf_doa_workspace_bytes(const bf_dims* dims, uint64_t block_len,
                                       uint64_t subarray);

/* FP64 smoothing (sub-arrays of `subarray` elements along the element index,
 * 0 = none), forward-backward averaging, diagonal loading diag_load*tr/M,
 * forgetting (S = forgetting*S + (1-forgetting)*R_block per block), FP64
 * Cholesky, and Bartlett / Capon powers on the grid l = l_first + i*l_step
 * (i < n_points) at m = m_fixed, summed over frequency; then the argmax and
 * parabolic peak of each block.  positions: [subarray][3] float (device) of
 * sub-array 0; wave_numbers [F] double.  Outputs (device): bartlett, capon
 * [blocks][n_points] double; l_est [blocks][2] double (Bartlett, Capon). */
BF_API bf_status bf_doa_scan(void* stream, const int32_t* covariance, const float* positions,
                             const double* wave_numbers, const bf_dims* dims, uint64_t block_len,
                             uint64_t subarray, double forgetting, double diag_load,
                             double l_first, double l_step, uint64_t n_points, double m_fixed,
                             double* bartlett, double* capon, double* l_est, void* workspace);

/* Channel-split DOA (no reference counterpart: the reference runs one job's
 * channels in one process).  The _slice entries are bf_doa_covariance_i32 and
 * bf_doa_scan on a contiguous slice of a job's channels -- dims.n_freq an even
 * count of 2 to 336, packed_voltage [T][slice][A], wave_numbers [slice] --
 * so that each GPU of a split job takes one slice; their bartlett and capon
 * outputs are the slice's partial sums over frequency (l_est is that of the
 * partial sums).  Summed over the slices (one all-reduce of
 * 2 x blocks x n_points doubles), they are the job's spectra up to the
 * order of the sum; bf_doa_peak then finds each block's peaks exactly as
 * bf_doa_scan does. */
BF_API bf_status bf_doa_covariance_i32_slice(void* stream, const uint8_t* packed_voltage,
                                             int32_t* covariance, const bf_dims* dims, uint64_t block_len);
BF_API bf_status bf_doa_scan_slice(void* stream, const int32_t* covariance, const float* positions,
                                   const double* wave_numbers, const bf_dims* dims, uint64_t block_len,
                                   uint64_t subarray, double forgetting, double diag_load,
                                   double l_first, double l_step, uint64_t n_points, double m_fixed,
                                   double* bartlett, double* capon, double* l_est, void* workspace);
BF_API bf_status bf_doa_peak(void* stream, const double* bartlett, const double* capon, uint64_t n_blocks,
                             uint64_t n_points, double l_first, double l_step, double* l_est);

/* The reference's adaptive tracker (CpuOptBeamTracker::run_into,
 * src/cpu_opt_beam_tracker.cpp:1619-2454) on the GPU: per window of
 * block_len spectra, the covariance fold above, then a coarse-to-fine
 * search -- a grid x grid lattice of (l, m) over +-fov around the previous
 * window's estimate (the prior for the first), `levels` 3 x 3 refinements at
 * halved pitch, the reference's 3-point quadratic interpolation -- with
 * Bartlett (estimator 0) or Capon (1) power summed over frequency; then the
 * beam along each window's estimate, per spectrum, in the reference's float32
 * order (its emission pass).  Fields follow CpuOptTrackerConfig
 * (include/beamformer/cpu_opt_beam_tracker.hpp:45-86). */
typedef struct bf_doa_track_config {
    uint64_t block_len;   /* integration_spectra: a multiple of 128 dividing n_time */
    uint64_t subarray;    /* spatial_smoothing_subarray_size: the search takes at most 16 elements
                           * after smoothing (0, no smoothing, only for n_ant <= 16) */
    uint32_t estimator;   /* 0 Bartlett, 1 Capon */
    uint32_t grid;        /* coarse_grid_resolution, 2 .. 64 */
    uint32_t levels;      /* refinement_levels, 0 .. 16 */
    uint32_t interp;      /* enable_quadratic_peak_interp */
    float fov_l, fov_m;   /* search_fov_l, search_fov_m */
    float forgetting;     /* forgetting_factor, (0, 1] */
    float diag_load;      /* diagonal_load */
    float prior_l, prior_m; /* the seeded trajectory's start direction */
} bf_doa_track_config;

BF_API uint64_t bf_doa_track_workspace_bytes(const bf_dims* dims, const bf_doa_track_config* config);

/* packed_voltage [T][F][A] (A = 32 or 64), positions [A][3] float, wave_numbers
 * [F] double, all device; outputs (device): window_directions [T/block_len][3]
 * float; intensity [T][F] float (per-spectrum beam power, may be NULL). */
BF_API bf_status bf_doa_track(void* stream, const uint8_t* packed_voltage, const float* positions,
                              const double* wave_numbers, const bf_dims* dims, const bf_doa_track_config* config,
                              float* window_directions, float* intensity, void* workspace);

/* ------------------------------------------------------------------------ */
/* Seeded synthetic voltages (no reference counterpart)                     */
/* ------------------------------------------------------------------------ */

/* Approximately Gaussian complex int4 noise (Irwin-Hall of eight 16-bit
 * uniforms) times `scale`, plus an optional source term mu ([U][F][A][2]
 * float, device, epoch u = t / epoch_len), rounded half-to-even and clipped
 * to [-8, 7].  Bit-identical to the CPU restatement in oracle/.  sample_offset
 * shifts the counter so shards and batches stay independent. */
BF_API bf_status bf_generate_voltage(void* stream, uint64_t seed, uint64_t sample_offset,
                                     float scale, const float* mu, uint64_t epoch_len,
                                     uint8_t* out, const bf_dims* dims);

/* Failure-path probe (no reference counterpart): one kernel waits, with the
 * same bounded mbarrier wait as the tensor-core kernels, on a barrier that
 * nothing arrives on; after limit_ns (at most 2e9) it gives up and sets bit
 * 30 of the device error word (read with bf_take_device_error).  Shows that
 * a wait that runs out surfaces on the host and leaves the context usable. */
BF_API bf_status bf_probe_bounded_wait(void* stream, uint64_t limit_ns);

/* Build check at run time (no reference counterpart): the binary and PTX
 * versions (cudaFuncAttributes) of a kernel of this library as loaded on the
 * current device, e.g. 100 and 100 for code built for sm_100a. */
BF_API bf_status bf_kernel_versions(int* binary_version, int* ptx_version);

/* Device generate_weights (reference src/weights.cpp:11-60): canonical
 * complex64 weights for n_shards blocks of dims->n_freq channels, written as
 * [shard][B][F][A][2] float, from positions [A][3], frequencies
 * [n_shards * F] (Hz) and unit beam directions [B][3] (all float, device).
 * Double-precision phase, then (float) cos / sin as in the reference. */
BF_API bf_status bf_generate_weights(void* stream, const float* positions, const float* frequencies,
                                     const float* directions, float* weights, const bf_dims* dims,
                                     uint64_t n_shards);

/* Loss-mask consumption.  The reference defines the per-shard loss mask
 * (include/beamformer/formats.hpp:22-30: uint8 [T][F], 0 = lost frame) but no
 * consumer.  In place on the packed voltage [T][F][A] (device, 16-byte
 * aligned): every byte of a lost frame becomes 0, so the frame adds nothing
 * to any beam, tracker or covariance.  valid_counts (device uint32
 * [ceil(T / integration_spectra)][F], may be null) receives the number of
 * valid frames per integration window and channel.  Nonzero mask bytes count
 * as valid.  Stream-ordered; allocates nothing. */
BF_API bf_status bf_apply_loss_mask(void* stream, uint8_t* packed_voltage, const uint8_t* loss_mask,
                                    const bf_dims* dims, uint64_t integration_spectra, uint32_t* valid_counts);

/* ------------------------------------------------------------------------ */
/* Served, continuously batched mode (no reference counterpart)             */
/* ------------------------------------------------------------------------ */
/*
 * A server owns one CUDA stream, an HBM arena of hbm_budget_bytes for
 * per-job device state, and device voltage pools (one per antenna count,
 * [pool_spectra][pool_channels][A] packed bytes from the seeded generator)
 * that stand in for the ingest buffers.  Jobs are submitted at any time and
 * queue first-in first-out; each bf_serve_step admits queued jobs while their
 * state fits the arena and a live slot is free, then runs one served window
 * (window_spectra spectra) of every live job as one CUDA-graph replay: the
 * jobs of each kernel class share one persistent launch over a device job
 * table, rewritten by one copy before the replay.  A job's window k reads
 * pool rows (pool_offset + k * window_spectra) mod pool_spectra.
 * Calls are host-side, not thread-safe for one server, and never block on
 * the GPU except bf_serve_sync, bf_serve_stats (which waits for the steps it
 * reports) and bf_serve_release of a job the GPU may still be using.
 */
typedef struct bf_server bf_server;

typedef enum bf_serve_kind { BF_SERVE_GRID = 0, BF_SERVE_TRACKER = 1 } bf_serve_kind;

typedef enum bf_job_state {
    BF_JOB_QUEUED = 0,     /* submitted, waiting for HBM or a slot */
    BF_JOB_LIVE = 1,       /* admitted; windows still to launch */
    BF_JOB_RUNNING = 2,    /* every window launched, not yet complete on the GPU */
    BF_JOB_DONE = 3,       /* results complete in device memory */
    BF_JOB_CANCELLED = 4,  /* cancelled; its state may be released */
    BF_JOB_UNKNOWN = 5
} bf_job_state;

typedef struct bf_serve_config {
    uint64_t hbm_budget_bytes;  /* admission budget for per-job device state */
    uint32_t max_jobs;          /* live slots */
    uint32_t window_spectra;    /* spectra per job per step; a multiple of 32 */
    uint64_t pool_spectra;      /* rows per voltage pool; a multiple of window_spectra */
    uint32_t shard_channels;    /* channels per shard (336) */
    uint32_t max_shards;        /* shards per pool row (pool_channels = max_shards * shard_channels) */
    uint64_t pool_seed;         /* pool for A antennas: bf_generate_voltage(seed + A, 0, scale) */
    float pool_scale;
    /* > 0: also admit only while the predicted device time of a window stays
     * within this many microseconds (a job that alone exceeds it is admitted
     * when nothing else is live).  0: HBM budget and slots only. */
    float window_budget_us;
    /* Windows each step serves per live job (0 or 1: one).  More windows per
     * step load each grid channel's weights once for all of them and spread
     * the step's fixed costs, at the price of latency: a throughput setting
     * for a server that has fallen behind its stream.  A job's windows in one
     * step stop at its last window and at the end of the voltage pool. */
    uint32_t windows_per_step;
} bf_serve_config;

typedef struct bf_serve_job {
    int32_t kind;                 /* bf_serve_kind */
    uint32_t n_ant;               /* 32 or 64 */
    uint32_t n_shards;            /* 1 .. max_shards */
    uint32_t n_beams;             /* grid: beams (1..128); tracker: sources (1..16) */
    uint64_t n_spectra;           /* a multiple of window_spectra */
    uint64_t integration_spectra; /* divides window_spectra; grid: below 32 or a multiple of 32 */
    uint64_t pool_offset;         /* a multiple of window_spectra */
    const float* positions;       /* host [n_ant][3] metres */
    const float* frequencies;     /* host [n_shards * shard_channels] Hz */
    const float* directions;      /* grid: host [n_beams][3] unit vectors */
    const float* trajectories;    /* tracker: host [n_beams][4] l0, m0, dl, dm (per spectrum) */
    int32_t quantize;             /* grid: int8 chunk codes and parameters as well */
    int32_t pad;
} bf_serve_job;

typedef struct bf_serve_stats {
    uint64_t steps;               /* served windows launched */
    uint64_t steps_timed;         /* of which complete and timed */
    uint64_t job_windows;         /* job windows launched */
    uint64_t jobs_submitted, jobs_admitted, jobs_done, jobs_cancelled, jobs_rejected;
    uint64_t live_jobs, queued_jobs;
    uint64_t arena_bytes_in_use, arena_bytes_peak;
    uint64_t graph_captures;
    double beam_samples;          /* sum over launched job windows of spectra x channels x beams */
    double step_ms_total;         /* sum of per-step device time (CUDA events) */
    double step_ms_p50, step_ms_p99, step_ms_max;
    uint64_t kernel_launches;     /* kernels launched by the steps (one per non-empty class) */
    double predicted_ms_last;     /* cost model's device time of the last step */
} bf_serve_stats;

/* Footprint in the arena of one job (0 for an invalid job). */
BF_API uint64_t bf_serve_job_bytes(const bf_serve_config* config, const bf_serve_job* job);
BF_API bf_status bf_serve_create(const bf_serve_config* config, bf_server** server);
/* A scheduler-only server: the same admission, arena accounting, job tables
 * and job states with no device work (every step completes when issued;
 * results are not produced).  For testing the host logic without a GPU. */
BF_API bf_status bf_serve_create_host_only(const bf_serve_config* config, bf_server** server);
BF_API bf_status bf_serve_destroy(bf_server* server);
/* Validates and queues a job (host inputs are copied).  BF_ERR_RESOURCE when
 * its footprint exceeds the whole budget. */
BF_API bf_status bf_serve_submit(bf_server* server, const bf_serve_job* job, uint64_t* job_id);
/* Admits what fits, then launches one window of every live job. */
BF_API bf_status bf_serve_step(bf_server* server, uint32_t* n_live);
BF_API bf_status bf_serve_poll(bf_server* server, uint64_t job_id, int32_t* state);
/* When a job ran, in server steps (indices of bf_serve_step_times: the k-th
 * step that launched work).  submit_step: steps launched before its
 * submission; admit_step: the step that ran its first window; last_step: the
 * step that ran its last one; UINT64_MAX for steps not reached yet.  With the
 * step times and the stream time of each step a caller replays the job's
 * admission wait and completion latency. */
typedef struct bf_serve_job_info {
    int32_t state;
    uint32_t pad;
    uint64_t submit_step;
    uint64_t admit_step;
    uint64_t last_step;
    uint64_t windows_launched;
} bf_serve_job_info;
BF_API bf_status bf_serve_job_info_get(bf_server* server, uint64_t job_id, bf_serve_job_info* info);
/* Device pointers of a DONE job's results (any may be NULL): integrated
 * f32, grid [shard][W][F][B] / tracker [W][F_total][sources], W =
 * n_spectra / integration_spectra; codes i8 and params f32 pairs as in the
 * quantizer's layout.  Valid until bf_serve_release. */
BF_API bf_status bf_serve_result(bf_server* server, uint64_t job_id, float** integrated, int8_t** codes,
                                 float** params, uint64_t* n_windows);
BF_API bf_status bf_serve_cancel(bf_server* server, uint64_t job_id);
/* Job checkpoints (no reference counterpart).  bf_serve_checkpoint writes a
 * self-contained image of a queued, live, running or done job -- its
 * description, the windows served so far and their results -- into buffer
 * (host, capacity bytes); with buffer NULL it only sets *bytes.  For a job
 * with windows in flight it first waits for the server's launched windows.
 * bf_serve_restore queues the job of an image in a server with the same
 * window, shard and pool settings (BF_ERR_INVALID_ARGUMENT otherwise, or for
 * a damaged image); it resumes at its next window and its results equal
 * those of an uninterrupted run bit for bit, provided the target server's
 * voltage pool holds the same rows as the source's (the image records the
 * job's pool offset, not the pool's contents: rows written into only one of
 * the pools through bf_serve_pool change the restored job's results).  The
 * original job is not touched: cancel and release it as usual. */
BF_API bf_status bf_serve_checkpoint(bf_server* server, uint64_t job_id, void* buffer, uint64_t capacity,
                                     uint64_t* bytes);
BF_API bf_status bf_serve_restore(bf_server* server, const void* image, uint64_t bytes, uint64_t* job_id);
/* Returns the job's arena block (waits for the GPU if it may still use it). */
BF_API bf_status bf_serve_release(bf_server* server, uint64_t job_id);
/* Waits for every launched step; BF_ERR_TIMEOUT if a kernel reported a
 * bounded wait that ran out. */
BF_API bf_status bf_serve_sync(bf_server* server);
BF_API bf_status bf_serve_stats_get(bf_server* server, bf_serve_stats* stats);
/* Per-step device times (ms) of the timed steps, oldest first. */
BF_API bf_status bf_serve_step_times(bf_server* server, float* out, uint64_t capacity, uint64_t* count);
/* Ids of jobs that became DONE since the last call (up to capacity), oldest
 * first: a completion queue, so callers need not poll every job. */
BF_API bf_status bf_serve_take_done(bf_server* server, uint64_t* ids, uint64_t capacity, uint64_t* count);
/* The server's stream (cudaStream_t as void*), for reading results in order. */
BF_API void* bf_serve_stream(bf_server* server);
/* Ingest hook.  The reference feeds each job from host memory and names
 * ingest straight into GPU memory as the way past the host bounce
 * (info/cuda_implementation_investigation.md:70-76).  This returns the device
 * pool that jobs of n_ant antennas read, [pool_spectra][pool_channels][n_ant]
 * packed bytes (pool_channels = max_shards * shard_channels; shard s of a job
 * is channels [s * shard_channels, (s + 1) * shard_channels)).  A capture
 * stage -- GPUDirect RDMA, a peer copy, a kernel -- writes rows there in
 * stream order before the bf_serve_step whose windows read them: on
 * bf_serve_stream(server), or on its own stream followed by an event that
 * the caller makes the server stream wait on.  Window k of a job reads rows
 * (pool_offset + k * window_spectra) mod pool_spectra; rows that launched
 * windows may still read are rewritten only after those steps complete
 * (bf_serve_sync).  BF_ERR_LOGIC for a host-only server. */
BF_API bf_status bf_serve_pool(bf_server* server, uint64_t n_ant, uint8_t** pool, uint64_t* pool_spectra,
                               uint64_t* pool_channels);

#ifdef __cplusplus
}
#endif

#endif /* BF_B200_H */
