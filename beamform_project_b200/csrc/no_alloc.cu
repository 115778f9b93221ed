// no_alloc.cu -- an entry point for callers that cannot allocate device memory.
//
// bf_grid_tensor_quantized needs a small scratch buffer (one arrival counter
// per window and 16-channel group) that the caller allocates.  Some callers
// cannot do that: a real-time acquisition process whose device memory is
// carved up once at start-up and must not change while data flows, or a
// caller that reaches this library through a foreign-function interface
// holding only a stream and the data buffers, with no handle on a CUDA
// allocator.  bf_grid_tensor_quantized_static runs the same kernel with its
// scratch in the fixed array below, which every GPU that loads this library
// holds from the first use until the process exits.
#include "bf_internal.cuh"

namespace {

// Scratch of bf_grid_tensor_quantized_static: up to kStaticCounters 32-bit
// counters (64 KiB per device).
constexpr uint64_t kStaticCounters = 16384;
static __device__ __align__(256) unsigned g_static_counters[kStaticCounters];

// Device addresses of g_static_counters, one per device (see
// device_symbol_address: looked up again on every call outside capture).
bf::SymbolAddressCache g_address;

}  // namespace

extern "C" {

// See include/bf_b200.h.
BF_API bf_status bf_grid_tensor_quantized_static(void* stream, const uint8_t* packed_voltage,
                                                 const void* split_weights, float* integrated,
                                                 int8_t* codes, float* params, const bf_dims* dims,
                                                 uint64_t integration_spectra, uint64_t n_shards) {
    using namespace bf;
    clear_error();
    bf_status st = validate_dims(dims);
    if (st != BF_OK) return st;
    if (n_shards == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be positive");
    if (integration_spectra == 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must be positive");
    }
    if (integration_spectra > 32 && integration_spectra % 32 != 0) {
        return set_error(BF_ERR_UNSUPPORTED,
                         "the tensor-core kernel needs integration_spectra below 32 or a multiple of 32");
    }
    // The counters serve the quantizer fused into the long-window epilogue
    // (integration_spectra >= 32); short windows quantize in a second kernel
    // and use none, so only long windows are held to the array's size.
    if (integration_spectra >= 32) {
        const uint64_t needed = grid_tensor_counter_count(*dims, integration_spectra, n_shards);
        if (needed > kStaticCounters) {
            return set_error(BF_ERR_INVALID_ARGUMENT,
                             "request needs " + std::to_string(needed) +
                                 " scratch counters (n_shards * windows * ceil(n_freq / 16)); the "
                                 "allocation-free entry point holds at most " +
                                 std::to_string(kStaticCounters));
        }
    }
    if (packed_voltage == nullptr || split_weights == nullptr || integrated == nullptr || codes == nullptr ||
        params == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "every buffer must be given");
    }
    if (reinterpret_cast<uintptr_t>(packed_voltage) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(split_weights) % 16 != 0 || reinterpret_cast<uintptr_t>(integrated) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(params) % 8 != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         "packed_voltage, split_weights and integrated must be 16-byte aligned, params 8-byte");
    }
    void* scratch = nullptr;
    st = device_symbol_address(&g_static_counters, g_address, static_cast<cudaStream_t>(stream), &scratch,
                               "static scratch");
    if (st != BF_OK) return st;
    return launch_grid_tensor(static_cast<cudaStream_t>(stream), packed_voltage, split_weights, integrated, codes,
                              params, *dims, integration_spectra, n_shards, static_cast<unsigned*>(scratch));
}

}  // extern "C"
