// grid_tc.cu -- split-precision tcgen05 grid beamformer (placeholder).
#include "bf_internal.cuh"

namespace bf {

uint64_t split_weight_bytes(const bf_dims& d, uint64_t n_shards) {
    return n_shards * d.n_freq * 2ull * 256ull * 2ull * d.n_ant * 2ull;
}

bf_status launch_prepare_split(cudaStream_t, const float*, void*, const bf_dims&, uint64_t) {
    return set_error(BF_ERR_UNSUPPORTED, "tensor-core kernel not built");
}

bf_status launch_grid_tensor(cudaStream_t, const uint8_t*, const void*, float*, int8_t*, float*,
                             const bf_dims&, uint64_t, uint64_t) {
    return set_error(BF_ERR_UNSUPPORTED, "tensor-core kernel not built");
}

}  // namespace bf
