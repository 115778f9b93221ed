// selftest.cu -- exercises the bounded-wait path of the tensor-core kernels.
//
// Every mbarrier wait in grid_tc.cu and doa_cov.cu goes through
// sm100::mbar_wait, which gives up after a wall-clock limit and lets the
// kernel record an error code and return instead of hanging.  This probe
// waits on a barrier that nothing ever arrives on, with a caller-chosen limit
// (at most 2 s), and records bit 30 of the device error word when the wait
// runs out, so a test can check that the failure surfaces on the host and
// that the context stays usable.  No async copy or MMA is in flight.
#include "bf_internal.cuh"
#include "sm100.cuh"

namespace bf {
namespace {

using namespace sm100;

__global__ void bounded_wait_probe_kernel(uint64_t limit_ns, unsigned* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait(&bar, 0, limit_ns) && err != nullptr) atomicOr(err, 1u << 30);
}

}  // namespace
}  // namespace bf

extern "C" BF_API bf_status bf_probe_bounded_wait(void* stream, uint64_t limit_ns) {
    using namespace bf;
    clear_error();
    if (limit_ns == 0 || limit_ns > 2000000000ull) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "limit_ns must be between 1 and 2e9");
    }
    unsigned* err = device_error_word(static_cast<cudaStream_t>(stream));
    if (err == nullptr) return BF_ERR_CUDA;
    bounded_wait_probe_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limit_ns, err);
    return cuda_status(cudaGetLastError(), "bounded_wait_probe_kernel launch");
}

extern "C" BF_API bf_status bf_kernel_versions(int* binary_version, int* ptx_version) {
    using namespace bf;
    clear_error();
    if (binary_version == nullptr || ptx_version == nullptr) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "binary_version and ptx_version must be given");
    }
    cudaFuncAttributes attr{};
    BF_RETURN_IF(cuda_status(cudaFuncGetAttributes(&attr, bounded_wait_probe_kernel), "cudaFuncGetAttributes"));
    *binary_version = attr.binaryVersion;
    *ptx_version = attr.ptxVersion;
    return BF_OK;
}
