// Self-test of the failure path every TMA-fed kernel relies on: a bounded mbarrier wait that runs
// out reports a status the host reads, and the context stays usable afterwards. No counterpart in
// the reference. The kernel waits, through the same bounded-wait routine the kernels use, on an
// mbarrier that nothing arrives on (arrive = 0) or that it has completed itself (arrive = 1).
#include "common.cuh"
#include "tma.cuh"

namespace bd {

__global__ void k_selftest_wait(unsigned polls, int arrive, int* __restrict__ status) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_init_fence();
    if (arrive) mbar_arrive(&bar);
    *status = mbar_wait_limit(&bar, 0, polls) ? 0 : 1;
}

}  // namespace bd

using namespace bd;

extern "C" int bd_selftest_wait_timeout(int max_polls, int arrive, void* stream) {
    BD_REQUIRE(max_polls >= 1 && max_polls <= (1 << 20), "bd_selftest_wait_timeout: max_polls must be 1..2^20");
    cudaStream_t st = as_stream(stream);
    int* status = nullptr;
    BD_CUDA(cudaMallocAsync((void**)&status, sizeof(int), st));
    int host = -1;
    cudaError_t e = cudaMemsetAsync(status, 0xff, sizeof(int), st);
    if (e == cudaSuccess) {
        k_selftest_wait<<<1, 32, 0, st>>>((unsigned)max_polls, arrive ? 1 : 0, status);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e2 = cudaFreeAsync(status, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "bd_selftest_wait_timeout");
    if (e2 != cudaSuccess) return cuda_status(e2, "bd_selftest_wait_timeout: cudaFreeAsync");
    if (host == 1) return fail(BD_ERR_TIMEOUT, "bd_selftest_wait_timeout: the bounded wait gave up after %d polls",
                               max_polls);
    if (host != 0) return fail(BD_ERR_STATE, "bd_selftest_wait_timeout: the kernel did not report");
    return BD_OK;
}
