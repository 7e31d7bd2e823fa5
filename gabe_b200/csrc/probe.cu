// Diagnostic of the bounded device waits (include/gabe.h: gabe_wait_probe).
//
// Every wait of the library's kernels on an mbarrier (the bulk copies of
// the transform passes, the TMA loads and MMAs of the emulator's tcgen05
// forward) goes through tma::mbar_wait_for: a wait that sees no completion
// within its limit of GPU time raises ST_TIMEOUT in a status word and
// returns, so that a copy that never lands ends the kernel instead of
// hanging the GPU.  This entry point runs that wait on a barrier that
// nothing arrives at -- the failure made on purpose, without a fault -- so
// that a test can check that the wait gives up, the status reaches the
// host, and the context stays usable.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gabe.h"
#include "tma.cuh"

namespace {

__global__ void wait_probe_kernel(unsigned long long limit_ns, unsigned int *status, unsigned long long *waited_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        gabe::tma::mbar_init(&bar, 1);  // one arrival expected; none will come
        gabe::tma::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long t0 = gabe::tma::now_ns();
        gabe::tma::mbar_wait_for(&bar, 0, status, limit_ns);
        *waited_ns = gabe::tma::now_ns() - t0;
    }
}

}  // namespace

extern "C" int gabe_wait_probe(int64_t limit_ns, uint32_t *status_out, int64_t *waited_ns_out) {
    if (limit_ns <= 0 || limit_ns > 10000000000LL) return GABE_ERR_PARAM;
    unsigned int *st = nullptr;
    unsigned long long *w = nullptr;
    if (cudaMalloc(&st, sizeof(*st)) != cudaSuccess || cudaMalloc(&w, sizeof(*w)) != cudaSuccess ||
        cudaMemset(st, 0, sizeof(*st)) != cudaSuccess) {
        cudaGetLastError();
        if (st) cudaFree(st);
        return GABE_ERR_CUDA;
    }
    wait_probe_kernel<<<1, 32>>>((unsigned long long)limit_ns, st, w);
    unsigned int hs = 0;
    unsigned long long hw = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&hw, w, sizeof(hw), cudaMemcpyDeviceToHost);
    cudaFree(st);
    cudaFree(w);
    if (e != cudaSuccess) return GABE_ERR_CUDA;
    if (status_out) *status_out = hs;
    if (waited_ns_out) *waited_ns_out = (int64_t)hw;
    return (hs & gabe::ST_TIMEOUT) ? GABE_ERR_TIMEOUT : GABE_OK;
}
