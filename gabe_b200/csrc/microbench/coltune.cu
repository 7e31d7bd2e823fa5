// Microbenchmark of the column passes (fft3d.cuh col_fft_kernel, in place)
// along j and along i over ten 512^3 half spectra at 256, 512 and 1024
// threads per CTA, timed with CUDA events (best of 5 after one warm-up).
#include <cstdio>
#include <vector>
#include "fft3d.cuh"
using namespace gabe;
constexpr int N = 512;
constexpr long long nz = N / 2 + 1;
template <int T>
void run(float2 *X, int ncomp, const char *what, const f3d::ColArgs &a) {
    using G = f3d::ColGeom<N, T>;
    auto k = f3d::col_fft_kernel<N, f3d::kColInPlace, T>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM_BYTES);
    int per = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, T, G::SMEM_BYTES);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    if (per < 1) { printf("T=%d: no occupancy\n", T); return; }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float best = 1e9;
    const size_t bytes = (size_t)ncomp * N * N * nz * 8;
    for (int rep = 0; rep < 6; rep++) {
        cudaMemset(X, 0, bytes);
        cudaEventRecord(e0);
        k<<<nsm * per, T, G::SMEM_BYTES>>>(a);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms; cudaEventElapsedTime(&ms, e0, e1);
        if (rep >= 1 && ms < best) best = ms;
    }
    printf("%s T=%d per_sm=%d best %.3f ms  %.2f TB/s  %s\n", what, T, per, best, 2.0 * bytes / (best * 1e-3) / 1e12,
           cudaGetErrorString(cudaGetLastError()));
}
int main() {
    const int ncomp = 10;
    float2 *X;
    if (cudaMalloc(&X, (size_t)ncomp * N * N * nz * 8) != cudaSuccess) { printf("alloc failed\n"); return 1; }
    f3d::ColArgs aj{X, (long long)N * nz, 0, nz, ncomp * N, 1, (int)nz};
    f3d::ColArgs ai{X, (long long)N * N * nz, nz, (long long)N * nz, ncomp, N, (int)nz};
    run<512>(X, ncomp, "j", aj);
    run<256>(X, ncomp, "j", aj);
    run<1024>(X, ncomp, "j", aj);
    run<512>(X, ncomp, "i", ai);
    run<256>(X, ncomp, "i", ai);
    run<1024>(X, ncomp, "i", ai);
    cudaFree(X);
    return 0;
}
