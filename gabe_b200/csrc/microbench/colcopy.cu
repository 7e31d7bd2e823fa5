// Copy ceiling of the column passes' access pattern: tiles of W complex
// columns x N rows moved through a two-tile cp.async ring and stored out of
// place (one 512-thread CTA per SM), over ten 512^3 half spectra, in the
// geometry of the pass along i and of the pass along j, for W = 8, 16, 24;
// CUDA events, best of 3 after one warm-up.
#include <cstdio>
#include "sweep32.cuh"
constexpr int N = 512;
constexpr long long nz = N / 2 + 1;
template <int W>
__global__ void __launch_bounds__(512, 1) colcopy(const float2 *X, float2 *Y, long long s1, long long s2, long long sn,
                                                  int n1, int n2) {
    extern __shared__ __align__(16) float2 cs[];
    const int tid = threadIdx.x, T = blockDim.x;
    const int ncb = (int)((nz + W - 1) / W);
    const long long ntiles = (long long)n1 * n2 * ncb;
    auto base_of = [&](long long tile, int &wn) {
        const int cb = (int)(tile % ncb);
        const long long b = tile / ncb;
        const int b2 = (int)(b % n2), b1 = (int)(b / n2);
        wn = (int)min((long long)W, nz - cb * W);
        return b1 * s1 + b2 * s2 + cb * W;
    };
    auto issue = [&](long long tile, int buf) {
        int wn;
        const long long o = base_of(tile, wn);
        float2 *col = cs + buf * N * W;
        for (int t = tid; t < N * W; t += T) {
            const int n = t / W, w = t % W;
            if (w < wn) gabe::s32::cp_async8(col + t, X + o + n * sn + w);
        }
    };
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    gabe::s32::cp_commit();
    int it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        gabe::s32::cp_wait<0>();
        __syncthreads();
        const long long ahead = tile + gridDim.x;
        if (ahead < ntiles) issue(ahead, (it + 1) & 1);
        gabe::s32::cp_commit();
        int wn;
        const long long o = base_of(tile, wn);
        const float2 *col = cs + (it & 1) * N * W;
        for (int t = tid; t < N * W; t += T) {
            const int n = t / W, w = t % W;
            if (w < wn) __stcs(Y + o + n * sn + w, col[t]);
        }
    }
    gabe::s32::cp_wait<0>();
}
template <int W>
void run(const float2 *X, float2 *Y, const char *what, long long s1, long long s2, long long sn, int n1, int n2) {
    const size_t smem = 2 * (size_t)N * W * sizeof(float2);
    cudaFuncSetAttribute(colcopy<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    float best = 1e9;
    for (int r = 0; r < 4; r++) {
        cudaEventRecord(a);
        colcopy<W><<<nsm, 512, smem>>>(X, Y, s1, s2, sn, n1, n2);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms; cudaEventElapsedTime(&ms, a, b);
        if (r && ms < best) best = ms;
    }
    const double bytes = 2.0 * 10 * N * (double)N * nz * 8;
    printf("%s W=%2d  %.3f ms  %.2f TB/s  %s\n", what, W, best, bytes / (best * 1e-3) / 1e12, cudaGetErrorString(cudaGetLastError()));
}
int main() {
    const size_t n = 10ull * N * N * nz;
    float2 *X, *Y;
    if (cudaMalloc(&X, n * 8) != cudaSuccess || cudaMalloc(&Y, n * 8) != cudaSuccess) { printf("alloc\n"); return 1; }
    cudaMemset(X, 0, n * 8);
    // pass along i: lines (q, j), stride N nz; pass along j: lines (q, i), stride nz
    const long long si1 = (long long)N * N * nz, si2 = nz, sin = (long long)N * nz;
    const long long sj1 = (long long)N * nz, sjn = nz;
    run<8>(X, Y, "i", si1, si2, sin, 10, N);
    run<16>(X, Y, "i", si1, si2, sin, 10, N);
    run<24>(X, Y, "i", si1, si2, sin, 10, N);
    run<8>(X, Y, "j", sj1, 0, sjn, 10 * N, 1);
    run<16>(X, Y, "j", sj1, 0, sjn, 10 * N, 1);
    run<24>(X, Y, "j", sj1, 0, sjn, 10 * N, 1);
    cudaFree(X); cudaFree(Y);
    return 0;
}
