// Host side of the FP32 three-pass 3-D r2c (fft3d.cuh): persistent grids
// sized from the occupancy of each pass.
#include "fft3d.cuh"
#include "launch.h"

namespace gabe {

namespace {

template <typename K>
cudaError_t persistent_grid(K kernel, int threads, size_t smem, int *grid) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *grid = nsm * per_sm;
    return cudaSuccess;
}

template <int N>
cudaError_t col_pass_n(const f3d::ColArgs &a, cudaStream_t s) {
    int g = 0;
    cudaError_t e = persistent_grid(f3d::col_fft_kernel<N>, f3d::kFftThreads, f3d::ColGeom<N>::SMEM_BYTES, &g);
    if (e != cudaSuccess) return e;
    f3d::col_fft_kernel<N><<<g, f3d::kFftThreads, f3d::ColGeom<N>::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}

template <int N>
cudaError_t col_oop_n(const f3d::ColArgs &a, cudaStream_t s) {
    int g = 0;
    constexpr size_t smem = f3d::ColGeom<N>::SMEM_BYTES;
    cudaError_t e = persistent_grid(f3d::col_fft_kernel<N, f3d::kColOutOfPlace>, f3d::kFftThreads, smem, &g);
    if (e != cudaSuccess) return e;
    f3d::col_fft_kernel<N, f3d::kColOutOfPlace><<<g, f3d::kFftThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// one pass of the 3-D r2c: 0 rows along k, 1 along j within every (component,
// i) plane, 2 along i for every (component, j).  With a scratch array T of
// S's size the passes along j and i run out of place (S -> T, then T -> S):
// on B200 a column pass that writes another array than it reads is faster.
template <int N>
cudaError_t fft3d_pass_n(float *S, float *T, int ncomp, int pass, cudaStream_t s) {
    constexpr long long nz = N / 2 + 1;
    if (pass < 0 || pass > 2) return cudaErrorInvalidValue;
    float2 *X = reinterpret_cast<float2 *>(S);
    if (T && pass > 0) {
        float2 *Y = reinterpret_cast<float2 *>(T);
        f3d::ColArgs a = pass == 1 ? f3d::ColArgs{Y, (long long)N * nz, 0, nz, ncomp * N, 1, (int)nz}
                                   : f3d::ColArgs{X, (long long)N * N * nz, nz, (long long)N * nz, ncomp, N, (int)nz};
        a.src = pass == 1 ? X : Y;
        return col_oop_n<N>(a, s);
    }
    if (pass == 0) {
        using RG = f3d::RowGeom<N>;
        int g1 = 0;
        cudaError_t e = persistent_grid(f3d::row_r2c_kernel<N>, RG::T, RG::SMEM_BYTES, &g1);
        if (e != cudaSuccess) return e;
        f3d::row_r2c_kernel<N><<<g1, RG::T, RG::SMEM_BYTES, s>>>(S, (long long)ncomp * N * N);
        return cudaGetLastError();
    }
    if (pass == 1) return col_pass_n<N>(f3d::ColArgs{X, (long long)N * nz, 0, nz, ncomp * N, 1, (int)nz}, s);
    if (pass == 2) return col_pass_n<N>(f3d::ColArgs{X, (long long)N * N * nz, nz, (long long)N * nz, ncomp, N, (int)nz}, s);
    return cudaErrorInvalidValue;
}

template <int N>
cudaError_t fft3d_n(float *S, float *T, int ncomp, cudaStream_t s) {
    for (int pass = 0; pass < 3; pass++) {
        const cudaError_t e = fft3d_pass_n<N>(S, T, ncomp, pass, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int N, int MODE>
cudaError_t col_slab_n(const f3d::ColArgs &a, cudaStream_t s) {
    int g = 0;
    constexpr size_t smem = f3d::ColGeom<N>::SMEM_BYTES_SLAB;
    cudaError_t e = persistent_grid(f3d::col_fft_kernel<N, MODE>, f3d::kFftThreads, smem, &g);
    if (e != cudaSuccess) return e;
    f3d::col_fft_kernel<N, MODE><<<g, f3d::kFftThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// 2-D r2c of the nplanes planes [N][N+2] of S (rows along k in place, then
// along j) written to the transpose's send buffer
template <int N>
cudaError_t plane_scatter_n(float *S, void *send, int nplanes, int ranks, cudaStream_t s) {
    constexpr long long nz = N / 2 + 1;
    using RG = f3d::RowGeom<N>;
    int g1 = 0;
    cudaError_t e = persistent_grid(f3d::row_r2c_kernel<N>, RG::T, RG::SMEM_BYTES, &g1);
    if (e != cudaSuccess) return e;
    f3d::row_r2c_kernel<N><<<g1, RG::T, RG::SMEM_BYTES, s>>>(S, (long long)nplanes * N);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    f3d::ColArgs a{reinterpret_cast<float2 *>(S), (long long)N * nz, 0, nz, nplanes, 1, (int)nz};
    a.dst = static_cast<float2 *>(send);
    a.ranks = ranks;
    return col_slab_n<N, f3d::kColScatter>(a, s);
}

}  // namespace

bool fft3d_supported(int N) { return N == 64 || N == 128 || N == 256 || N == 512; }

cudaError_t fft_col_pass_f32(int N, void *X, long long s1, long long s2, long long sn, int n1, int n2, int ncol,
                             cudaStream_t s) {
    f3d::ColArgs a{static_cast<float2 *>(X), s1, s2, sn, n1, n2, ncol};
    switch (N) {
        case 64: return col_pass_n<64>(a, s);
        case 128: return col_pass_n<128>(a, s);
        case 256: return col_pass_n<256>(a, s);
        case 512: return col_pass_n<512>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t fft_col_gather_f32(int N, const void *recv, void *T, int ncomp, int m, int ranks, cudaStream_t s) {
    const long long nz = N / 2 + 1;
    f3d::ColArgs a{static_cast<float2 *>(T), (long long)N * m * nz, nz, (long long)m * nz, ncomp, m, (int)nz};
    a.src = static_cast<const float2 *>(recv);
    a.ranks = ranks;
    switch (N) {
        case 64: return col_slab_n<64, f3d::kColGather>(a, s);
        case 128: return col_slab_n<128, f3d::kColGather>(a, s);
        case 256: return col_slab_n<256, f3d::kColGather>(a, s);
        case 512: return col_slab_n<512, f3d::kColGather>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t fft_plane_scatter_f32(int N, float *S, void *send, int nplanes, int ranks, cudaStream_t s) {
    switch (N) {
        case 64: return plane_scatter_n<64>(S, send, nplanes, ranks, s);
        case 128: return plane_scatter_n<128>(S, send, nplanes, ranks, s);
        case 256: return plane_scatter_n<256>(S, send, nplanes, ranks, s);
        case 512: return plane_scatter_n<512>(S, send, nplanes, ranks, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t fft3d_pass_f32(int N, float *S, float *T, int ncomp, int pass, cudaStream_t s) {
    switch (N) {
        case 64: return fft3d_pass_n<64>(S, T, ncomp, pass, s);
        case 128: return fft3d_pass_n<128>(S, T, ncomp, pass, s);
        case 256: return fft3d_pass_n<256>(S, T, ncomp, pass, s);
        case 512: return fft3d_pass_n<512>(S, T, ncomp, pass, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t fft3d_r2c_f32(int N, float *S, float *T, int ncomp, cudaStream_t s) {
    switch (N) {
        case 64: return fft3d_n<64>(S, T, ncomp, s);
        case 128: return fft3d_n<128>(S, T, ncomp, s);
        case 256: return fft3d_n<256>(S, T, ncomp, s);
        case 512: return fft3d_n<512>(S, T, ncomp, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gabe
