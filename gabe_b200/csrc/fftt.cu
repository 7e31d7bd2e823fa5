// Host side of the FP32 transposed three-pass transform and the fused pass
// along i + k-space update (fftt.cuh): persistent grids sized from each
// kernel's occupancy.
#include "fftt.cuh"
#include "launch.h"

namespace gabe {

namespace {

template <typename K>
cudaError_t grid_of(K kernel, int threads, size_t smem, int *grid) {
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

// Launch shapes: threads per CTA and ring depth of the passes with bulk copies.
constexpr int kRowT = 128;
constexpr int kColT = 512, kColNB = 2;
constexpr int kIkT = 192, kIkNB = 1, kIkMinB = 2;

template <int N>
cudaError_t rows_n(const float *S, float2 *T1, int ncomp, unsigned int *status, cudaStream_t s) {
    constexpr size_t smem = f3t::RowTGeom<N, kRowT>::SMEM_BYTES;
    auto k = f3t::rowt_kernel<N, kRowT>;
    int g = 0;
    cudaError_t e = grid_of(k, kRowT, smem, &g);
    if (e != cudaSuccess) return e;
    k<<<g, kRowT, smem, s>>>(S, T1, (long long)ncomp * N * N, status);
    return cudaGetLastError();
}

template <int N>
cudaError_t cols_n(const float2 *T1, float2 *T2, int ncomp, unsigned int *status, cudaStream_t s) {
    constexpr size_t smem = f3t::LineRing<N, f3t::kColW, kColNB>::SMEM_BYTES;
    int g = 0;
    cudaError_t e = grid_of(f3t::colt_kernel<N, kColT, kColNB>, kColT, smem, &g);
    if (e != cudaSuccess) return e;
    f3t::colt_kernel<N, kColT, kColNB><<<g, kColT, smem, s>>>(T1, T2, ncomp, status);
    return cudaGetLastError();
}

// The fused pass forms the polarization tensors in FP32 (pol_tensors32):
// 2.68 against 3.31 ms at 512^3 with FP64 ones, whose square roots and
// divisions held its warps at the barriers.
template <int N>
cudaError_t ik_n(const f3t::IkArgs &a, cudaStream_t s) {
    constexpr size_t smem = f3t::LineRing<N, 2 * kSrc, kIkNB, 2 * kSrc>::SMEM_BYTES;
    auto k = f3t::ikspace_kernel<N, kIkT, kIkNB, kIkMinB>;
    int g = 0;
    cudaError_t e = grid_of(k, kIkT, smem, &g);
    if (e != cudaSuccess) return e;
    k<<<g, kIkT, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

bool fftt_supported(int N) { return N == 64 || N == 128 || N == 256 || N == 512; }

cudaError_t fftt_rows_f32(int N, const float *S, void *T1, int ncomp, unsigned int *status, cudaStream_t s) {
    float2 *o = static_cast<float2 *>(T1);
    switch (N) {
        case 64: return rows_n<64>(S, o, ncomp, status, s);
        case 128: return rows_n<128>(S, o, ncomp, status, s);
        case 256: return rows_n<256>(S, o, ncomp, status, s);
        case 512: return rows_n<512>(S, o, ncomp, status, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t fftt_cols_f32(int N, const void *T1, void *T2, int ncomp, unsigned int *status, cudaStream_t s) {
    const float2 *i = static_cast<const float2 *>(T1);
    float2 *o = static_cast<float2 *>(T2);
    switch (N) {
        case 64: return cols_n<64>(i, o, ncomp, status, s);
        case 128: return cols_n<128>(i, o, ncomp, status, s);
        case 256: return cols_n<256>(i, o, ncomp, status, s);
        case 512: return cols_n<512>(i, o, ncomp, status, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t fftt_ikspace_f32(int N, const void *T2, void *G, const DevScalars *sc, const LatticeConsts &c, int slot,
                             unsigned int *status, cudaStream_t s) {
    f3t::IkArgs a{static_cast<const float2 *>(T2), static_cast<float2 *>(G), sc, c, slot, status};
    switch (N) {
        case 64: return ik_n<64>(a, s);
        case 128: return ik_n<128>(a, s);
        case 256: return ik_n<256>(a, s);
        case 512: return ik_n<512>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gabe
