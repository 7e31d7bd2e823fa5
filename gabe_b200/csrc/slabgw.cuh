// GW branch of a lattice split into slabs along i (slab.cu), for FP32
// storage (kernels_f32.cu) and FP64 (kernels_f64.cu, reference operation
// order: no FMA contraction).
//
// The 3-D transform of the ten source arrays (fft_stresstensor,
// g2evolutionpert.cpp:183-195) runs as
//   1. a 2-D r2c over (j, k) of every own plane, S[q][il][ky][kz],
//      il < nplanes, into the send buffer in blocks by destination rank:
//      rank r' receives the ky columns it owns, [y0_r', y0_r' + m_r'), of
//      every plane.  FP32: the library's passes (fft3d.cuh), the one along
//      j writing the blocks directly; FP64: cuFFT D2Z in place and the
//      pack (below);
//   2. the all-to-all, by the caller;
//   3. the pass along i into T[q][i][y][kz], i the global plane.  FP32: the
//      library's column pass reading its lines from the receive blocks;
//      FP64: the unpack (below) and a strided cuFFT Z2Z;
// and the k-space update (kspace.cuh kspace_update) takes the rank's own
// k-points, (kx, y0 + y, kz), from T with the amplitudes G[4][kx][y][kz].
// Planes (i) and columns (ky) are split over the ranks with one rule:
// rank r owns [p0(r), p0(r) + n(r)), n(r) = N/W + (r < N%W), contiguous.
#pragma once

#include "kspace.cuh"
#include "slabsplit.h"

namespace gabe {


// A row of nz complex values copied by one warp, up to nine loads per lane
// in flight before the stores (one round for nz <= 288).
template <typename T>
__device__ __forceinline__ void row_copy(Cplx<T> *dst, const Cplx<T> *src, int nz, int lane) {
    constexpr int U = 9;
    for (int base = 0; base < nz; base += 32 * U) {
        Cplx<T> v[U];
#pragma unroll
        for (int u = 0; u < U; u++)
            if (base + lane + 32 * u < nz) v[u] = src[base + lane + 32 * u];
#pragma unroll
        for (int u = 0; u < U; u++)
            if (base + lane + 32 * u < nz) dst[base + lane + 32 * u] = v[u];
    }
}

// 2-D transforms of this rank's planes -> send buffer, blocks by destination
// rank r' (offset ncomp nloc nz p0(r') complex), each [ncomp][nloc][n(r')][nz]
// (ncomp = 10 sources, or 2 fields for the spectra).  One warp per row of
// nz values: the row's destination is worked out once, the copy is
// contiguous.
template <typename T>
__global__ void __launch_bounds__(256) slab_gw_pack_kernel(const Cplx<T> *S, Cplx<T> *send, int N, int nloc,
                                                           Split sp, int ncomp) {
    const int nz = N / 2 + 1, lane = threadIdx.x & 31;
    const int rows = ncomp * nloc * N;  // < 2^31 for N <= 512
    const int w0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int row = w0; row < rows; row += nw) {
        const int j = row % N, t = row / N, il = t % nloc, q = t / nloc;
        const int r = sp.owner(j), m = sp.n(r), y = j - sp.p0(r);
        const size_t dst = (size_t)ncomp * nloc * nz * sp.p0(r) + (((size_t)q * nloc + il) * m + y) * nz;
        const size_t src = (size_t)row * nz;
        row_copy(send + dst, S + src, nz, lane);
    }
}

// Receive buffer (blocks by source rank r, offset ncomp m nz p0(r), each
// [ncomp][n(r)][m][nz]) -> T[ncomp][N][m][nz], one warp per row of T.
template <typename T>
__global__ void __launch_bounds__(256) slab_gw_unpack_kernel(const Cplx<T> *recv, Cplx<T> *Tt, int N, int m,
                                                             Split sp, int ncomp) {
    const int nz = N / 2 + 1, lane = threadIdx.x & 31;
    const int rows = ncomp * N * m;
    const int w0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int row = w0; row < rows; row += nw) {
        const int y = row % m, t = row / m, i = t % N, q = t / N;
        const int r = sp.owner(i), nr = sp.n(r), il = i - sp.p0(r);
        const size_t src = (size_t)ncomp * m * nz * sp.p0(r) + (((size_t)q * nr + il) * m + y) * nz;
        const size_t dst = (size_t)row * nz;
        row_copy(Tt + dst, recv + src, nz, lane);
    }
}

// TT projection and both RK2 stages for this rank's k-points (kspace.cuh).
template <typename T>
__global__ void __launch_bounds__(256) slab_kspace_kernel(const Cplx<T> *Tt, Cplx<T> *G, const DevScalars *sc,
                                                          LatticeConsts c, int m, int y0) {
    const int N = c.N, nz = N / 2 + 1;
    const size_t M = (size_t)N * m * nz;
    const KsCoef<T> kc = ks_coef<T>(c, sc->gw[0]);
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % nz);
        const size_t t = idx / nz;
        const int y = (int)(t % m), i = (int)(t / m), j = y0 + y;
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        kspace_update<T>(kc, px, py, kz, M, Tt, G, idx);
    }
}

// Amplitudes -> the reference's 12 components (h or l: which = 0 / 1) for
// points m0 .. m0+cnt-1 of this rank's [N][m][nz] k-points; dst [12][cnt].
template <typename T>
__global__ void slab_gw_unpack_amplitudes_kernel(const Cplx<T> *G, size_t cnt, size_t m0, int N, int m, int y0,
                                                 int which, double *dst) {
    const int nz = N / 2 + 1;
    const size_t M = (size_t)N * m * nz;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
        const size_t idx = m0 + q;
        const int kz = (int)(idx % nz);
        const size_t t = idx / nz;
        const int y = (int)(t % m), i = (int)(t / m), j = y0 + y;
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        double ep[6] = {0, 0, 0, 0, 0, 0}, ex[6] = {0, 0, 0, 0, 0, 0};
        if (px || py || kz) pol_tensors(px, py, kz, ep, ex);
        const Cplx<T> ap = G[(size_t)(2 * which) * M + idx], ax = G[(size_t)(2 * which + 1) * M + idx];
#pragma unroll
        for (int c6 = 0; c6 < 6; c6++) {
            dst[(size_t)(2 * c6) * cnt + q] = ep[c6] * (double)ap.re + ex[c6] * (double)ax.re;
            dst[(size_t)(2 * c6 + 1) * cnt + q] = ep[c6] * (double)ap.im + ex[c6] * (double)ax.im;
        }
    }
}

// host launchers, instantiated by the FP32 and FP64 units
inline unsigned slab_grid(size_t n) { return (unsigned)(n / 256 + 1 < 148 * 8 ? n / 256 + 1 : 148 * 8); }

template <typename T>
cudaError_t slab_gw_pack(const void *S, void *send, int N, int nloc, int W, int ncomp, cudaStream_t s) {
    slab_gw_pack_kernel<T><<<slab_grid((size_t)ncomp * nloc * N * 32), 256, 0, s>>>(
        static_cast<const Cplx<T> *>(S), static_cast<Cplx<T> *>(send), N, nloc, Split(N, W), ncomp);
    return cudaGetLastError();
}
template <typename T>
cudaError_t slab_gw_unpack(const void *recv, void *Tt, int N, int m, int W, int ncomp, cudaStream_t s) {
    slab_gw_unpack_kernel<T><<<slab_grid((size_t)ncomp * N * m * 32), 256, 0, s>>>(
        static_cast<const Cplx<T> *>(recv), static_cast<Cplx<T> *>(Tt), N, m, Split(N, W), ncomp);
    return cudaGetLastError();
}
template <typename T>
cudaError_t slab_kspace(const void *Tt, void *G, const DevScalars *sc, const LatticeConsts &c, int m, int y0,
                        cudaStream_t s) {
    slab_kspace_kernel<T><<<slab_grid((size_t)c.N * m * (c.N / 2 + 1)), 256, 0, s>>>(
        static_cast<const Cplx<T> *>(Tt), static_cast<Cplx<T> *>(G), sc, c, m, y0);
    return cudaGetLastError();
}
template <typename T>
cudaError_t slab_gw_amplitudes(const void *G, size_t cnt, size_t m0, int N, int m, int y0, int which, double *dst,
                               cudaStream_t s) {
    slab_gw_unpack_amplitudes_kernel<T><<<slab_grid(cnt), 256, 0, s>>>(static_cast<const Cplx<T> *>(G), cnt, m0, N, m,
                                                                        y0, which, dst);
    return cudaGetLastError();
}

}  // namespace gabe
