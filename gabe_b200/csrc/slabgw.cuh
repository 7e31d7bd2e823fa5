// GW branch of a lattice split into slabs along i (slab.cu), FP32 storage.
//
// The 3-D transform of the ten source arrays (fft_stresstensor,
// g2evolutionpert.cpp:183-195) runs as
//   1. a 2-D r2c over (j, k) of every own plane (cuFFT, in place):
//      S[q][il][ky][kz], il < nplanes;
//   2. a transpose between the ranks: rank r' receives the ky columns it
//      owns, [y0_r', y0_r' + m_r'), of every plane -- pack (below), an
//      all-to-all by the caller, unpack (below) into T[q][i][y][kz] with i
//      the global plane;
//   3. the pass along i (fft3d.cuh col_fft_kernel) on T;
// and the k-space update (kspace.cuh kspace_update) takes the rank's own
// k-points, (kx, y0 + y, kz), from T with the amplitudes G[4][kx][y][kz].
// Planes (i) and columns (ky) are split over the ranks with one rule:
// rank r owns [p0(r), p0(r) + n(r)), n(r) = N/W + (r < N%W), contiguous.
#pragma once

#include "kspace.cuh"
#include "slabsplit.h"

namespace gabe {


// A row of nz <= 257 complex values copied by one warp, every load issued
// before the first store (nine per lane in flight).
__device__ __forceinline__ void row_copy(Cplx<float> *dst, const Cplx<float> *src, int nz, int lane) {
    constexpr int U = 9;  // ceil(257 / 32)
    Cplx<float> v[U];
#pragma unroll
    for (int u = 0; u < U; u++)
        if (lane + 32 * u < nz) v[u] = src[lane + 32 * u];
#pragma unroll
    for (int u = 0; u < U; u++)
        if (lane + 32 * u < nz) dst[lane + 32 * u] = v[u];
}

// 2-D transforms of this rank's planes -> send buffer, blocks by destination
// rank r' (offset ncomp nloc nz p0(r') complex), each [ncomp][nloc][n(r')][nz]
// (ncomp = 10 sources, or 2 fields for the spectra).  One warp per row of
// nz values: the row's destination is worked out once, the copy is
// contiguous.
__global__ void __launch_bounds__(256) slab_gw_pack_kernel(const Cplx<float> *S, Cplx<float> *send, int N, int nloc,
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
__global__ void __launch_bounds__(256) slab_gw_unpack_kernel(const Cplx<float> *recv, Cplx<float> *T, int N, int m,
                                                             Split sp, int ncomp) {
    const int nz = N / 2 + 1, lane = threadIdx.x & 31;
    const int rows = ncomp * N * m;
    const int w0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int row = w0; row < rows; row += nw) {
        const int y = row % m, t = row / m, i = t % N, q = t / N;
        const int r = sp.owner(i), nr = sp.n(r), il = i - sp.p0(r);
        const size_t src = (size_t)ncomp * m * nz * sp.p0(r) + (((size_t)q * nr + il) * m + y) * nz;
        const size_t dst = (size_t)row * nz;
        row_copy(T + dst, recv + src, nz, lane);
    }
}

// TT projection and both RK2 stages for this rank's k-points (kspace.cuh).
__global__ void __launch_bounds__(256) slab_kspace_kernel(const Cplx<float> *T, Cplx<float> *G, const DevScalars *sc,
                                                          LatticeConsts c, int m, int y0) {
    const int N = c.N, nz = N / 2 + 1;
    const size_t M = (size_t)N * m * nz;
    const KsCoef<float> kc = ks_coef<float>(c, sc->gw[0]);
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % nz);
        const size_t t = idx / nz;
        const int y = (int)(t % m), i = (int)(t / m), j = y0 + y;
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        kspace_update<float>(kc, px, py, kz, M, T, G, idx);
    }
}

// Amplitudes -> the reference's 12 components (h or l: which = 0 / 1) for
// points m0 .. m0+cnt-1 of this rank's [N][m][nz] k-points; dst [12][cnt].
__global__ void slab_gw_unpack_amplitudes_kernel(const Cplx<float> *G, size_t cnt, size_t m0, int N, int m, int y0,
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
        const Cplx<float> ap = G[(size_t)(2 * which) * M + idx], ax = G[(size_t)(2 * which + 1) * M + idx];
#pragma unroll
        for (int c6 = 0; c6 < 6; c6++) {
            dst[(size_t)(2 * c6) * cnt + q] = ep[c6] * (double)ap.re + ex[c6] * (double)ax.re;
            dst[(size_t)(2 * c6 + 1) * cnt + q] = ep[c6] * (double)ap.im + ex[c6] * (double)ax.im;
        }
    }
}

}  // namespace gabe
