// |k|-binned power spectra (specOut, g2spectra.cpp:23-234).
//
// One pass over the half spectrum accumulates, per native bin
// b = (int)|n| (g2spectra.cpp:74-89), the weighted power of both fields
// (weight 2 for 0 < kz < N/2, 1 on the kz = 0 and kz = N/2 planes) and of
// the GW momenta l with the reference's component weights (:133-144).  With
// gw_spec_quirk the kz = 0 plane reads l at kz = N/2, as the reference's
// loop does (:149-164, k is left at N/2 by the preceding loop).  Sums are
// FP64: per-block shared-memory histograms, then a fixed-order reduction
// over blocks.  Normalisation to the file columns happens on the host.
#pragma once

#include "common.cuh"
#include "kspace.cuh"

namespace gabe {

struct BinArgs {
    const void *F;          // complex field spectra, 2 slots [2][N][N][N/2+1]
    const void *G;          // GW amplitudes [4][N][N][N/2+1] complex (h+, hx, l+, lx) or null
    double *part_sum;       // [nblocks][nseries][nbins]
    unsigned int *part_cnt; // [nblocks][nbins]
    int N, nbins, nseries, quirk;
    double zero_re[2];      // FP32 path: N^3 fbar per field, added to F(k=0) of the fluctuations
    int fix_zero;
    // a slab's k-points (slab.cu): F and G hold [..][N][m][N/2+1] with ky = y0 + y; m = 0: all of them
    int m, y0;
    int gt;                 // G in the transposed order [4][kz][ky][kx] (fftt.cuh); whole lattices only
};

template <typename T>
__global__ void __launch_bounds__(256) bin_kernel(BinArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *hs = reinterpret_cast<double *>(smem_raw);                      // [nseries][nbins]
    unsigned int *hc = reinterpret_cast<unsigned int *>(hs + a.nseries * a.nbins);  // [nbins]
    const int N = a.N, nz = N / 2 + 1, nb = a.nbins, ns = a.nseries;
    const int ny = a.m ? a.m : N;  // ky rows held
    const size_t M = (size_t)N * ny * nz;
    for (int q = threadIdx.x; q < ns * nb; q += blockDim.x) hs[q] = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) hc[q] = 0u;
    __syncthreads();
    const T *F = static_cast<const T *>(a.F);
    const T *G = static_cast<const T *>(a.G);
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = a.y0 + (int)(t % ny), i = (int)(t / ny);
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        const int b = (int)sqrt((double)px * px + (double)py * py + (double)kz * kz);
        const bool edge = (kz == 0) || (kz == N / 2);
        const double w = edge ? 1.0 : 2.0;
        atomicAdd(&hc[b], edge ? 1u : 2u);
        for (int f = 0; f < 2; f++) {
            double re = (double)F[2 * ((size_t)f * M + idx)], im = (double)F[2 * ((size_t)f * M + idx) + 1];
            if (a.fix_zero && idx == 0 && a.y0 == 0) re += a.zero_re[f];  // k = 0
            atomicAdd(&hs[f * nb + b], w * (re * re + im * im));
        }
        if (ns > 2) {
            // sum_ij |l_ij|^2 with the reference's weights (diagonal 1,
            // off-diagonal 2) = 2 (|l+|^2 + |lx|^2) for a TT tensor
            const size_t src = a.gt ? g_index(i, j, (a.quirk && kz == 0) ? N / 2 : kz, N, 1)
                                    : ((a.quirk && kz == 0) ? idx + (size_t)(N / 2) : idx);
            const double pr = (double)G[2 * (2 * M + src)], pi = (double)G[2 * (2 * M + src) + 1];
            const double xr = (double)G[2 * (3 * M + src)], xi = (double)G[2 * (3 * M + src) + 1];
            const double p = 2. * ((pr * pr + pi * pi) + (xr * xr + xi * xi));
            atomicAdd(&hs[2 * nb + b], w * p);
        }
    }
    __syncthreads();
    double *ps = a.part_sum + (size_t)blockIdx.x * ns * nb;
    unsigned int *pc = a.part_cnt + (size_t)blockIdx.x * nb;
    for (int q = threadIdx.x; q < ns * nb; q += blockDim.x) ps[q] = hs[q];
    for (int q = threadIdx.x; q < nb; q += blockDim.x) pc[q] = hc[q];
}

// Fixed-order sum of the block histograms: one thread per (series, bin).
static __global__ void bin_reduce_kernel(const double *part_sum, const unsigned int *part_cnt, int nblocks, int nseries,
                                  int nbins, double *sum, double *cnt) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nseries * nbins) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += part_sum[(size_t)b * nseries * nbins + q];
        sum[q] = s;
    }
    if (q < nbins) {
        unsigned long long n = 0;
        for (int b = 0; b < nblocks; b++) n += part_cnt[(size_t)b * nbins + q];
        cnt[q] = (double)n;
    }
}

}  // namespace gabe
