// FP32 transforms of the GW sources without cuFFT's 3-D plan.
//
// The reference transforms each of its source arrays with one 3-D r2c FFT
// (fft_stresstensor, g2evolutionpert.cpp:183-195).  A 3-D FFT of an N^3 array
// that does not fit on chip costs at least one HBM round trip per pass; a
// library plan makes three (r2c along k, then j, then i).  Here the first two
// are one kernel and the third is fused into the k-space update
// (kspace_fused.cuh), so the sources make one round trip less and the
// partially transformed data is read exactly once by the TT projection.
//
// plane_r2c_kernel: a 2-D r2c over the (j, k) plane of every (source, i).
// One thread-block cluster of CS CTAs owns one plane at a time (persistent
// loop over planes); CTA r of the cluster holds rows j in [r R, r R + R),
// R = N / CS, in shared memory.
//   1. rows: pairs of real rows (2p, 2p+1) form one complex sequence
//      z = x_2p + i x_2p+1 of length N, transformed in shared memory by a
//      four-step FFT (N = L1 L2: L2-point FFTs in registers, twiddles
//      W_N^(n1 k2), L1-point FFTs in registers);
//   2. exchange: after a cluster barrier every CTA reads, through distributed
//      shared memory, the columns kz in [r C, r C + C) (C = N / (2 CS)) of all
//      N rows from the CTAs that hold them, separating each pair with
//      X_2p[kz] = (Z[kz] + conj Z[N-kz]) / 2,
//      X_2p+1[kz] = (Z[kz] - conj Z[N-kz]) / 2i.
//      The kz = 0 and kz = N/2 values of a row are real, so they travel as
//      one packed complex column X[0] + i X[N/2];
//   3. columns: the same four-step FFT along j; the packed column is split
//      into its two Hermitian halves, A[ky] = (W[ky] + conj W[-ky]) / 2 and
//      B[ky] = (W[ky] - conj W[-ky]) / 2i, which are the kz = 0 and kz = N/2
//      columns;
//   4. the result goes back in place in the layout a library r2c leaves:
//      rows of N/2+1 complex values in the N+2 reals of the input row.
// Conventions are FFTW's: forward sign e^{-i}, unnormalised.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace gabe {
namespace pfft {

// cos(pi m / 16) for m = 0..8 (the real parts of the 32nd roots of unity).
constexpr double kCos16[9] = {1.0,
                              0.98078528040323044913,
                              0.92387953251128675613,
                              0.83146961230254523708,
                              0.70710678118654752440,
                              0.55557023301960222474,
                              0.38268343236508977173,
                              0.19509032201612826785,
                              0.0};
__host__ __device__ constexpr double cos32(int m) {
    m &= 31;
    if (m > 16) m = 32 - m;
    return m <= 8 ? kCos16[m] : -kCos16[16 - m];
}
__host__ __device__ constexpr double sin32(int m) { return cos32(8 - m); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// v * W_32^M, W_32 = exp(-2 pi i / 32), with M known at compile time.
template <int M>
__device__ __forceinline__ float2 mulw(float2 v) {
    constexpr int m = M & 31;
    if constexpr (m == 0) {
        return v;
    } else if constexpr (m == 8) {
        return make_float2(v.y, -v.x);
    } else if constexpr (m == 16) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (m == 24) {
        return make_float2(-v.y, v.x);
    } else {
        constexpr float c = (float)cos32(m), s = (float)sin32(m);
        return make_float2(v.x * c + v.y * s, v.y * c - v.x * s);
    }
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
__host__ __device__ constexpr int bitrev(int x, int bits) {
    int r = 0;
    for (int b = 0; b < bits; b++) r = (r << 1) | ((x >> b) & 1);
    return r;
}

template <int R, int I>
__device__ __forceinline__ void bitrev_swap(float2 (&x)[R]) {
    if constexpr (I < R) {
        constexpr int J = bitrev(I, ilog2(R));
        if constexpr (J > I) {
            const float2 t = x[I];
            x[I] = x[J];
            x[J] = t;
        }
        bitrev_swap<R, I + 1>(x);
    }
}

template <int R, int LEN, int J>
__device__ __forceinline__ void butterflies(float2 (&x)[R]) {
    if constexpr (J < LEN / 2) {
#pragma unroll
        for (int i = 0; i < R; i += LEN) {
            const float2 u = x[i + J], v = mulw<J * (32 / LEN)>(x[i + J + LEN / 2]);
            x[i + J] = cadd(u, v);
            x[i + J + LEN / 2] = csub(u, v);
        }
        butterflies<R, LEN, J + 1>(x);
    }
}

template <int R, int LEN>
__device__ __forceinline__ void stages(float2 (&x)[R]) {
    if constexpr (LEN <= R) {
        butterflies<R, LEN, 0>(x);
        stages<R, 2 * LEN>(x);
    }
}

// In-register forward DFT of R <= 32 points, natural order in and out
// (radix-2 decimation in time).
template <int R>
__device__ __forceinline__ void fft_reg(float2 (&x)[R]) {
    static_assert(R >= 2 && R <= 32 && (R & (R - 1)) == 0, "R must be a power of two in [2, 32]");
    bitrev_swap<R, 0>(x);
    stages<R, 2>(x);
}

// Per-N configuration: cluster size, four-step split N = L1 L2, shared-memory
// padding (one float every G) and row pitch, chosen so that the strided
// accesses of both four-step passes hit distinct banks.
template <int N>
struct PlaneCfg;
template <>
struct PlaneCfg<512> {
    static constexpr int CS = 16, L1 = 32, L2 = 16, G = 32, PITCH = 536;
};
template <>
struct PlaneCfg<256> {
    static constexpr int CS = 4, L1 = 16, L2 = 16, G = 16, PITCH = 280;
};
template <>
struct PlaneCfg<128> {
    static constexpr int CS = 2, L1 = 16, L2 = 8, G = 16, PITCH = 140;
};
template <>
struct PlaneCfg<64> {
    static constexpr int CS = 1, L1 = 8, L2 = 8, G = 8, PITCH = 76;
};

constexpr int kPlaneThreads = 256;

template <int N>
struct PlaneGeom {
    using C_ = PlaneCfg<N>;
    static constexpr int CS = C_::CS, L1 = C_::L1, L2 = C_::L2, G = C_::G, PITCH = C_::PITCH;
    static constexpr int R = N / CS;        // rows per CTA
    static constexpr int P = R / 2;         // row pairs per CTA
    static constexpr int C = N / (2 * CS);  // packed columns per CTA
    static constexpr int T = kPlaneThreads;
    static constexpr int ROW_FLOATS = R * PITCH;
    static constexpr int SMEM_FLOATS = ROW_FLOATS + 2 * N;  // + twiddle table
    static constexpr size_t SMEM_BYTES = (size_t)SMEM_FLOATS * sizeof(float);
    static_assert(L1 * L2 == N, "four-step split");
    static_assert(2 * N * C <= ROW_FLOATS, "column data fits the row buffer");
    static_assert((P * L1) % T == 0 && (P * L2) % T == 0, "row passes divide over the threads");
    static_assert((C * L1) % T == 0 && (C * L2) % T == 0, "column passes divide over the threads");
    static_assert(((N / 2) * C) % T == 0 && (R * (N / 2)) % T == 0, "exchange and load divide over the threads");
    __device__ static __forceinline__ int pad(int s) { return s + s / G; }
};

template <int N>
__global__ void __launch_bounds__(kPlaneThreads, 3) plane_r2c_kernel(float *S, int nplanes) {
    namespace cg = cooperative_groups;
    using Gm = PlaneGeom<N>;
    constexpr int CS = Gm::CS, L1 = Gm::L1, L2 = Gm::L2, PITCH = Gm::PITCH, R = Gm::R, P = Gm::P, C = Gm::C,
                  T = Gm::T;
    constexpr int RP = N + 2;  // reals per row in HBM
    extern __shared__ __align__(16) float smem[];
    float *rows = smem;                                            // [R][PITCH] real rows, padded
    float2 *col = reinterpret_cast<float2 *>(smem);                // [N][C] complex columns (aliases rows)
    float2 *tw = reinterpret_cast<float2 *>(smem + Gm::ROW_FLOATS);  // [k2][n1]: W_N^(n1 k2)

    cg::cluster_group cluster = cg::this_cluster();
    const int r = (int)cluster.block_rank();
    const int tid = threadIdx.x;
    const int cid = blockIdx.x / CS, ncl = gridDim.x / CS;

    // stored as [k2][n1] so that lanes (consecutive n1) read consecutive words
    for (int m = tid; m < N; m += T) {
        const int k2 = m / L1, n1 = m % L1;
        double sn, cs;
        sincospi(2.0 * (n1 * k2) / N, &sn, &cs);
        tw[m] = make_float2((float)cs, (float)-sn);
    }

    for (int pl = cid; pl < nplanes; pl += ncl) {
        float *plane = S + (size_t)pl * N * RP;
        __syncthreads();  // previous plane's shared data fully consumed; twiddles ready
        // ---- load rows r R .. r R + R - 1 ----
        {
            constexpr int NL = R * (N / 2) / T, BL = NL < 16 ? NL : 16;  // loads in flight per batch
            static_assert(NL % BL == 0, "load batches");
#pragma unroll
            for (int b = 0; b < NL; b += BL) {
                float2 v[BL];
#pragma unroll
                for (int q = 0; q < BL; q++) {
                    const int t = (b + q) * T + tid, jj = t / (N / 2), m = t % (N / 2);
                    v[q] = __ldcs(reinterpret_cast<const float2 *>(plane + (size_t)(r * R + jj) * RP) + m);
                }
#pragma unroll
                for (int q = 0; q < BL; q++) {
                    const int t = (b + q) * T + tid, jj = t / (N / 2), m = t % (N / 2);
                    float *dst = rows + jj * PITCH + Gm::pad(2 * m);
                    dst[0] = v[q].x;
                    dst[1] = v[q].y;
                }
            }
        }
        __syncthreads();
        // ---- row pass 1: L2-point FFTs over n2, twiddle W_N^(n1 k2) ----
#pragma unroll
        for (int t0 = 0; t0 < P * L1; t0 += T) {
            const int t = t0 + tid, p = t / L1, n1 = t % L1;
            float *re = rows + 2 * p * PITCH, *im = re + PITCH;
            float2 x[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) {
                const int a = Gm::pad(n1 + L1 * n2);
                x[n2] = make_float2(re[a], im[a]);
            }
            fft_reg<L2>(x);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) {
                const float2 y = k2 ? cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
                const int a = Gm::pad(n1 + L1 * k2);
                re[a] = y.x;
                im[a] = y.y;
            }
        }
        __syncthreads();
        // ---- row pass 2: L1-point FFTs over n1, result in natural order ----
        {
            constexpr int NT = P * L2 / T;
            float2 y[NT][L1];
#pragma unroll
            for (int q = 0; q < NT; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                const float *re = rows + 2 * p * PITCH, *im = re + PITCH;
#pragma unroll
                for (int n1 = 0; n1 < L1; n1++) {
                    const int a = Gm::pad(n1 + L1 * k2);
                    y[q][n1] = make_float2(re[a], im[a]);
                }
                fft_reg<L1>(y[q]);
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < NT; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                float *re = rows + 2 * p * PITCH, *im = re + PITCH;
#pragma unroll
                for (int k1 = 0; k1 < L1; k1++) {
                    const int a = Gm::pad(k2 + L2 * k1);
                    re[a] = y[q][k1].x;
                    im[a] = y[q][k1].y;
                }
            }
        }
        cluster.sync();  // every CTA's row spectra are complete
        // ---- exchange: columns r C .. r C + C - 1 of all N rows ----
        {
            constexpr int NE = (N / 2) * C / T;
            float2 xe[NE][2];  // 2 NE complex values per thread stay in registers across the barrier
            // raw Z[kz] (xe[q][0]) and Z[N-kz] (xe[q][1]) of every task in flight at once; for
            // kz = 0 the partner is Z[N/2], the other real value of the packed column
#pragma unroll
            for (int q = 0; q < NE; q++) {
                const int t = q * T + tid, g = t / C, c = t % C;
                const int s = (2 * g) / R, p = g - s * P;
                const float *rre = cluster.map_shared_rank(rows, s) + 2 * p * PITCH;
                const float *rim = rre + PITCH;
                const int kz = r * C + c, km = kz == 0 ? N / 2 : N - kz;
                xe[q][0] = make_float2(rre[Gm::pad(kz)], rim[Gm::pad(kz)]);
                xe[q][1] = make_float2(rre[Gm::pad(km)], rim[Gm::pad(km)]);
            }
#pragma unroll
            for (int q = 0; q < NE; q++) {
                const int t = q * T + tid, c = t % C;
                const float zr = xe[q][0].x, zi = xe[q][0].y, mr = xe[q][1].x, mi = xe[q][1].y;
                if (r * C + c == 0) {
                    xe[q][0] = make_float2(zr, mr);
                    xe[q][1] = make_float2(zi, mi);
                } else {
                    xe[q][0] = make_float2(0.5f * (zr + mr), 0.5f * (zi - mi));
                    xe[q][1] = make_float2(0.5f * (zi + mi), 0.5f * (mr - zr));
                }
            }
            cluster.sync();  // all remote reads of this plane's rows are done
#pragma unroll
            for (int q = 0; q < NE; q++) {
                const int t = q * T + tid, g = t / C, c = t % C;
                col[(2 * g) * C + c] = xe[q][0];
                col[(2 * g + 1) * C + c] = xe[q][1];
            }
        }
        __syncthreads();
        // ---- column pass 1 ----
#pragma unroll
        for (int t0 = 0; t0 < C * L1; t0 += T) {
            const int t = t0 + tid, n1 = t / C, c = t % C;
            float2 x[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) x[n2] = col[(n1 + L1 * n2) * C + c];
            fft_reg<L2>(x);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) col[(n1 + L1 * k2) * C + c] = k2 ? cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
        }
        __syncthreads();
        // ---- column pass 2, straight to HBM ----
#pragma unroll
        for (int t0 = 0; t0 < C * L2; t0 += T) {
            const int t = t0 + tid, k2 = t / C, c = t % C;
            float2 y[L1];
#pragma unroll
            for (int n1 = 0; n1 < L1; n1++) y[n1] = col[(n1 + L1 * k2) * C + c];
            fft_reg<L1>(y);
            const int kz = r * C + c;
            if (kz == 0) {  // packed column: back in place (slot k1 + L1 k2 holds ky = k2 + L2 k1)
#pragma unroll
                for (int k1 = 0; k1 < L1; k1++) col[(k1 + L1 * k2) * C] = y[k1];
            } else {
#pragma unroll
                for (int k1 = 0; k1 < L1; k1++)
                    __stcs(reinterpret_cast<float2 *>(plane + (size_t)(k2 + L2 * k1) * RP + 2 * kz), y[k1]);
            }
        }
        if (r == 0) {
            __syncthreads();
            for (int ky = tid; ky < N; ky += T) {
                const int km = (N - ky) & (N - 1);
                const float2 w = col[((ky / L2) + L1 * (ky % L2)) * C], wm = col[((km / L2) + L1 * (km % L2)) * C];
                float *row = plane + (size_t)ky * RP;
                __stcs(reinterpret_cast<float2 *>(row), make_float2(0.5f * (w.x + wm.x), 0.5f * (w.y - wm.y)));
                __stcs(reinterpret_cast<float2 *>(row + N), make_float2(0.5f * (w.y + wm.y), 0.5f * (wm.x - w.x)));
            }
        }
    }
}

}  // namespace pfft
}  // namespace gabe
