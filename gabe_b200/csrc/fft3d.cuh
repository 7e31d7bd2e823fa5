// FP32 3-D r2c of the GW source arrays in three streaming passes.
//
// The reference transforms each source array with one 3-D r2c FFT
// (fft_stresstensor, g2evolutionpert.cpp:183-195).  Each 512^3 array is
// larger than the chip's on-chip storage, so the transform is three passes
// over HBM, one per axis.  Each pass here is a persistent batched 1-D FFT
// whose global accesses are whole 128-byte lines:
//   pass 1 (row_r2c_kernel): rows along k, N reals -> N/2+1 complex, in
//          place in the N+2 reals of the row.  Two real rows travel as one
//          complex sequence z = x_a + i x_b (four-step FFT in shared memory)
//          and are separated with X_a[k] = (Z[k] + conj Z[N-k]) / 2,
//          X_b[k] = (Z[k] - conj Z[N-k]) / 2i;
//   pass 2 (col_fft_kernel along j) and pass 3 (along i): complex columns of
//          stride nz (resp. N nz); a tile is 16 adjacent columns (16 complex
//          = one 128-byte line per row) of one plane (resp. one row j).
// The layout is that of a library in-place r2c: S[q][i][j][N+2] reals before,
// S[q][kx][ky][kz] complex (kz < N/2+1) after.  Forward sign e^{-i},
// unnormalised (FFTW's convention).  The column passes also run out of place
// (the handle's default: they write a second array faster than their input)
// and, for a lattice split into slabs, straight into and out of the blocks
// of the ranks' transpose (scatter along j, gather along i).
#pragma once

#include "fftreg.cuh"
#include "slabsplit.h"
#include "sweep32.cuh"

namespace gabe {
namespace f3d {

using pfft::FourStep;

constexpr int kFftThreads = 512;
constexpr int kFftBufs = 2;  // tile buffers: copies run one tile ahead (a third buffer measured slower)

// W_N^(n1 k2) for the four-step split N = L1 L2, stored [k2][n1].
template <int N>
__device__ __forceinline__ void twiddles(float2 *tw) {
    constexpr int L1 = FourStep<N>::L1;
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        const int k2 = m / L1, n1 = m % L1;
        double sn, cs;
        sincospi(2.0 * (n1 * k2) / N, &sn, &cs);
        tw[m] = make_float2((float)cs, (float)-sn);
    }
}

// All passes are persistent kernels with a ring of tile buffers in shared
// memory: the copies (cp.async) of the next tile are in flight while the
// current one is transformed, so HBM streams during the FFT arithmetic.

// ---------------------------------------------------------------------------
// pass 1: r2c along k of every row (nrows rows of N+2 reals)
// ---------------------------------------------------------------------------
// 128-thread CTAs, several per SM (one computes while the others' copies
// stream), each with two buffers of R = 16 rows.  Rows land in shared memory
// with 8-byte cp.async copies, unpadded: within each run of L1 reals
// (one four-step chunk) the pairs of reals are permuted by an XOR with the
// chunk's index, so that the stride-L1 reads of the second four-step pass
// fall on distinct banks while every pair stays 8-byte aligned.
template <int N, int R_ = 16, int NB_ = 2, int T_ = 128, int PAD_ = 0>
struct RowGeom {
    using C_ = FourStep<N>;
    static constexpr int L1 = C_::L1, L2 = C_::L2;
    static constexpr int R = R_, P = R / 2, T = T_, NB = NB_;  // rows per tile, pairs, threads, buffers
    static constexpr int PITCH = N + PAD_;                     // floats per shared row
    static constexpr int BUF = R * PITCH;                       // floats per tile buffer
    static constexpr int SMEM_FLOATS = NB * BUF + 2 * N;        // + twiddles
    static constexpr size_t SMEM_BYTES = (size_t)SMEM_FLOATS * sizeof(float);
    static constexpr int NT2 = (P * L2 + T - 1) / T;  // pass-2 tasks per thread
    static_assert(L1 % 2 == 0 && L1 <= 32, "pair swizzle within a chunk of L1 reals");
    // shared position of real e of a row
    __device__ static __forceinline__ int phys(int e) {
        constexpr int CPR = 32 / L1, H = L1 / 2;  // chunks per 32-bank row, pairs per chunk
        const int c = e / L1, q = (e % L1) >> 1;
        return c * L1 + 2 * (q ^ ((c / CPR) % H)) + (e & 1);
    }
};

// Two CTAs per SM at N = 512: without a third CTA's register cap (149) the
// kernel keeps more of each FFT in flight (2.37 against 2.80 ms for ten
// 512^3 arrays, measured on B200 across R = 4 .. 32, 2 .. 4 buffers and
// 1 .. 8 CTAs per SM).
template <int N, int R_ = 16, int NB_ = 2, int MINB = (N >= 512 ? 2 : 3)>
__global__ void __launch_bounds__(RowGeom<N, R_, NB_>::T, MINB) row_r2c_kernel(float *S, long long nrows) {
    using Gm = RowGeom<N, R_, NB_>;
    constexpr int L1 = Gm::L1, L2 = Gm::L2, PITCH = Gm::PITCH, R = Gm::R, P = Gm::P, T = Gm::T, NT2 = Gm::NT2,
                  NB = Gm::NB;
    constexpr int RP = N + 2, NH = N / 2 + 1;
    extern __shared__ __align__(16) float smem[];
    float2 *tw = reinterpret_cast<float2 *>(smem + NB * Gm::BUF);
    const int tid = threadIdx.x;
    twiddles<N>(tw);
    const long long ntiles = nrows / R;
    // rows of tile `tile` into buffer `b`: rows start on 8-byte boundaries (N+2 even)
    auto issue = [&](long long tile, int b) {
        const float *g = S + tile * R * RP;
        float *rows = smem + b * Gm::BUF;
#pragma unroll 4
        for (int t = tid; t < R * (N / 2); t += T) {
            const int jj = t / (N / 2), m = t % (N / 2);
            s32::cp_async8(rows + jj * PITCH + Gm::phys(2 * m), g + jj * RP + 2 * m);
        }
    };
#pragma unroll
    for (int q = 0; q < NB - 1; q++) {
        if (blockIdx.x + q * (long long)gridDim.x < ntiles) issue(blockIdx.x + q * (long long)gridDim.x, q);
        s32::cp_commit();
    }
    int it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        float *rows = smem + (it % NB) * Gm::BUF;
        float *g = S + tile * R * RP;
        s32::cp_wait<NB - 2>();
        __syncthreads();  // this tile landed; the buffer of tile it-1 is consumed
        const long long ahead = tile + (long long)(NB - 1) * gridDim.x;
        if (ahead < ntiles) issue(ahead, (it + NB - 1) % NB);
        s32::cp_commit();
        // four-step pass 1: L2-point FFTs over n2 (stride L1), twiddle W_N^(n1 k2), in place
#pragma unroll
        for (int t0 = 0; t0 < P * L1; t0 += T) {
            const int t = t0 + tid, p = t / L1, n1 = t % L1;
            if (t >= P * L1) break;  // N = 64: fewer tasks than threads
            float *re = rows + 2 * p * PITCH, *im = re + PITCH;
            float2 x[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) {
                const int a = Gm::phys(n1 + L1 * n2);
                x[n2] = make_float2(re[a], im[a]);
            }
            pfft::fft_reg<L2>(x);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) {
                const float2 y = k2 ? pfft::cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
                const int a = Gm::phys(n1 + L1 * k2);
                re[a] = y.x;
                im[a] = y.y;
            }
        }
        __syncthreads();
        // pass 2: L1-point FFTs over n1, written back in natural order k = k2 + L2 k1
        {
            float2 y[NT2][L1];
#pragma unroll
            for (int q = 0; q < NT2; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                if (t < P * L2) {
                    const float *re = rows + 2 * p * PITCH, *im = re + PITCH;
#pragma unroll
                    for (int n1 = 0; n1 < L1; n1++) {
                        const int a = Gm::phys(n1 + L1 * k2);
                        y[q][n1] = make_float2(re[a], im[a]);
                    }
                    pfft::fft_reg<L1>(y[q]);
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < NT2; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                if (t < P * L2) {
                    float *re = rows + 2 * p * PITCH, *im = re + PITCH;
#pragma unroll
                    for (int k1 = 0; k1 < L1; k1++) {
                        const int a = Gm::phys(k2 + L2 * k1);
                        re[a] = y[q][k1].x;
                        im[a] = y[q][k1].y;
                    }
                }
            }
        }
        __syncthreads();
        // separate each pair and write N/2+1 complex values per row
        for (int t = tid; t < P * NH; t += T) {
            const int p = t / NH, k = t % NH, km = (N - k) & (N - 1);
            const float *re = rows + 2 * p * PITCH, *im = re + PITCH;
            const int ak = Gm::phys(k & (N - 1)), am = Gm::phys(km);
            const float zr = re[ak], zi = im[ak], mr = re[am], mi = im[am];
            __stcs(reinterpret_cast<float2 *>(g + (2 * p) * RP) + k, make_float2(0.5f * (zr + mr), 0.5f * (zi - mi)));
            __stcs(reinterpret_cast<float2 *>(g + (2 * p + 1) * RP) + k,
                   make_float2(0.5f * (zi + mi), 0.5f * (mr - zr)));
        }
    }
    s32::cp_wait<0>();
}

// ---------------------------------------------------------------------------
// passes 2 and 3: forward C2C along a strided axis
// ---------------------------------------------------------------------------
// Lines: for b1 < n1, b2 < n2 and column c < ncol the N values at
// base + b1 s1 + b2 s2 + n sn + c (complex units).
struct ColArgs {
    float2 *X;
    long long s1, s2, sn;
    int n1, n2, ncol;
    // Forms for a lattice split into slabs (slabgw.cuh), r the owner of
    // index n among `ranks` ranks:
    // gather (kColGather), the pass along i: the lines are read from the
    // receive buffer of the transpose, blocks by source rank of
    // [n1][n(r)][..] with the plane stride sn -- value n of line (b1, b2) at
    // src + (n1 p0(r) + n - p0(r) + b1 n(r)) sn + b2 s2 -- and written to X;
    // scatter (kColScatter), the pass along j (n2 = 1): lines read from X,
    // output value n of line b1 written to the send buffer of the transpose,
    // blocks by destination rank of [n1][n(r)][ncol], at
    // dst + (n1 p0(r) + n - p0(r) + b1 n(r)) ncol.
    // out of place (kColOutOfPlace): the lines are read from src with X's
    // layout and written to X.
    const float2 *src = nullptr;
    float2 *dst = nullptr;
    int ranks = 0;
};

constexpr int kColInPlace = 0, kColGather = 1, kColScatter = 2, kColOutOfPlace = 3;

template <int N, int T_ = kFftThreads>
struct ColGeom {
    static constexpr int L1 = FourStep<N>::L1, L2 = FourStep<N>::L2;
    static constexpr int W = 16, T = T_;  // columns per tile, threads
    static constexpr int BUF = N * W;                // complex per tile buffer
    static constexpr int SMEM_C = kFftBufs * BUF + N;  // tile ring + twiddles (complex)
    static constexpr size_t SMEM_BYTES = (size_t)SMEM_C * sizeof(float2);
    static constexpr size_t SMEM_BYTES_SLAB = SMEM_BYTES + 2 * N * sizeof(long long);  // + per-index offsets
};

template <int N, int MODE = kColInPlace, int T_ = kFftThreads>
__global__ void __launch_bounds__(T_, 1) col_fft_kernel(ColArgs a) {
    using Gm = ColGeom<N, T_>;
    constexpr int L1 = Gm::L1, L2 = Gm::L2, W = Gm::W, T = Gm::T;
    extern __shared__ __align__(16) float2 cs[];
    float2 *tw = cs + kFftBufs * Gm::BUF;  // [k2][n1]
    // slab forms: offset of index n for b1 = 0 and its growth per b1
    long long *goff = reinterpret_cast<long long *>(tw + N), *gq = goff + N;
    const int tid = threadIdx.x;
    twiddles<N>(tw);
    if constexpr (MODE == kColGather || MODE == kColScatter) {
        const Split sp(N, a.ranks);
        const long long unit = MODE == kColGather ? a.sn : (long long)a.ncol;
        for (int n = tid; n < N; n += T) {
            const int r = sp.owner(n), p0 = sp.p0(r);
            goff[n] = ((long long)a.n1 * p0 + (n - p0)) * unit;
            gq[n] = (long long)sp.n(r) * unit;
        }
        __syncthreads();  // the offsets are read by the first copies
    }
    const int ncb = (a.ncol + W - 1) / W;
    const long long ntiles = (long long)a.n1 * a.n2 * ncb;
    auto tile_base = [&](long long tile, int &wn) {
        const int cb = (int)(tile % ncb);
        const long long b = tile / ncb;
        const int b2 = (int)(b % a.n2), b1 = (int)(b / a.n2);
        wn = min(W, a.ncol - cb * W);  // columns in this tile
        return a.X + b1 * a.s1 + b2 * a.s2 + cb * W;
    };
    auto issue = [&](long long tile, int b) {
        int wn;
        const float2 *base = tile_base(tile, wn);
        float2 *col = cs + b * Gm::BUF;
        if constexpr (MODE == kColGather) {
            const int cb = (int)(tile % ncb);
            const long long bb = tile / ncb;
            const int b2 = (int)(bb % a.n2), b1 = (int)(bb / a.n2);
            const float2 *g = a.src + b2 * a.s2 + cb * W;
            for (int t = tid; t < N * W; t += T) {
                const int n = t / W, w = t % W;
                if (w < wn) s32::cp_async8(col + t, g + goff[n] + b1 * gq[n] + w);
            }
        } else {
            const float2 *rb = MODE == kColOutOfPlace ? a.src + (base - a.X) : base;
            for (int t = tid; t < N * W; t += T) {
                const int n = t / W, w = t % W;
                if (w < wn) s32::cp_async8(col + t, rb + n * a.sn + w);
            }
        }
    };
#pragma unroll
    for (int q = 0; q < kFftBufs - 1; q++) {
        if (blockIdx.x + q * (long long)gridDim.x < ntiles) issue(blockIdx.x + q * (long long)gridDim.x, q);
        s32::cp_commit();
    }
    int it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        float2 *col = cs + (it % kFftBufs) * Gm::BUF;
        int wn;
        float2 *base = tile_base(tile, wn);
        s32::cp_wait<kFftBufs - 2>();
        __syncthreads();  // this tile landed; the buffer of tile it-1 is consumed
        const long long ahead = tile + (long long)(kFftBufs - 1) * gridDim.x;
        if (ahead < ntiles) issue(ahead, (it + kFftBufs - 1) % kFftBufs);
        s32::cp_commit();
        // four-step pass 1: L2-point FFTs over n2, twiddle, in place
        for (int t = tid; t < W * L1; t += T) {
            const int w = t % W, n1 = t / W;
            float2 x[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) x[n2] = col[(n1 + L1 * n2) * W + w];
            pfft::fft_reg<L2>(x);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) col[(n1 + L1 * k2) * W + w] = k2 ? pfft::cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
        }
        __syncthreads();
        // pass 2: L1-point FFTs over n1, straight to HBM in natural order
        for (int t = tid; t < W * L2; t += T) {
            const int w = t % W, k2 = t / W;
            float2 y[L1];
#pragma unroll
            for (int n1 = 0; n1 < L1; n1++) y[n1] = col[(n1 + L1 * k2) * W + w];
            pfft::fft_reg<L1>(y);
            if (w < wn) {
                if constexpr (MODE == kColScatter) {
                    const int cb = (int)(tile % ncb);
                    const long long b1 = tile / ncb / a.n2;
                    float2 *g = a.dst + cb * W + w;
#pragma unroll
                    for (int k1 = 0; k1 < L1; k1++) {
                        const int k = k2 + L2 * k1;
                        __stcs(g + goff[k] + b1 * gq[k], y[k1]);
                    }
                } else {
#pragma unroll
                    for (int k1 = 0; k1 < L1; k1++) __stcs(base + (k2 + L2 * k1) * a.sn + w, y[k1]);
                }
            }
        }
    }
    s32::cp_wait<0>();
}

}  // namespace f3d
}  // namespace gabe
