// Spectra emulator: MLP forward, backward and AdamW as hand-written kernels
// (include/gabe_mlp.h).  No counterpart in the reference.
//
// One tiled GEMM kernel serves the three products of every layer
// (activations X [B][K], weights W [K][N], pre-activations Z [B][N]):
//
//   forward       Z  = X W + b          M=B, N=N, K=K      epilogue: bias, SiLU, store Z and H
//   data grad     dX = (dZ W^T) * SiLU'(Z_prev)            M=B, N=K, K=N
//   weight grad   dW = X^T dZ                              M=K, N=N, K=B
//
// Operands are addressed through (row, column) strides, so transposes cost
// nothing but coalescing.  64x64 output tiles, 16-deep k slices in shared
// memory, 4x4 outputs per thread, FP32 FMA accumulation.  Activations are
// read as BF16 (or FP32) and widened on the way into shared memory; weights
// are FP32.  With BF16 activations the forward of every layer after the
// first runs on tensor cores instead (tc::gemm_tc_kernel, BF16 weight
// copies); the first layer (a handful of inputs) and the backward products
// stay on this kernel.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/gabe.h"
#include "../../include/gabe_mlp.h"
#include "umma.cuh"

namespace {

using bf16 = __nv_bfloat16;

template <typename T>
__device__ __forceinline__ float ldf(const T *p, long long i);
template <>
__device__ __forceinline__ float ldf<float>(const float *p, long long i) { return p[i]; }
template <>
__device__ __forceinline__ float ldf<bf16>(const bf16 *p, long long i) { return __bfloat162float(p[i]); }

template <typename T>
__device__ __forceinline__ T cvt(float v);
template <>
__device__ __forceinline__ float cvt<float>(float v) { return v; }
template <>
__device__ __forceinline__ bf16 cvt<bf16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
// SiLU of the forward epilogues of the first-layer and tcgen05 kernels:
// the fast exponential and division intrinsics (two special-function
// operations per value, a few ulp of FP32, far below the BF16 rounding of
// the stored activations), since the accurate expf and IEEE division
// bounded those epilogues (608 against 185 us per 1M-row hidden layer).
// A reciprocal by Newton-Raphson steps on the FMA pipe instead of the
// second special-function operation measured slower (225 us): the
// epilogue is bound by issue as much as by that pipe.  z -> -inf gives 0,
// z -> +inf gives z.
__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigmoid(z);
    return s * (1.f + z * (1.f - s));
}

enum Epi { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_BWD_DATA = 2, EPI_BWD_WEIGHT = 3 };

struct GemmArgs {
    int M, N, K;
    const void *A;
    long long sam, sak;  // A(m, k) = A[m * sam + k * sak]
    const float *B;
    long long sbk, sbn;  // B(k, n) = B[k * sbk + n * sbn]
    const float *bias;   // EPI_HIDDEN, EPI_OUT
    void *Z;             // EPI_HIDDEN: pre-activation out (may be null); EPI_BWD_DATA: pre-activation in
    void *C;             // H (activation type), Y, dX or dW (FP32)
    long long ldc;
    int kchunk;          // EPI_BWD_WEIGHT: k range of split blockIdx.z (a multiple of BK)
    float *dbp;          // EPI_BWD_WEIGHT: column sums of B per split ([splits][N])
};

constexpr int BM = 64, BN = 64, BK = 16, kThreads = 256;

// TA: type of A; TACT: activation storage type (Z/H of the epilogues).
template <typename TA, typename TACT, int EPI>
__global__ void __launch_bounds__(kThreads) gemm_kernel(GemmArgs g) {
    __shared__ __align__(16) float As[BK][BM];
    __shared__ __align__(16) float Bs[BK][BN];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const TA *A = static_cast<const TA *>(g.A);
    float acc[4][4] = {};
    // split-K (weight gradient): this block sums k in [kb, ke) and writes
    // its partial product to slice blockIdx.z of the output
    const int kb = EPI == EPI_BWD_WEIGHT ? blockIdx.z * g.kchunk : 0;
    const int ke = EPI == EPI_BWD_WEIGHT ? min(g.K, kb + g.kchunk) : g.K;
    float csum = 0.f;  // EPI_BWD_WEIGHT, first row of tiles: column sums of B (the bias gradient)
    for (int k0 = kb; k0 < ke; k0 += BK) {
        // A tile: 64 (m) x 16 (k); each thread 4 elements along the
        // operand's contiguous direction
        if (g.sak == 1) {
            const int m = tid / 4, kk = (tid % 4) * 4;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int gm = m0 + m, gk = k0 + kk + q;
                As[kk + q][m] = (gm < g.M && gk < ke) ? ldf(A, gm * g.sam + gk) : 0.f;
            }
        } else {
            const int kk = tid / 16, m = (tid % 16) * 4;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int gm = m0 + m + q, gk = k0 + kk;
                As[kk][m + q] = (gm < g.M && gk < ke) ? ldf(A, gm * g.sam + gk * g.sak) : 0.f;
            }
        }
        // B tile: 16 (k) x 64 (n)
        if (g.sbn == 1) {
            const int kk = tid / 16, n = (tid % 16) * 4;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int gk = k0 + kk, gn = n0 + n + q;
                Bs[kk][n + q] = (gk < ke && gn < g.N) ? g.B[gk * g.sbk + gn] : 0.f;
            }
        } else {
            const int n = tid / 4, kk = (tid % 4) * 4;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int gk = k0 + kk + q, gn = n0 + n;
                Bs[kk + q][n] = (gk < ke && gn < g.N) ? g.B[gk + gn * g.sbn] : 0.f;
            }
        }
        __syncthreads();
        if (EPI == EPI_BWD_WEIGHT && blockIdx.y == 0 && tid < BN) {
#pragma unroll
            for (int kk = 0; kk < BK; kk++) csum += Bs[kk][tid];
        }
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            const float4 a = *reinterpret_cast<const float4 *>(&As[kk][ty * 4]);
            const float4 b = *reinterpret_cast<const float4 *>(&Bs[kk][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    if (EPI == EPI_BWD_WEIGHT && blockIdx.y == 0 && tid < BN && n0 + tid < g.N)
        g.dbp[(long long)blockIdx.z * g.N + n0 + tid] = csum;
    float *Cz = static_cast<float *>(g.C) + (EPI == EPI_BWD_WEIGHT ? (long long)blockIdx.z * g.M * g.ldc : 0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + ty * 4 + i;
        if (m >= g.M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + tx * 4 + j;
            if (n >= g.N) continue;
            const long long o = (long long)m * g.ldc + n;
            const float v = acc[i][j];
            if (EPI == EPI_HIDDEN) {
                const float z = v + g.bias[n];
                if (g.Z) static_cast<TACT *>(g.Z)[o] = cvt<TACT>(z);
                static_cast<TACT *>(g.C)[o] = cvt<TACT>(silu(z));
            } else if (EPI == EPI_OUT) {
                static_cast<float *>(g.C)[o] = v + g.bias[n];
            } else if (EPI == EPI_BWD_DATA) {
                static_cast<float *>(g.C)[o] = v * dsilu(ldf(static_cast<const TACT *>(g.Z), o));
            } else {
                Cz[o] = v;
            }
        }
    }
}

// Forward of the first layer (NIN <= 8 inputs): z = x W0 + b0, h = SiLU(z),
// the sum over k in order as the tiled kernel forms it.  A row is made by
// G = N / 8 consecutive threads (G divides the block), 8 consecutive
// outputs each, so every store is a whole 16-byte (BF16) or 32-byte (FP32)
// piece of a coalesced row.  Each thread keeps its 8 columns of W0 and b0
// in registers for all its rows (a reload per row held the loads' queue
// full) and makes RPT rows per pass, their inputs loaded together, so that
// RPT loads are in flight instead of one (one row per pass left the kernel
// bound by the inputs' load latency).
constexpr int kFirstMaxIn = 8, kFirstRows = 4;

template <typename TACT, int NIN>
__global__ void __launch_bounds__(256) first_layer_kernel(const float *x, int rows, const float *W, const float *b,
                                                          int N, TACT *H, TACT *Z) {
    constexpr int RPT = kFirstRows;
    const int G = N / 8, rpb = 256 / G;  // threads per row, rows per block pass
    const int n0 = (threadIdx.x % G) * 8;
    float w[NIN][8], bias[8];
#pragma unroll
    for (int k = 0; k < NIN; k++)
#pragma unroll
        for (int j = 0; j < 8; j++) w[k][j] = W[(long long)k * N + n0 + j];
#pragma unroll
    for (int j = 0; j < 8; j++) bias[j] = b[n0 + j];
    const long long stride = (long long)gridDim.x * rpb;
    for (long long r0 = (long long)blockIdx.x * rpb + threadIdx.x / G; r0 < rows; r0 += RPT * stride) {
        float xv[RPT][NIN];
#pragma unroll
        for (int q = 0; q < RPT; q++) {
            const long long r = r0 + q * stride;
#pragma unroll
            for (int k = 0; k < NIN; k++) xv[q][k] = r < rows ? x[r * NIN + k] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < RPT; q++) {
            const long long r = r0 + q * stride;
            if (r >= rows) break;
            float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < NIN; k++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[j] = fmaf(xv[q][k], w[k][j], acc[j]);
            TACT hv[8], zv[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const float z = acc[j] + bias[j];
                hv[j] = cvt<TACT>(silu_fast(z));
                zv[j] = cvt<TACT>(z);
            }
            constexpr int V = 8 * sizeof(TACT) / 16;  // 16-byte pieces per thread
            const uint4 *hs = reinterpret_cast<const uint4 *>(hv), *zs = reinterpret_cast<const uint4 *>(zv);
            uint4 *ho = reinterpret_cast<uint4 *>(H + r * N + n0);
#pragma unroll
            for (int u = 0; u < V; u++) ho[u] = hs[u];
            if (Z) {
                uint4 *zo = reinterpret_cast<uint4 *>(Z + r * N + n0);
#pragma unroll
                for (int u = 0; u < V; u++) zo[u] = zs[u];
            }
        }
    }
}

template <typename TACT, int NIN>
void launch_first(const float *x, int rows, const float *W, const float *b, int N, TACT *H, TACT *Z,
                  cudaStream_t s) {
    const int rpb = 256 / (N / 8);
    const long long blocks = ((long long)rows + (long long)rpb * kFirstRows - 1) / ((long long)rpb * kFirstRows);
    const int grid = (int)(blocks < 148 * 8 ? blocks : 148 * 8);
    first_layer_kernel<TACT, NIN><<<grid, 256, 0, s>>>(x, rows, W, b, N, H, Z);
}

template <typename TACT>
void launch_first_n(int n_in, const float *x, int rows, const float *W, const float *b, int N, TACT *H, TACT *Z,
                    cudaStream_t s) {
    switch (n_in) {
        case 1: return launch_first<TACT, 1>(x, rows, W, b, N, H, Z, s);
        case 2: return launch_first<TACT, 2>(x, rows, W, b, N, H, Z, s);
        case 3: return launch_first<TACT, 3>(x, rows, W, b, N, H, Z, s);
        case 4: return launch_first<TACT, 4>(x, rows, W, b, N, H, Z, s);
        case 5: return launch_first<TACT, 5>(x, rows, W, b, N, H, Z, s);
        case 6: return launch_first<TACT, 6>(x, rows, W, b, N, H, Z, s);
        case 7: return launch_first<TACT, 7>(x, rows, W, b, N, H, Z, s);
        default: return launch_first<TACT, 8>(x, rows, W, b, N, H, Z, s);
    }
}

// ---------------------------------------------------------------------------
// Tensor-core forward of the layers fed by BF16 activations (all but the
// first): Z = H W + b with H [M][K] BF16 and the layer's weights as a BF16
// copy kept transposed, Wt [N][K] (k contiguous), multiplied by
// mma.sync.m16n8k16 (BF16 x BF16, FP32 accumulation).  128 x 128 output
// tiles, 8 warps of 64 x 32, 32-deep k slices in a 4-stage cp.async ring,
// fragments by ldmatrix; rows padded to 40 BF16 so that the eight 16-byte
// rows of each ldmatrix hit distinct banks.
// Epilogue as the SIMT kernel's: bias and SiLU into Z and H (BF16), or bias
// into the FP32 output.
// ---------------------------------------------------------------------------
namespace tc {

constexpr int BM = 128, BN = 128, BK = 32, LDS = BK + 8, T = 256;

struct Args {
    int M, N, K;
    const bf16 *A;    // [M][K]
    const bf16 *Wt;   // [N][K]
    const float *bias;
    bf16 *Z;          // EPI_HIDDEN: pre-activation (may be null)
    void *C;          // EPI_HIDDEN: H (BF16); EPI_OUT: y (FP32), [M][N]
};

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(void *s, const void *g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr(s)), "l"(g) : "memory");
}

__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(saddr(p)));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared memory: STAGES ring slots of one 128 x 32 A tile and one 128 x 32
// Wt tile; slices k0 + BK (STAGES - 1) ahead are in flight while slice k0
// is multiplied, so global latency hides behind three slices of MMAs.
constexpr int STAGES = 4;
constexpr size_t SMEM_BYTES = (size_t)STAGES * 2 * BM * LDS * sizeof(bf16);

template <int EPI>
__global__ void __launch_bounds__(T, 2) gemm_tc_kernel(Args g) {
    extern __shared__ __align__(16) unsigned char smraw[];
    auto As = reinterpret_cast<bf16(*)[BM][LDS]>(smraw);                                   // [STAGES][BM][LDS]
    auto Bs = reinterpret_cast<bf16(*)[BN][LDS]>(smraw + (size_t)STAGES * BM * LDS * sizeof(bf16));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;  // 2 x 4 warps: 64 rows x 32 columns each
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nk = g.K / BK;
    // one 16-byte piece (8 BF16) of a 128 x 32 tile per thread and round
    auto load = [&](int st, int k0) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int idx = tid + r * T, row = idx >> 2, c8 = (idx & 3) * 8;
            const int gm = m0 + row, gn = n0 + row;
            if (gm < g.M) cp16(&As[st][row][c8], g.A + (long long)gm * g.K + k0 + c8);
            else *reinterpret_cast<uint4 *>(&As[st][row][c8]) = make_uint4(0, 0, 0, 0);
            if (gn < g.N) cp16(&Bs[st][row][c8], g.Wt + (long long)gn * g.K + k0 + c8);
            else *reinterpret_cast<uint4 *>(&Bs[st][row][c8]) = make_uint4(0, 0, 0, 0);
        }
    };
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
#pragma unroll
    for (int q = 0; q < STAGES - 1; q++) {  // prologue: slices 0 .. STAGES-2, one commit group each
        if (q < nk) load(q, q * BK);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int kc = 0; kc < nk; kc++) {
        const int st = kc % STAGES;
        asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 2) : "memory");  // slice kc has landed
        __syncthreads();  // ... for every thread; every warp is done with slice kc-1
        if (kc + STAGES - 1 < nk) load((kc + STAGES - 1) % STAGES, (kc + STAGES - 1) * BK);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
#pragma unroll
        for (int ks = 0; ks < BK / 16; ks++) {
            uint32_t a[4][4], b[2][4];
#pragma unroll
            for (int mf = 0; mf < 4; mf++)
                ldsm4(a[mf], &As[st][wm * 64 + mf * 16 + (lane & 7) + ((lane >> 3) & 1) * 8][ks * 16 + (lane >> 4) * 8]);
#pragma unroll
            for (int nb = 0; nb < 2; nb++)
                ldsm4(b[nb], &Bs[st][wn * 32 + nb * 16 + (lane & 7) + (lane >> 4) * 8][ks * 16 + ((lane >> 3) & 1) * 8]);
#pragma unroll
            for (int mf = 0; mf < 4; mf++)
#pragma unroll
                for (int nf = 0; nf < 4; nf++)
                    mma_bf16(acc[mf][nf], a[mf], b[nf >> 1][(nf & 1) * 2], b[nf >> 1][(nf & 1) * 2 + 1]);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    const int gr = lane >> 2, gc = (lane & 3) * 2;
#pragma unroll
    for (int mf = 0; mf < 4; mf++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int m = m0 + wm * 64 + mf * 16 + gr + 8 * h;
            if (m >= g.M) continue;
#pragma unroll
            for (int nf = 0; nf < 4; nf++) {
                const int n = n0 + wn * 32 + nf * 8 + gc;
                if (n >= g.N) continue;
                const float z0 = acc[mf][nf][2 * h] + g.bias[n], z1 = acc[mf][nf][2 * h + 1] + g.bias[n + 1];
                const long long o = (long long)m * g.N + n;
                if constexpr (EPI == EPI_HIDDEN) {
                    if (g.Z) *reinterpret_cast<__nv_bfloat162 *>(g.Z + o) = __floats2bfloat162_rn(z0, z1);
                    *reinterpret_cast<__nv_bfloat162 *>(static_cast<bf16 *>(g.C) + o) =
                        __floats2bfloat162_rn(silu(z0), silu(z1));
                } else {
                    *reinterpret_cast<float2 *>(static_cast<float *>(g.C) + o) = make_float2(z0, z1);
                }
            }
        }
}

// BF16 transposed copies Wt_l [N][K] of the weights W_l [K][N] of layers
// 1 .. nl-1 (the layers the tensor-core forward runs).
struct WtTable {
    int nl;
    long long offW[17], offWt[17];
    int K[17], N[17];
};

__global__ void weights_bf16t_kernel(const float *params, bf16 *wt, WtTable t) {
    for (int l = 1; l < t.nl; l++) {
        const long long n = (long long)t.K[l] * t.N[l];
        const float *W = params + t.offW[l];
        bf16 *Wt = wt + t.offWt[l];
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
             i += (long long)gridDim.x * blockDim.x) {
            const int nn = (int)(i / t.K[l]), k = (int)(i % t.K[l]);
            Wt[i] = __float2bfloat16_rn(W[(long long)k * t.N[l] + nn]);
        }
    }
}

}  // namespace tc

// ---------------------------------------------------------------------------
// Fifth-generation tensor-core (tcgen05) forward of the layers fed by BF16
// activations whose BF16 weights fit in shared memory (K <= 256 and
// N <= 256, K a multiple of 64, N of 32): Z = H W + b with H [M][K] and
// Wt [N][K] (k contiguous).  A persistent CTA per SM keeps the layer's
// weights resident (one tiled TMA load of K/64 slices of N x 64) and
// streams 128-row tiles of H through a ring of 128 x 64 stages:
//   warp 0 (one thread)  tiled TMA loads of H into the ring,
//   warp 1 (one thread)  tcgen05.mma 128 x N x 16 into a TMEM accumulator,
//                        two accumulators of N columns alternating by tile,
//                        tcgen05.commit releasing ring stages and
//                        signalling finished accumulators,
//   warps 2-17           TMEM -> registers (tcgen05.ld), bias and SiLU;
//                        warp w reads TMEM lanes 32 (w % 4) .. + 31 (its
//                        sub-partition's rows) and every fourth 32-column
//                        chunk, so the epilogue of tile t overlaps the MMAs
//                        of tile t + 1.  Each 32 x 32 block goes through a
//                        swizzled shared-memory buffer (one per warp) and
//                        out by a tiled TMA store, so HBM sees whole lines
//                        (a thread storing its own row touched 32 lines per
//                        warp store, each 32-byte sector in two halves).
// Every mbarrier wait is bounded (tma::mbar_wait); a wait that gives up
// raises ST_TIMEOUT in the status word, the loader waits for the loads it
// issued, the MMA thread for its MMAs, and the block frees its TMEM.
// ---------------------------------------------------------------------------
namespace t5 {

using gabe::tma::mbar_wait;

constexpr int BM = 128, BK = 64, NEPI = 16, NT = 64 + 32 * NEPI;  // NEPI epilogue warps
constexpr int kMaxStages = 8;
constexpr int kTmemCols = 512;                 // two accumulators of up to 256 columns
constexpr int kStageBytes = BM * BK * 2;        // one 128 x 64 BF16 tile of H
constexpr size_t kFixedBytes = 1024 + 1024 + 256;  // alignment slack, bias, barriers

struct Args {
    int M, N, K, stages;
    const float *bias;
    bf16 *Z;                // EPI_HIDDEN: pre-activation (may be null)
    unsigned int *status;
};

// Output element size of the epilogue (BF16 hidden activations, FP32 output).
template <int EPI>
__host__ __device__ constexpr int out_bytes() {
    return EPI == EPI_HIDDEN ? 2 : 4;
}

// Shared memory: weights, ring stages, a staging buffer of 32 x 32 output
// elements per epilogue warp, bias, barriers.
__host__ __device__ inline size_t smem_bytes(int N, int K, int stages, int esize) {
    return kFixedBytes + (size_t)N * K * 2 + (size_t)stages * kStageBytes + (size_t)NEPI * 32 * 32 * esize;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

template <int EPI>
__global__ void __launch_bounds__(NT, 1)
    gemm_umma_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                     const __grid_constant__ CUtensorMap mapC, Args g) {
    namespace tma = gabe::tma;
    namespace umma = gabe::umma;
    extern __shared__ unsigned char smraw[];
    const uint32_t s0 = tma::saddr(smraw);
    unsigned char *sm = smraw + (((s0 + 1023u) & ~1023u) - s0);  // 1024-byte aligned for the swizzle
    const int N = g.N, K = g.K, KB = K / BK, S = g.stages;
    unsigned char *Bs = sm;                                   // K/64 slices of N x 128 bytes
    unsigned char *As = sm + (size_t)N * K * 2;               // S stages of 128 x 128 bytes
    constexpr int ES = out_bytes<EPI>(), SBUF = 32 * 32 * ES;  // one staging buffer
    unsigned char *Cs = As + (size_t)S * kStageBytes;         // [NEPI][SBUF]
    float *bias_s = reinterpret_cast<float *>(Cs + (size_t)NEPI * SBUF);  // 256 floats
    uint64_t *full = reinterpret_cast<uint64_t *>(bias_s + 256);
    uint64_t *empty = full + kMaxStages, *bfull = empty + kMaxStages, *tfull = bfull + 1, *tempty = tfull + 2,
             *done = tempty + 2;
    uint32_t *tbase_s = reinterpret_cast<uint32_t *>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = (g.M + BM - 1) / BM;

    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            tma::mbar_init(&full[s], 1);
            tma::mbar_init(&empty[s], 1);
        }
        tma::mbar_init(bfull, 1);
        for (int b = 0; b < 2; b++) {
            tma::mbar_init(&tfull[b], 1);
            tma::mbar_init(&tempty[b], 32 * NEPI);  // every epilogue thread
        }
        tma::mbar_init(done, 1);
        tma::fence_barrier_init();
    }
    for (int n = tid; n < N; n += NT) bias_s[n] = g.bias[n];
    if (warp == 1) umma::tmem_alloc(tbase_s, kTmemCols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tbase = *tbase_s;

    if (warp == 0) {
        if (lane == 0) {
            int fills[kMaxStages];
            for (int s = 0; s < kMaxStages; s++) fills[s] = 0;
            tma::mbar_arrive_expect(bfull, (uint32_t)(N * K * 2));
            for (int kb = 0; kb < KB; kb++) umma::load_2d(Bs + (size_t)kb * N * 128, &mapB, kb * BK, 0, bfull);
            int it = 0;
            bool ok = true;
            for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x)
                for (int kb = 0; kb < KB; kb++, it++) {
                    const int s = it % S;
                    if (!mbar_wait(&empty[s], (uint32_t)(((it / S) & 1) ^ 1), g.status)) {
                        ok = false;
                        break;
                    }
                    fills[s]++;
                    tma::mbar_arrive_expect(&full[s], (uint32_t)kStageBytes);
                    umma::load_2d(As + (size_t)s * kStageBytes, &mapA, kb * BK, tile * BM, &full[s]);
                }
            // every load issued has landed before the block may exit
            tma::drain(full, fills, S, g.status);
            mbar_wait(bfull, 0, g.status);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = umma::idesc_bf16(BM, N);
            bool ok = mbar_wait(bfull, 0, g.status);
            int it = 0, local = 0;
            for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x, local++) {
                const int b = local & 1;
                if (!mbar_wait(&tempty[b], (uint32_t)(((local >> 1) & 1) ^ 1), g.status)) break;
                umma::fence_after();
                const uint32_t d = tbase + (uint32_t)(b * 256);
                for (int kb = 0; kb < KB; kb++, it++) {
                    const int s = it % S;
                    if (!mbar_wait(&full[s], (uint32_t)((it / S) & 1), g.status)) {
                        ok = false;
                        break;
                    }
                    umma::fence_after();
                    const uint32_t sa = tma::saddr(As + (size_t)s * kStageBytes);
                    const uint32_t sb = tma::saddr(Bs + (size_t)kb * N * 128);
#pragma unroll
                    for (int k = 0; k < BK / 16; k++)
                        umma::mma_bf16(d, umma::desc_k128(sa + 32 * k), umma::desc_k128(sb + 32 * k), idesc,
                                       (uint32_t)((kb | k) != 0));
                    umma::commit(&empty[s]);  // the stage is free once these MMAs have read it
                }
                if (ok) umma::commit(&tfull[b]);
            }
            umma::commit(done);  // arrives once every MMA issued above has completed
            mbar_wait(done, 0, g.status);
        }
    } else {
        constexpr int NH = NEPI / 4;  // epilogue warps per TMEM lane quarter
        const int q = warp & 3, h = (warp - 2) >> 2, nch = N / 32;
        unsigned char *sb = Cs + (size_t)(warp - 2) * SBUF;
        int local = 0, cnt = 0;  // tiles and staged blocks of this warp
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, local++) {
            const int b = local & 1;
            const bool mine = mbar_wait(&tfull[b], (uint32_t)((local >> 1) & 1), g.status);
            if (!__all_sync(0xffffffffu, mine)) break;
            umma::fence_after();
            const int r0 = tile * BM + q * 32, row = r0 + lane;
            // (a warp whose rows all lie past M stages nothing: every staged
            // block is stored, so the buffer accounting below holds)
            for (int c = h; r0 < g.M && c < nch; c += NH, cnt++) {
                float v[32];
                umma::tmem_ld32(tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 256 + c * 32), v);
                const int n0 = c * 32;
                const float4 *bq = reinterpret_cast<const float4 *>(bias_s + n0);
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const float4 bb = bq[u];
                    v[4 * u] += bb.x;
                    v[4 * u + 1] += bb.y;
                    v[4 * u + 2] += bb.z;
                    v[4 * u + 3] += bb.w;
                }
                // the previous block's store must have read the buffer
                if (cnt >= 1) {
                    if (lane == 0) umma::store_wait_read<0>();
                    __syncwarp();
                }
                if constexpr (EPI == EPI_HIDDEN) {
                    // row `lane` of the block: 64 bytes, 16-byte unit u at u ^ ((lane / 2) % 4) (64-byte swizzle)
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        *reinterpret_cast<uint4 *>(sb + lane * 64 + ((u ^ ((lane >> 1) & 3)) << 4)) =
                            make_uint4(pack_bf16(silu_fast(v[8 * u]), silu_fast(v[8 * u + 1])),
                                       pack_bf16(silu_fast(v[8 * u + 2]), silu_fast(v[8 * u + 3])),
                                       pack_bf16(silu_fast(v[8 * u + 4]), silu_fast(v[8 * u + 5])),
                                       pack_bf16(silu_fast(v[8 * u + 6]), silu_fast(v[8 * u + 7])));
                    if (g.Z && row < g.M) {
                        uint4 *zo = reinterpret_cast<uint4 *>(g.Z + (long long)row * N + n0);
#pragma unroll
                        for (int u = 0; u < 4; u++)
                            zo[u] = make_uint4(pack_bf16(v[8 * u], v[8 * u + 1]), pack_bf16(v[8 * u + 2], v[8 * u + 3]),
                                               pack_bf16(v[8 * u + 4], v[8 * u + 5]),
                                               pack_bf16(v[8 * u + 6], v[8 * u + 7]));
                    }
                } else {
                    // row `lane`: 128 bytes, 16-byte unit u at u ^ (lane % 8) (128-byte swizzle)
#pragma unroll
                    for (int u = 0; u < 8; u++)
                        *reinterpret_cast<float4 *>(sb + lane * 128 + ((u ^ (lane & 7)) << 4)) =
                            make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                }
                tma::fence_proxy_async();  // the block's shared writes precede the store's reads
                __syncwarp();
                if (lane == 0) umma::store_2d(&mapC, n0, r0, sb);
            }
            umma::fence_before();
            umma::mbar_arrive(&tempty[b]);
        }
        if (lane == 0) umma::store_wait_all();
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 1) {
        umma::fence_after();
        umma::tmem_free(tbase, kTmemCols);
    }
}

}  // namespace t5

// dW = sum over splits of the partial products, db = sum of the partial
// column sums; fixed order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(256) splitk_reduce_kernel(const float *ws, const float *dbp, int splits,
                                                            long long mn, int N, float *dW, float *db) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < mn + N;
         i += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        if (i < mn)
            for (int z = 0; z < splits; z++) s += ws[z * mn + i];
        else
            for (int z = 0; z < splits; z++) s += dbp[(long long)z * N + (i - mn)];
        (i < mn ? dW[i] : db[i - mn]) = s;
    }
}

struct TrainScalars {
    double loss_last;
    double loss_sum;  // sum of batch losses since the last read
    long long loss_n;
    long long step;       // Adam steps taken
    long long batch_idx;  // batches taken since the last reset
    float inv_count;
    unsigned int counter;
};

constexpr int kLossBlocks = 148;

// Rows perm[batch_idx * B + i] of x and t into the batch buffers.
__global__ void gather_kernel(const float *x, const float *t, const int32_t *perm, const TrainScalars *ts, int B,
                              int nin, int nout, float *xb, float *tb) {
    const long long base = ts->batch_idx * (long long)B;
    const int w = nin + nout;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)B * w;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / w), c = (int)(q % w);
        const long long r = perm[base + i];
        if (c < nin) xb[(long long)i * nin + c] = x[r * nin + c];
        else tb[(long long)i * nout + (c - nin)] = t[r * nout + (c - nin)];
    }
}

// dY = 2 (y - t) on finite targets (0 elsewhere), unnormalised; the loss
// sum/count and 1/count (applied in the Adam step) from fixed-order block
// partials.  The last block also advances the step and batch counters.
__global__ void __launch_bounds__(256) loss_kernel(const float *y, const float *t, long long n, float *dy,
                                                   double2 *part, TrainScalars *ts, int count_batch) {
    double s = 0., c = 0.;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float tv = t[i];
        if (isfinite(tv)) {
            const float d = y[i] - tv;
            dy[i] = 2.f * d;
            s += (double)d * d;
            c += 1.;
        } else {
            dy[i] = 0.f;
        }
    }
    __shared__ double rs[256], rc[256];
    rs[threadIdx.x] = s;
    rc[threadIdx.x] = c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            rs[threadIdx.x] += rs[threadIdx.x + w];
            rc[threadIdx.x] += rc[threadIdx.x + w];
        }
        __syncthreads();
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = make_double2(rs[0], rc[0]);
        __threadfence();
        last = atomicAdd(&ts->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double S = 0., C = 0.;
        for (unsigned b = 0; b < gridDim.x; b++) {
            const double2 p = __ldcg(&part[b]);
            S += p.x;
            C += p.y;
        }
        const double L = C > 0. ? S / C : 0.;
        ts->loss_last = L;
        ts->inv_count = C > 0. ? (float)(1. / C) : 0.f;
        if (count_batch) {
            ts->loss_sum += L;
            ts->loss_n += 1;
            ts->step += 1;
            ts->batch_idx += 1;
        }
        ts->counter = 0u;
    }
}

// grad *= 1/count (for gabe_mlp_loss_grad)
__global__ void scale_kernel(float *g, long long n, const TrainScalars *ts) {
    const float s = ts->inv_count;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        g[i] *= s;
}

struct AdamHyper {
    float lr, b1, b2, eps, wd, lr_min;
    long long decay_steps;  // cosine from lr to lr_min over this many steps (0 = constant lr)
};

// AdamW with bias correction; the gradient is the unnormalised batch
// gradient times 1/count.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, long long n, AdamHyper h,
                            const TrainScalars *ts) {
    const float inv = ts->inv_count;
    const double t = (double)ts->step;
    const float bc1 = (float)(1. - pow((double)h.b1, t)), bc2 = (float)(1. - pow((double)h.b2, t));
    float lr = h.lr;
    if (h.decay_steps > 0) {
        const double f = fmin(t - 1., (double)h.decay_steps) / (double)h.decay_steps;
        lr = (float)(h.lr_min + 0.5 * (h.lr - h.lr_min) * (1. + cos(M_PI * f)));
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] * inv;
        float pi = p[i];
        pi -= lr * h.wd * pi;
        const float mi = h.b1 * m[i] + (1.f - h.b1) * gi;
        const float vi = h.b2 * v[i] + (1.f - h.b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] = pi - lr * (mi / bc1) / (sqrtf(vi / bc2) + h.eps);
    }
}

}  // namespace

struct gabe_mlp {
    gabe_mlp_params p{};
    int dev = 0;
    bool f32act = false;
    cudaStream_t stream = nullptr;
    int nl = 0;                      // layers (depth + 1)
    std::vector<int> K, N;           // per layer
    std::vector<long long> offW, offb;
    long long P = 0;
    float *params = nullptr, *grads = nullptr, *mom = nullptr, *vel = nullptr;
    float *xb = nullptr, *tb = nullptr, *y = nullptr, *dy = nullptr, *d0 = nullptr, *d1 = nullptr;
    float *ws = nullptr, *dbp = nullptr;  // split-K partials of the weight gradient
    bf16 *wt = nullptr;              // BF16 transposed weights of layers >= 1 (tensor-core forward)
    tc::WtTable wtab{};
    unsigned int *status = nullptr;  // device word: a bounded wait of the tcgen05 forward gave up
    int umma_stages[17] = {};        // per layer: ring stages of the tcgen05 forward, 0 = mma.sync kernel
    void *Z = nullptr, *H = nullptr;  // [depth][max_rows][width] activation type
    double2 *part = nullptr;
    TrainScalars *ts = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void *g_x = nullptr, *g_t = nullptr, *g_perm = nullptr;
    int g_batch = 0;
    std::string err;
};

namespace {

thread_local std::string g_mlp_create_error;

int mset(gabe_mlp *m, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (m) m->err = buf;
    else g_mlp_create_error = buf;
    return code;
}

#define MCK(m, call)                                                                                   \
    do {                                                                                               \
        cudaError_t _e = (call);                                                                       \
        if (_e != cudaSuccess) return mset((m), GABE_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

size_t act_size(const gabe_mlp *m) { return m->f32act ? sizeof(float) : sizeof(bf16); }

void *act_at(const gabe_mlp *m, void *base, int layer) {
    return static_cast<char *>(base) + (size_t)layer * m->p.max_rows * m->p.width * act_size(m);
}

constexpr int kMaxSplits = 16;

template <typename TA, typename TACT, int EPI>
int launch_gemm(gabe_mlp *m, const GemmArgs &g, int splits = 1) {
    const dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, splits);
    gemm_kernel<TA, TACT, EPI><<<grid, kThreads, 0, m->stream>>>(g);
    MCK(m, cudaGetLastError());
    return GABE_OK;
}

// Refreshes the BF16 transposed weight copies after the FP32 weights changed.
int refresh_wt(gabe_mlp *m) {
    if (m->f32act) return GABE_OK;
    tc::weights_bf16t_kernel<<<148, 256, 0, m->stream>>>(m->params, m->wt, m->wtab);
    MCK(m, cudaGetLastError());
    return GABE_OK;
}

template <int EPI>
int launch_tc(gabe_mlp *m, const tc::Args &a) {
    const dim3 grid((a.N + tc::BN - 1) / tc::BN, (a.M + tc::BM - 1) / tc::BM);
    MCK(m, cudaFuncSetAttribute(tc::gemm_tc_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tc::SMEM_BYTES));
    tc::gemm_tc_kernel<EPI><<<grid, tc::T, tc::SMEM_BYTES, m->stream>>>(a);
    MCK(m, cudaGetLastError());
    return GABE_OK;
}

// cuTensorMapEncodeTiled, looked up once through the runtime (no link
// dependency on the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiledFn) nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// 2-D BF16 tensor map of a row-major [rows][K] matrix, boxes of box_rows x 64
// with the 128-byte swizzle; rows beyond `rows` read as zeros.
bool encode_k_major(CUtensorMap *map, const bf16 *base, int K, int rows, int box_rows) {
    const EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    const cuuint32_t box[2] = {(cuuint32_t)t5::BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of a row-major [rows][N] output (BF16 or FP32, esize bytes),
// boxes of 32 x 32 with the swizzle whose span is one box row (64 or 128
// bytes), as the epilogue lays its staging buffers out.
bool encode_out(CUtensorMap *map, void *base, int esize, int N, int rows) {
    const EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)N * esize};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims,
              strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              esize == 2 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Ring stages of the tcgen05 forward for a K x N layer on this device, 0 if
// the layer does not take it (shape, resident weights too large, no tensor
// map encoder).
int umma_stages_for(int dev, int K, int N, int esize) {
    if (K % t5::BK || K > 256 || N % 32 || N > 256 || !encode_fn()) return 0;
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const long long room = (long long)optin - (long long)t5::smem_bytes(N, K, 0, esize);
    const long long st = room / t5::kStageBytes;
    return st < 2 ? 0 : (int)(st > t5::kMaxStages ? t5::kMaxStages : st);
}

constexpr int kNoTensorMap = -1;  // launch_umma: no tensor map for these operands; use the mma.sync kernel

template <int EPI>
int launch_umma(gabe_mlp *m, const tc::Args &a, int stages) {
    CUtensorMap ma, mb, mc;
    if (!encode_k_major(&ma, a.A, a.K, a.M, t5::BM) || !encode_k_major(&mb, a.Wt, a.K, a.N, a.N) ||
        !encode_out(&mc, a.C, t5::out_bytes<EPI>(), a.N, a.M))
        return kNoTensorMap;  // e.g. an output pointer off a 16-byte boundary
    t5::Args g{a.M, a.N, a.K, stages, a.bias, a.Z, m->status};
    const size_t smem = t5::smem_bytes(a.N, a.K, stages, t5::out_bytes<EPI>());
    MCK(m, cudaFuncSetAttribute(t5::gemm_umma_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nsm = 0;
    MCK(m, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->dev));
    const int tiles = (a.M + t5::BM - 1) / t5::BM;
    const int grid = tiles < nsm ? tiles : nsm;
    t5::gemm_umma_kernel<EPI><<<grid, t5::NT, smem, m->stream>>>(ma, mb, mc, g);
    MCK(m, cudaGetLastError());
    return GABE_OK;
}

// Input activations of layer l: x (FP32) for l = 0, H[l-1] otherwise.
// With BF16 activations every layer after the first runs on tensor cores.
template <typename TACT>
int forward_rows(gabe_mlp *m, const float *x, int rows, float *y, bool keep_z) {
    for (int l = 0; l < m->nl; l++) {
        if (l == 0 && m->nl > 1 && m->K[0] <= kFirstMaxIn && 256 % (m->N[0] / 8) == 0) {
            launch_first_n<TACT>(m->K[0], x, rows, m->params + m->offW[0], m->params + m->offb[0], m->N[0],
                                 static_cast<TACT *>(act_at(m, m->H, 0)),
                                 keep_z ? static_cast<TACT *>(act_at(m, m->Z, 0)) : nullptr, m->stream);
            MCK(m, cudaGetLastError());
            continue;
        }
        if constexpr (sizeof(TACT) == 2) {
            if (l > 0) {
                tc::Args a{};
                a.M = rows;
                a.N = m->N[l];
                a.K = m->K[l];
                a.A = static_cast<const bf16 *>(act_at(m, m->H, l - 1));
                a.Wt = m->wt + m->wtab.offWt[l];
                a.bias = m->params + m->offb[l];
                const bool last = l + 1 == m->nl;
                a.Z = (!last && keep_z) ? static_cast<bf16 *>(act_at(m, m->Z, l)) : nullptr;
                a.C = last ? static_cast<void *>(y) : act_at(m, m->H, l);
                const int st = m->umma_stages[l];
                int rc = st ? (last ? launch_umma<EPI_OUT>(m, a, st) : launch_umma<EPI_HIDDEN>(m, a, st))
                            : kNoTensorMap;
                if (rc == kNoTensorMap) rc = last ? launch_tc<EPI_OUT>(m, a) : launch_tc<EPI_HIDDEN>(m, a);
                if (rc) return rc;
                continue;
            }
        }
        GemmArgs g{};
        g.M = rows;
        g.N = m->N[l];
        g.K = m->K[l];
        g.A = l == 0 ? static_cast<const void *>(x) : act_at(m, m->H, l - 1);
        g.sam = m->K[l];
        g.sak = 1;
        g.B = m->params + m->offW[l];
        g.sbk = m->N[l];
        g.sbn = 1;
        g.bias = m->params + m->offb[l];
        g.ldc = m->N[l];
        int rc;
        if (l + 1 < m->nl) {
            g.Z = keep_z ? act_at(m, m->Z, l) : nullptr;
            g.C = act_at(m, m->H, l);
            rc = l == 0 ? launch_gemm<float, TACT, EPI_HIDDEN>(m, g) : launch_gemm<TACT, TACT, EPI_HIDDEN>(m, g);
        } else {
            g.C = y;
            rc = l == 0 ? launch_gemm<float, TACT, EPI_OUT>(m, g) : launch_gemm<TACT, TACT, EPI_OUT>(m, g);
        }
        if (rc) return rc;
    }
    return GABE_OK;
}

// Gradients of the unnormalised loss sum (dy holds 2 (y - t) on finite
// targets) into m->grads.
template <typename TACT>
int backward_rows(gabe_mlp *m, const float *x, int rows) {
    float *delta = m->dy, *other = m->d0;
    for (int l = m->nl - 1; l >= 0; l--) {
        const int K = m->K[l], N = m->N[l];
        // dW_l = input^T delta
        GemmArgs w{};
        w.M = K;
        w.N = N;
        w.K = rows;
        w.A = l == 0 ? static_cast<const void *>(x) : act_at(m, m->H, l - 1);
        w.sam = 1;
        w.sak = K;
        w.B = delta;
        w.sbk = N;
        w.sbn = 1;
        w.C = m->ws;
        w.ldc = N;
        w.dbp = m->dbp;
        // enough splits of the batch to give about two blocks per SM
        const int tiles = ((K + BM - 1) / BM) * ((N + BN - 1) / BN);
        int splits = (296 + tiles - 1) / tiles;
        splits = splits < 1 ? 1 : (splits > kMaxSplits ? kMaxSplits : splits);
        int chunk = (rows + splits - 1) / splits;
        chunk = (chunk + BK - 1) / BK * BK;
        splits = (rows + chunk - 1) / chunk;
        w.kchunk = chunk;
        int rc = l == 0 ? launch_gemm<float, TACT, EPI_BWD_WEIGHT>(m, w, splits)
                        : launch_gemm<TACT, TACT, EPI_BWD_WEIGHT>(m, w, splits);
        if (rc) return rc;
        splitk_reduce_kernel<<<148, 256, 0, m->stream>>>(m->ws, m->dbp, splits, (long long)K * N, N,
                                                         m->grads + m->offW[l], m->grads + m->offb[l]);
        MCK(m, cudaGetLastError());
        if (l == 0) break;
        // delta_{l-1} = (delta W_l^T) * SiLU'(Z_{l-1})
        GemmArgs d{};
        d.M = rows;
        d.N = K;
        d.K = N;
        d.A = delta;
        d.sam = N;
        d.sak = 1;
        d.B = m->params + m->offW[l];
        d.sbk = 1;
        d.sbn = N;
        d.Z = act_at(m, m->Z, l - 1);
        d.C = other;
        d.ldc = K;
        if ((rc = launch_gemm<float, TACT, EPI_BWD_DATA>(m, d))) return rc;
        delta = other;
        other = (other == m->d0) ? m->d1 : m->d0;
    }
    return GABE_OK;
}

int fwd(gabe_mlp *m, const float *x, int rows, float *y, bool keep_z) {
    return m->f32act ? forward_rows<float>(m, x, rows, y, keep_z) : forward_rows<bf16>(m, x, rows, y, keep_z);
}

int bwd(gabe_mlp *m, const float *x, int rows) {
    return m->f32act ? backward_rows<float>(m, x, rows) : backward_rows<bf16>(m, x, rows);
}

int train_step(gabe_mlp *m, const float *x, const float *t, const int32_t *perm, int B) {
    const int nin = m->p.n_in, nout = m->p.n_out;
    gather_kernel<<<148, 256, 0, m->stream>>>(x, t, perm, m->ts, B, nin, nout, m->xb, m->tb);
    MCK(m, cudaGetLastError());
    int rc = fwd(m, m->xb, B, m->y, true);
    if (rc) return rc;
    loss_kernel<<<kLossBlocks, 256, 0, m->stream>>>(m->y, m->tb, (long long)B * nout, m->dy, m->part, m->ts, 1);
    MCK(m, cudaGetLastError());
    if ((rc = bwd(m, m->xb, B))) return rc;
    AdamHyper h{m->p.lr, m->p.beta1, m->p.beta2, m->p.eps, m->p.weight_decay, m->p.lr_min, m->p.decay_steps};
    adam_kernel<<<148 * 4, 256, 0, m->stream>>>(m->params, m->grads, m->mom, m->vel, m->P, h, m->ts);
    MCK(m, cudaGetLastError());
    return refresh_wt(m);
}

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void free_all(gabe_mlp *m) {
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    if (m->graph) cudaGraphDestroy(m->graph);
    void *bufs[] = {m->params, m->grads, m->mom, m->vel, m->xb, m->tb, m->y, m->dy, m->d0, m->d1, m->Z, m->H,
                    m->part, m->ts, m->ws, m->dbp, m->wt, m->status};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (m->stream) cudaStreamDestroy(m->stream);
}

}  // namespace

extern "C" {

void gabe_mlp_default_params(gabe_mlp_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->struct_size = sizeof(gabe_mlp_params);
    p->n_in = 3;
    p->width = 256;
    p->depth = 4;
    p->n_out = 192;
    p->max_rows = 65536;
    p->lr = 1e-3f;
    p->beta1 = 0.9f;
    p->beta2 = 0.999f;
    p->eps = 1e-8f;
    p->weight_decay = 0.f;
    p->lr_min = 0.f;
    p->decay_steps = 0;
    p->seed = 1;
    p->device = -1;
}

int gabe_mlp_create(const gabe_mlp_params *p, gabe_mlp **out) {
    if (!out) return mset(nullptr, GABE_ERR_PARAM, "out is NULL");
    *out = nullptr;
    if (!p || p->struct_size != (int32_t)sizeof(gabe_mlp_params)) return mset(nullptr, GABE_ERR_PARAM, "bad gabe_mlp_params");
    if (p->n_in < 1 || p->n_in > 64 || p->width < 64 || p->width > 4096 || p->width % 64 || p->depth < 1 ||
        p->depth > 16 || p->n_out < 1 || p->n_out > 4096 || p->max_rows < 1 || p->max_rows > (1 << 21))
        return mset(nullptr, GABE_ERR_PARAM, "invalid MLP shape");
    if (!(p->lr >= 0) || !(p->beta1 >= 0 && p->beta1 < 1) || !(p->beta2 >= 0 && p->beta2 < 1) || !(p->eps > 0) ||
        !(p->weight_decay >= 0) || !(p->lr_min >= 0) || p->decay_steps < 0)
        return mset(nullptr, GABE_ERR_PARAM, "invalid optimiser parameters");
    gabe_mlp *m = new (std::nothrow) gabe_mlp();
    if (!m) return mset(nullptr, GABE_ERR_NOMEM, "host allocation failed");
    m->p = *p;
    m->f32act = (p->flags & GABE_MLP_FP32_ACT) != 0;
    m->nl = p->depth + 1;
    long long nwt = 0;
    m->wtab.nl = m->nl;
    for (int l = 0; l < m->nl; l++) {
        m->K.push_back(l == 0 ? p->n_in : p->width);
        m->N.push_back(l + 1 == m->nl ? p->n_out : p->width);
        m->offW.push_back(m->P);
        m->wtab.offW[l] = m->P;
        m->wtab.K[l] = m->K[l];
        m->wtab.N[l] = m->N[l];
        m->wtab.offWt[l] = nwt;
        if (l > 0) nwt += (long long)m->K[l] * m->N[l];
        m->P += (long long)m->K[l] * m->N[l];
        m->offb.push_back(m->P);
        m->P += m->N[l];
    }
    auto fail = [&](int code) {
        g_mlp_create_error = m->err;
        free_all(m);
        delete m;
        return code;
    };
    if (p->device >= 0 && cudaSetDevice(p->device) != cudaSuccess) {
        cudaGetLastError();
        mset(m, GABE_ERR_CUDA, "cudaSetDevice(%d) failed", p->device);
        return fail(GABE_ERR_CUDA);
    }
    if (cudaGetDevice(&m->dev) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        mset(m, GABE_ERR_CUDA, "no CUDA device");
        return fail(GABE_ERR_CUDA);
    }
    const size_t R = p->max_rows, W = p->width, A = act_size(m);
    const size_t wide = (size_t)(p->n_out > p->width ? p->n_out : p->width);
    struct {
        void **ptr;
        size_t bytes;
    } allocs[] = {
        {(void **)&m->params, (size_t)m->P * 4}, {(void **)&m->grads, (size_t)m->P * 4},
        {(void **)&m->mom, (size_t)m->P * 4},    {(void **)&m->vel, (size_t)m->P * 4},    {(void **)&m->xb, R * p->n_in * 4}, {(void **)&m->tb, R * p->n_out * 4},
        {(void **)&m->y, R * p->n_out * 4}, {(void **)&m->dy, R * p->n_out * 4}, {(void **)&m->d0, R * wide * 4},
        {(void **)&m->d1, R * wide * 4}, {&m->Z, (size_t)p->depth * R * W * A}, {&m->H, (size_t)p->depth * R * W * A},
        {(void **)&m->part, kLossBlocks * sizeof(double2)}, {(void **)&m->ts, sizeof(TrainScalars)},
        {(void **)&m->ws, (size_t)kMaxSplits * wide * wide * 4}, {(void **)&m->dbp, (size_t)kMaxSplits * wide * 4},
        {(void **)&m->wt, (size_t)(nwt > 0 ? nwt : 1) * sizeof(bf16)}, {(void **)&m->status, sizeof(unsigned int)},
    };
    for (auto &a : allocs) {
        if (cudaMalloc(a.ptr, a.bytes) != cudaSuccess) {
            cudaGetLastError();
            mset(m, GABE_ERR_NOMEM, "cudaMalloc(%zu bytes) failed", a.bytes);
            return fail(GABE_ERR_NOMEM);
        }
    }
    // Glorot-uniform weights, zero biases, from the seed
    std::vector<float> h(m->P, 0.f);
    uint64_t s = p->seed;
    for (int l = 0; l < m->nl; l++) {
        const double a = std::sqrt(6.0 / (m->K[l] + m->N[l]));
        for (long long i = 0; i < (long long)m->K[l] * m->N[l]; i++) {
            const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
            h[m->offW[l] + i] = (float)((2. * u - 1.) * a);
        }
    }
    TrainScalars ts{};
    if (cudaMemcpyAsync(m->params, h.data(), m->P * 4, cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->mom, 0, m->P * 4, m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->vel, 0, m->P * 4, m->stream) != cudaSuccess ||
        cudaMemcpyAsync(m->ts, &ts, sizeof(ts), cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->status, 0, sizeof(unsigned int), m->stream) != cudaSuccess ||
        refresh_wt(m) != GABE_OK || cudaStreamSynchronize(m->stream) != cudaSuccess) {
        cudaGetLastError();
        mset(m, GABE_ERR_CUDA, "initialisation copies failed");
        return fail(GABE_ERR_CUDA);
    }
    // tcgen05 forward for the BF16 layers whose weights fit in shared memory
    if (!m->f32act && !(p->flags & GABE_MLP_MMA_SYNC))
        for (int l = 1; l < m->nl; l++)
            m->umma_stages[l] = umma_stages_for(m->dev, m->K[l], m->N[l], l + 1 == m->nl ? 4 : 2);
    *out = m;
    return GABE_OK;
}

int gabe_mlp_destroy(gabe_mlp *m) {
    if (!m) return GABE_OK;
    cudaSetDevice(m->dev);
    if (m->stream) cudaStreamSynchronize(m->stream);
    free_all(m);
    delete m;
    return GABE_OK;
}

int64_t gabe_mlp_num_params(const gabe_mlp *m) { return m ? m->P : 0; }

int gabe_mlp_set_params(gabe_mlp *m, const float *h_params) {
    if (!m || !h_params) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    MCK(m, cudaMemcpyAsync(m->params, h_params, m->P * 4, cudaMemcpyHostToDevice, m->stream));
    int rc = refresh_wt(m);
    if (rc) return rc;
    MCK(m, cudaStreamSynchronize(m->stream));
    return GABE_OK;
}

int gabe_mlp_get_params(gabe_mlp *m, float *h_params) {
    if (!m || !h_params) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    MCK(m, cudaMemcpyAsync(h_params, m->params, m->P * 4, cudaMemcpyDeviceToHost, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    return GABE_OK;
}

int gabe_mlp_forward(gabe_mlp *m, const float *x, int64_t n, float *y) {
    if (!m || n < 0 || (n > 0 && (!x || !y))) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    for (int64_t r0 = 0; r0 < n; r0 += m->p.max_rows) {
        const int rows = (int)((n - r0) < m->p.max_rows ? (n - r0) : m->p.max_rows);
        int rc = fwd(m, x + r0 * m->p.n_in, rows, y + r0 * m->p.n_out, false);
        if (rc) return rc;
    }
    return GABE_OK;
}

int gabe_mlp_loss_grad(gabe_mlp *m, const float *x, const float *t, int64_t n, double *h_loss, float *h_grad) {
    if (!m || !x || !t || n < 1 || n > m->p.max_rows || !h_loss) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    const int rows = (int)n;
    int rc = fwd(m, x, rows, m->y, true);
    if (rc) return rc;
    loss_kernel<<<kLossBlocks, 256, 0, m->stream>>>(m->y, t, (long long)rows * m->p.n_out, m->dy, m->part, m->ts, 0);
    MCK(m, cudaGetLastError());
    if (h_grad) {
        if ((rc = bwd(m, x, rows))) return rc;
        scale_kernel<<<148, 256, 0, m->stream>>>(m->grads, m->P, m->ts);
        MCK(m, cudaGetLastError());
        MCK(m, cudaMemcpyAsync(h_grad, m->grads, m->P * 4, cudaMemcpyDeviceToHost, m->stream));
    }
    TrainScalars ts;
    MCK(m, cudaMemcpyAsync(&ts, m->ts, sizeof(ts), cudaMemcpyDeviceToHost, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    *h_loss = ts.loss_last;
    return GABE_OK;
}

int gabe_mlp_train(gabe_mlp *m, const float *x, const float *t, const int32_t *perm, int32_t batch, int32_t nbatch) {
    if (!m || !x || !t || !perm || batch < 1 || batch > m->p.max_rows || nbatch < 0) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    if (!(m->p.flags & GABE_MLP_NO_GRAPH) &&
        (!m->gexec || m->g_x != x || m->g_t != t || m->g_perm != perm || m->g_batch != batch)) {
        if (m->gexec) cudaGraphExecDestroy(m->gexec);
        if (m->graph) cudaGraphDestroy(m->graph);
        m->gexec = nullptr;
        m->graph = nullptr;
        MCK(m, cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        int rc = train_step(m, x, t, perm, batch);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(m->stream, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc ? rc : mset(m, GABE_ERR_CUDA, "capture of the training step failed: %s", cudaGetErrorString(e));
        }
        m->graph = g;
        MCK(m, cudaGraphInstantiate(&m->gexec, g, 0));
        m->g_x = x;
        m->g_t = t;
        m->g_perm = perm;
        m->g_batch = batch;
    }
    for (int s = 0; s < nbatch; s++) {
        if (m->gexec) MCK(m, cudaGraphLaunch(m->gexec, m->stream));
        else {
            int rc = train_step(m, x, t, perm, batch);
            if (rc) return rc;
        }
    }
    return GABE_OK;
}

int gabe_mlp_set_schedule(gabe_mlp *m, float lr, float lr_min, int32_t decay_steps) {
    if (!m || !(lr >= 0) || !(lr_min >= 0) || decay_steps < 0) return GABE_ERR_PARAM;
    m->p.lr = lr;
    m->p.lr_min = lr_min;
    m->p.decay_steps = decay_steps;
    // the captured step holds the hyper-parameters by value
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->gexec = nullptr;
    m->graph = nullptr;
    return GABE_OK;
}

int gabe_mlp_reset_batches(gabe_mlp *m) {
    if (!m) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    MCK(m, cudaMemsetAsync(&m->ts->batch_idx, 0, sizeof(long long), m->stream));
    return GABE_OK;
}

int gabe_mlp_train_loss(gabe_mlp *m, double *h_mean_loss, int64_t *h_steps) {
    if (!m) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    TrainScalars ts;
    MCK(m, cudaMemcpyAsync(&ts, m->ts, sizeof(ts), cudaMemcpyDeviceToHost, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    if (h_mean_loss) *h_mean_loss = ts.loss_n ? ts.loss_sum / (double)ts.loss_n : 0.;
    if (h_steps) *h_steps = ts.step;
    const double zero = 0.;
    const long long zn = 0;
    MCK(m, cudaMemcpyAsync(&m->ts->loss_sum, &zero, sizeof(zero), cudaMemcpyHostToDevice, m->stream));
    MCK(m, cudaMemcpyAsync(&m->ts->loss_n, &zn, sizeof(zn), cudaMemcpyHostToDevice, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    return GABE_OK;
}

int gabe_mlp_sync(gabe_mlp *m) {
    if (!m) return GABE_ERR_PARAM;
    MCK(m, cudaSetDevice(m->dev));
    MCK(m, cudaStreamSynchronize(m->stream));
    unsigned int st = 0;
    MCK(m, cudaMemcpy(&st, m->status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st) return mset(m, GABE_ERR_TIMEOUT, "a bounded wait of the tensor-core forward gave up (status %u)", st);
    return GABE_OK;
}

int gabe_mlp_forward_form(const gabe_mlp *m, int32_t layer) {
    if (!m || layer < 0 || layer >= m->nl) return -1;
    if (layer == 0 || m->f32act) return 0;
    return m->umma_stages[layer] ? 2 : 1;
}

void *gabe_mlp_stream(const gabe_mlp *m) { return m ? (void *)m->stream : nullptr; }

int gabe_mlp_launches_per_train_step(const gabe_mlp *m) {
    return m ? 3 + 3 * m->nl + (m->nl - 1) + (m->f32act ? 0 : 1) : 0;
}


int gabe_mlp_launches_per_forward(const gabe_mlp *m) { return m ? m->nl : 0; }

const char *gabe_mlp_last_error(const gabe_mlp *m) { return m ? m->err.c_str() : g_mlp_create_error.c_str(); }

}  // extern "C"
