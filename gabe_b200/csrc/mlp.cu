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

// Input activations of layer l: x (FP32) for l = 0, H[l-1] otherwise.
// With BF16 activations every layer after the first runs on tensor cores.
template <typename TACT>
int forward_rows(gabe_mlp *m, const float *x, int rows, float *y, bool keep_z) {
    for (int l = 0; l < m->nl; l++) {
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
                const int rc = last ? launch_tc<EPI_OUT>(m, a) : launch_tc<EPI_HIDDEN>(m, a);
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
                    m->part, m->ts, m->ws, m->dbp, m->wt};
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
        {(void **)&m->wt, (size_t)(nwt > 0 ? nwt : 1) * sizeof(bf16)},
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
        refresh_wt(m) != GABE_OK || cudaStreamSynchronize(m->stream) != cudaSuccess) {
        cudaGetLastError();
        mset(m, GABE_ERR_CUDA, "initialisation copies failed");
        return fail(GABE_ERR_CUDA);
    }
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
    return GABE_OK;
}

void *gabe_mlp_stream(const gabe_mlp *m) { return m ? (void *)m->stream : nullptr; }

int gabe_mlp_launches_per_train_step(const gabe_mlp *m) {
    return m ? 3 + 3 * m->nl + (m->nl - 1) + (m->f32act ? 0 : 1) : 0;
}


int gabe_mlp_launches_per_forward(const gabe_mlp *m) { return m ? m->nl : 0; }

const char *gabe_mlp_last_error(const gabe_mlp *m) { return m ? m->err.c_str() : g_mlp_create_error.c_str(); }

}  // extern "C"
