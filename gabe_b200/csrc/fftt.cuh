// FP32 3-D r2c of the GW sources in three passes with transposed outputs,
// the last pass fused with the TT projection and h/l update.
//
// The reference transforms each source array with one 3-D r2c FFT
// (fft_stresstensor, g2evolutionpert.cpp:183-195) and then updates h and l
// per k-point (evolve_perts, :343-455).  A 512^3 array does not fit on chip,
// so the transform is one HBM pass per axis.  Here every pass reads whole
// lines of its own axis as contiguous runs and writes its output transposed,
// so that the next pass's lines are contiguous again:
//
//   pass 1 (rowt_kernel)   S[q][i][j][N+2] reals   -> T1[q][i][kz][j]
//          rows along k, two real rows as one complex sequence, 16-row
//          tiles landed by one bulk copy each, each kz written as one
//          128-byte piece of 16 consecutive j (eight 16-byte pair stores);
//   pass 2 (colt_kernel)   T1 lines along j         -> T2[q][kz][ky][i]
//          16 lines of consecutive i per tile, landed in shared memory by
//          bulk copies (cp.async.bulk + mbarrier), each ky written as one
//          128-byte piece of 16 consecutive i;
//   pass 3 (ikspace_kernel) T2 lines along i + amplitudes G[p][kz][ky][kx]
//          the ten source lines of one (kz, ky) land by bulk copies and are
//          transformed along i in shared memory, each thread reads its
//          k-points' amplitudes into registers, and the k-space update
//          (kspace_update_vals) runs on each kx; only the amplitudes go back
//          to HBM.
//
// The transformed sources never return to HBM after pass 2, and the
// amplitudes are kept in the transposed order [p][kz][ky][kx]
// (g_index with gt = 1) for the life of the handle.  q runs over the
// ten source arrays (stage-0 11,12,13,22,23, then stage 1); forward sign
// e^{-i}, unnormalised, as FFTW's r2c.
#pragma once

#include "fft3d.cuh"
#include "kspace.cuh"
#include "tma.cuh"

namespace gabe {
namespace f3t {

using pfft::FourStep;

// ---------------------------------------------------------------------------
// pass 1: rows along k -> T1[q][i][kz][j]
// ---------------------------------------------------------------------------
// A tile of 16 rows (8 pairs, each two real rows taken as one complex
// sequence) is one contiguous run of 16 (N + 2) floats in S and lands in
// shared memory by one bulk copy (cp.async.bulk + mbarrier) into a linear
// buffer.  The four-step FFT's first pass reads the pairs from
// the linear buffer (lanes over consecutive elements: conflict-free) and
// writes its output into a work buffer in the pair-preserving XOR swizzle of
// fft3d.cuh, so that the second pass's stride-L1 reads fall on distinct
// banks; the linear buffer is refilled as soon as the first pass has read
// it.  The separated pairs go straight to HBM: each thread separates one
// pair of rows at one kz (lanes over the 8 pairs, 4 kz per warp) and stores
// it as one 16-byte value, eight lanes making the 128-byte piece of 16 rows.
// Work rows sit N + 2 floats apart, so that the eight pairs' rows start on
// different banks.  One linear buffer per CTA (70 KB of shared memory with
// the work buffer and twiddles), refilled after the first pass while the
// second pass and the output run, and two CTAs per SM.  Measured at 512^3,
// same bytes, bit-identical output: 1.80 ms, against 2.08 with two linear
// buffers (103 KB per CTA), 2.00 and 1.97 with three CTAs per SM under
// 168- and 128-register caps, 2.13 for tiles landed by 8-byte cp.async
// copies straight into the swizzled layout; staging the output as
// [kz][16 rows] in shared memory and writing it
// piece by piece 3.30 ms against 2.28 (the extra barrier and shared-memory
// round trip held the 8 warps per SM); separating the pairs from the
// pass-2 registers through warp shuffles, with no write-back, 2.68 ms
// against 2.13 (each warp store then spans 16 lines instead of 4).
template <int N, int T_ = 128, int NB_ = 1>
struct RowTGeom {
    using RG = f3d::RowGeom<N, 16, 1, T_, 2>;  // the work buffer (swizzled, pitch N + 2)
    static constexpr int R = 16, RP = N + 2, NB = NB_;
    static constexpr size_t HEAD = 128;                          // NB mbarriers
    static constexpr size_t TW_BYTES = (size_t)N * sizeof(float2);  // twiddles of the four-step
    static constexpr size_t LIN_BYTES = (size_t)R * RP * sizeof(float);
    static constexpr size_t SMEM_BYTES = HEAD + TW_BYTES + NB * LIN_BYTES + (size_t)RG::BUF * sizeof(float);
    static_assert(LIN_BYTES % 16 == 0 && (HEAD + TW_BYTES) % 16 == 0, "bulk copies of 16-byte multiples");
};

template <int N, int T_ = 128, int MINB = 2, int NB_ = 1>
__global__ void __launch_bounds__(T_, MINB)
    rowt_kernel(const float *S, float2 *T1, long long nrows, unsigned int *status) {
    using G = RowTGeom<N, T_, NB_>;
    using Gm = typename G::RG;
    constexpr int L1 = Gm::L1, L2 = Gm::L2, PITCH = Gm::PITCH, R = Gm::R, P = Gm::P, T = Gm::T, NT2 = Gm::NT2;
    constexpr int RP = G::RP, NB = G::NB, NH = N / 2 + 1;
    static_assert(R == 16 && P == 8, "one 128-byte output piece per kz");
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm);
    float2 *tw = reinterpret_cast<float2 *>(sm + G::HEAD);
    float *lin0 = reinterpret_cast<float *>(sm + G::HEAD + G::TW_BYTES);  // [NB][R][RP]
    float *rows = lin0 + NB * R * RP;                                     // work buffer [R][PITCH], swizzled
    const int tid = threadIdx.x;
    const long long ntiles = nrows / R;
    if (tid == 0) {
        for (int b = 0; b < NB; b++) tma::mbar_init(&bar[b], 1);
        tma::fence_barrier_init();
    }
    f3d::twiddles<N>(tw);
    __syncthreads();
    int fills[NB] = {};  // thread 0: fills issued per buffer
    auto issue = [&](long long tile, int b) {
        fills[b]++;
        tma::mbar_arrive_expect(&bar[b], (uint32_t)G::LIN_BYTES);
        tma::load(lin0 + b * R * RP, S + tile * R * RP, (uint32_t)G::LIN_BYTES, &bar[b]);
    };
    if (tid == 0)
        for (int q = 0; q < NB; q++) {
            const long long t = blockIdx.x + (long long)q * gridDim.x;
            if (t < ntiles) issue(t, q);
        }
    int it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int b = it % NB;
        const bool ok = tma::mbar_wait(&bar[b], (uint32_t)((it / NB) & 1), status);
        if (__syncthreads_or(!ok)) {  // also: every thread is done with tile it-1's work buffer
            if (tid == 0) tma::drain(bar, fills, NB, status);
            break;
        }
        const float *lin = lin0 + b * R * RP;
        // four-step pass 1: L2-point FFTs over n2 (stride L1), twiddle W_N^(n1 k2), in place
        // two adjacent n1 per thread: each pair of reals is one 8-byte access
        for (int t = tid; t < P * (L1 / 2); t += T) {
            const int p = t / (L1 / 2), n1 = 2 * (t % (L1 / 2));
            const float *lre = lin + 2 * p * RP, *lim = lre + RP;
            float *re = rows + 2 * p * PITCH, *im = re + PITCH;
            float2 xa[L2], xb[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) {
                const float2 r2 = *reinterpret_cast<const float2 *>(lre + n1 + L1 * n2);
                const float2 i2 = *reinterpret_cast<const float2 *>(lim + n1 + L1 * n2);
                xa[n2] = make_float2(r2.x, i2.x);
                xb[n2] = make_float2(r2.y, i2.y);
            }
            pfft::fft_reg<L2>(xa);
            pfft::fft_reg<L2>(xb);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) {
                const float2 ya = k2 ? pfft::cmul(xa[k2], tw[k2 * L1 + n1]) : xa[k2];
                const float2 yb = k2 ? pfft::cmul(xb[k2], tw[k2 * L1 + n1 + 1]) : xb[k2];
                const int a = Gm::phys(n1 + L1 * k2);
                *reinterpret_cast<float2 *>(re + a) = make_float2(ya.x, yb.x);
                *reinterpret_cast<float2 *>(im + a) = make_float2(ya.y, yb.y);
            }
        }
        __syncthreads();  // pass 1 done: the linear buffer may be refilled
        if (tid == 0) {
            const long long ahead = tile + (long long)NB * gridDim.x;
            if (ahead < ntiles) {
                tma::fence_proxy_async();  // the buffer's reads by pass 1 precede its refill
                issue(ahead, b);
            }
        }
        // pass 2: L1-point FFTs over n1, written back in natural order k = k2 + L2 k1
        {
            float2 y[NT2][L1];
#pragma unroll
            for (int q = 0; q < NT2; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                if (t < P * L2) {
                    const float *re = rows + 2 * p * PITCH, *im = re + PITCH;
#pragma unroll
                    for (int n1 = 0; n1 < L1; n1 += 2) {
                        const int a = Gm::phys(n1 + L1 * k2);
                        const float2 r2 = *reinterpret_cast<const float2 *>(re + a);
                        const float2 i2 = *reinterpret_cast<const float2 *>(im + a);
                        y[q][n1] = make_float2(r2.x, i2.x);
                        y[q][n1 + 1] = make_float2(r2.y, i2.y);
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
        const long long qi = tile / (N / R);  // q N + i
        const int j0 = (int)(tile % (N / R)) * R;
        float2 *o = T1 + qi * NH * N + j0;
        // pair p of kz k -> rows j0 + 2p, j0 + 2p + 1 of T1[q][i][k] as one 16-byte store
        for (int t = tid; t < P * NH; t += T) {
            const int p = t % P, k = t / P, km = (N - k) & (N - 1);
            const float *re = rows + 2 * p * PITCH, *im = re + PITCH;
            const int ak = Gm::phys(k & (N - 1)), am = Gm::phys(km);
            const float zr = re[ak], zi = im[ak], mr = re[am], mi = im[am];
            __stcs(reinterpret_cast<float4 *>(o + (long long)k * N + 2 * p),
                   make_float4(0.5f * (zr + mr), 0.5f * (zi - mi), 0.5f * (zi + mi), 0.5f * (mr - zr)));
        }
    }
}

// ---------------------------------------------------------------------------
// Four-step FFT of whole lines held contiguously in shared memory
// ---------------------------------------------------------------------------
// Line w occupies [w * PL, w * PL + N) complex (PL = N + 2: 16-byte aligned
// for the bulk copies, and consecutive lines 4 banks apart).  Step A: for
// each (w, n1) the L2-point FFT of elements n1 + L1 n2, twiddled, in place
// (lanes over n1: consecutive words).
template <int N, int T>
__device__ __forceinline__ void lines_step_a(float2 *buf, int nlines, const float2 *tw) {
    constexpr int L1 = FourStep<N>::L1, L2 = FourStep<N>::L2, PL = N + 2;
    for (int t = threadIdx.x; t < nlines * L1; t += T) {
        const int w = t / L1, n1 = t % L1;
        float2 *ln = buf + w * PL;
        float2 x[L2];
#pragma unroll
        for (int n2 = 0; n2 < L2; n2++) x[n2] = ln[n1 + L1 * n2];
        pfft::fft_reg<L2>(x);
#pragma unroll
        for (int k2 = 0; k2 < L2; k2++) ln[n1 + L1 * k2] = k2 ? pfft::cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
    }
}

// Step B input of task (w, k2): the L1 elements L1 k2 .. L1 k2 + L1 - 1 of
// line w (16-byte loads), transformed in registers; y[k1] is output element
// k2 + L2 k1.
template <int N>
__device__ __forceinline__ void lines_step_b(const float2 *buf, int w, int k2, float2 (&y)[FourStep<N>::L1]) {
    constexpr int L1 = FourStep<N>::L1, PL = N + 2;
    const float4 *src = reinterpret_cast<const float4 *>(buf + w * PL + L1 * k2);
#pragma unroll
    for (int h = 0; h < L1 / 2; h++) {
        const float4 v = src[h];
        y[2 * h] = make_float2(v.x, v.y);
        y[2 * h + 1] = make_float2(v.z, v.w);
    }
    pfft::fft_reg<L1>(y);
}

// Shared-memory ring of NB tiles, each of nl lines of pitch N + 2, filled by
// bulk copies; barrier b completes when tile buffer b has landed.
// EXTRA lines of pitch N + 2 follow the ring (a result area).
template <int N, int NL, int NB, int EXTRA = 0>
struct LineRing {
    static constexpr int PL = N + 2, BUF = NL * PL;
    static constexpr size_t HEAD = 128;  // NB mbarriers (8 bytes each)
    static constexpr size_t SMEM_BYTES =
        HEAD + (size_t)N * sizeof(float2) + ((size_t)NB * BUF + (size_t)EXTRA * PL) * sizeof(float2);
    static_assert(NB * 8 <= (int)HEAD, "barriers fit the head");
    __device__ static uint64_t *bars(unsigned char *sm) { return reinterpret_cast<uint64_t *>(sm); }
    __device__ static float2 *twid(unsigned char *sm) { return reinterpret_cast<float2 *>(sm + HEAD); }
    __device__ static float2 *buf(unsigned char *sm, int b) { return twid(sm) + N + b * BUF; }
    __device__ static float2 *extra(unsigned char *sm) { return twid(sm) + N + NB * BUF; }
};

// ---------------------------------------------------------------------------
// pass 2: along j, T1[q][i][kz][j] -> T2[q][kz][ky][i]
// ---------------------------------------------------------------------------
constexpr int kColW = 16;  // lines (consecutive i) per tile: one 128-byte output piece per ky

template <int N, int T, int NB, int MINB = 1>
__global__ void __launch_bounds__(T, MINB) colt_kernel(const float2 *__restrict__ T1, float2 *__restrict__ T2, int ncomp,
                                                    unsigned int *status) {
    using Rg = LineRing<N, kColW, NB>;
    constexpr int L1 = FourStep<N>::L1, L2 = FourStep<N>::L2, NH = N / 2 + 1, W = kColW;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t *bar = Rg::bars(sm);
    float2 *tw = Rg::twid(sm);
    const int tid = threadIdx.x;
    const long long ntiles = (long long)ncomp * NH * (N / W);
    if (tid == 0) {
        for (int b = 0; b < NB; b++) tma::mbar_init(&bar[b], 1);
        tma::fence_barrier_init();
    }
    f3d::twiddles<N>(tw);
    __syncthreads();
    int fills[NB] = {};  // thread 0: fills issued per buffer
    // tile = (q NH + kz) (N / W) + ib: lines i = ib W + w of (q, kz)
    auto issue = [&](long long tile, int b) {
        fills[b]++;
        const int ib = (int)(tile % (N / W));
        const long long qk = tile / (N / W);
        const int kz = (int)(qk % NH), q = (int)(qk / NH);
        float2 *dst = Rg::buf(sm, b);
        tma::mbar_arrive_expect(&bar[b], W * N * (uint32_t)sizeof(float2));
        for (int w = 0; w < W; w++)
            tma::load(dst + w * Rg::PL, T1 + (((long long)q * N + ib * W + w) * NH + kz) * N,
                      N * (uint32_t)sizeof(float2), &bar[b]);
    };
    if (tid == 0)
        for (int q = 0; q < NB - 1; q++) {
            const long long t = blockIdx.x + (long long)q * gridDim.x;
            if (t < ntiles) issue(t, q);
        }
    int it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int b = it % NB;
        if (tid == 0) {
            const long long ahead = tile + (long long)(NB - 1) * gridDim.x;
            if (ahead < ntiles) {
                tma::fence_proxy_async();  // the buffer's last reads (tile it-1) precede its refill
                issue(ahead, (it + NB - 1) % NB);
            }
        }
        const bool ok = tma::mbar_wait(&bar[b], (uint32_t)((it / NB) & 1), status);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) tma::drain(bar, fills, NB, status);
            break;
        }
        float2 *buf = Rg::buf(sm, b);
        lines_step_a<N, T>(buf, W, tw);
        __syncthreads();
        const int ib = (int)(tile % (N / W));
        const long long qk = tile / (N / W);  // q NH + kz
        float2 *o = T2 + qk * N * N + ib * W;
        for (int t = tid; t < W * L2; t += T) {
            const int w = t % W, k2 = t / W;
            float2 y[L1];
            lines_step_b<N>(buf, w, k2, y);
#pragma unroll
            for (int k1 = 0; k1 < L1; k1++) __stcs(o + (long long)(k2 + L2 * k1) * N + w, y[k1]);
        }
        __syncthreads();  // buffer b consumed
    }
}

// ---------------------------------------------------------------------------
// pass 3: along i, fused with the TT projection and both RK2 stages of h, l
// ---------------------------------------------------------------------------

struct IkArgs {
    const float2 *T2;  // [10][NH][N][N]
    float2 *G;         // [4][NH][N][N]
    const DevScalars *sc;
    LatticeConsts c;
    int slot;
    unsigned int *status;
};

// Three barriers per (kz, ky): after the bulk copies land, after step A, and
// after step B, whose results go to a separate area (the transformed source
// lines) so that it needs no barrier between its reads and writes.  The
// amplitudes are read straight from global memory: each thread loads its
// k-points' four amplitudes into registers when a task starts (the loads
// overlap the wait for the source lines), so the ring holds only the ten
// source lines and two CTAs fit on an SM -- one CTA's transforms fill the
// other's barrier waits (1.69 ms at 512^3 for two CTAs of 192 threads,
// 1.75 for 256, against 2.28 for one CTA of 512 threads with the amplitude
// lines in its ring).  Buffer b is refilled as
// soon as step B has read it (third barrier), while the k-space phase of
// the same task runs.
template <int N, int T, int NB, int MINB>
__global__ void __launch_bounds__(T, MINB) ikspace_kernel(IkArgs a) {
    using Rg = LineRing<N, 2 * kSrc, NB, 2 * kSrc>;
    constexpr int L1 = FourStep<N>::L1, L2 = FourStep<N>::L2, NH = N / 2 + 1, PL = Rg::PL;
    constexpr int KPT = (N + T - 1) / T;  // k-points per thread
    constexpr long long M = (long long)NH * N * N;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t *bar = Rg::bars(sm);
    float2 *tw = Rg::twid(sm);
    float2 *xs = Rg::extra(sm);  // [10][PL]: the source lines transformed along i, natural order
    const int tid = threadIdx.x;
    constexpr long long ntasks = (long long)NH * N;  // task = kz N + ky
    const KsCoef<float> kc = ks_coef<float>(a.c, a.sc->gw[a.slot]);
    if (tid == 0) {
        for (int b = 0; b < NB; b++) tma::mbar_init(&bar[b], 1);
        tma::fence_barrier_init();
    }
    f3d::twiddles<N>(tw);
    __syncthreads();
    int fills[NB] = {};  // thread 0: fills issued per buffer
    auto issue = [&](long long task, int b) {
        fills[b]++;
        float2 *dst = Rg::buf(sm, b);
        tma::mbar_arrive_expect(&bar[b], 2 * kSrc * N * (uint32_t)sizeof(float2));
        for (int q = 0; q < 2 * kSrc; q++)
            tma::load(dst + q * PL, a.T2 + q * M + task * N, N * (uint32_t)sizeof(float2), &bar[b]);
    };
    if (tid == 0)
        for (int q = 0; q < NB; q++) {
            const long long t = blockIdx.x + (long long)q * gridDim.x;
            if (t < ntasks) issue(t, q);
        }
    int it = 0;
    for (long long task = blockIdx.x; task < ntasks; task += gridDim.x, it++) {
        const int b = it % NB;
        float2 *gl = a.G + task * N;
        float2 gv[KPT][4];
#pragma unroll
        for (int r = 0; r < KPT; r++) {
            const int kx = tid + r * T;
#pragma unroll
            for (int p = 0; p < 4; p++) gv[r][p] = kx < N ? __ldcs(gl + p * M + kx) : make_float2(0.f, 0.f);
        }
        const bool ok = tma::mbar_wait(&bar[b], (uint32_t)((it / NB) & 1), a.status);
        if (__syncthreads_or(!ok)) {  // also: every thread is done with task it-1's k-space phase (xs)
            if (tid == 0) tma::drain(bar, fills, NB, a.status);
            break;
        }
        float2 *buf = Rg::buf(sm, b);
        lines_step_a<N, T>(buf, 2 * kSrc, tw);
        __syncthreads();
        // step B over the ten source lines (lanes over lines) into xs in natural order
        for (int t = tid; t < 2 * kSrc * L2; t += T) {
            const int w = t % (2 * kSrc), k2 = t / (2 * kSrc);
            float2 y[L1];
            lines_step_b<N>(buf, w, k2, y);
            float2 *ln = xs + w * PL;
#pragma unroll
            for (int k1 = 0; k1 < L1; k1++) ln[k2 + L2 * k1] = y[k1];
        }
        __syncthreads();
        if (tid == 0) {
            const long long ahead = task + (long long)NB * gridDim.x;
            if (ahead < ntasks) {
                tma::fence_proxy_async();  // the buffer's reads by steps A and B precede its refill
                issue(ahead, b);
            }
        }
        const int kz = (int)(task / N), ky = (int)(task % N);
        const int py = ky <= N / 2 ? ky : ky - N;
#pragma unroll
        for (int r = 0; r < KPT; r++) {
            const int kx = tid + r * T;
            if (kx >= N) break;
            Cplx<float> s[10], g[4];
#pragma unroll
            for (int q = 0; q < 2 * kSrc; q++) {
                const float2 v = xs[q * PL + kx];
                s[q] = {v.x, v.y};
            }
#pragma unroll
            for (int p = 0; p < 4; p++) g[p] = {gv[r][p].x, gv[r][p].y};
            const int px = kx <= N / 2 ? kx : kx - N;
            kspace_update_vals<float, true>(kc, px, py, kz, s, g);
#pragma unroll
            for (int p = 0; p < 4; p++) __stcs(gl + p * M + kx, make_float2(g[p].re, g[p].im));
        }
    }
}

}  // namespace f3t
}  // namespace gabe
