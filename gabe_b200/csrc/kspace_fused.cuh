// FP32 k-space update with the last FFT pass fused in.
//
// After the 2-D r2c of every (j, k) plane (cuFFT's batched 2-D plan, or the
// plane kernel of planefft.cuh) the sources still need their transform along
// i.  Done as a separate pass it writes ten N^2(N/2+1) complex arrays that
// the k-space update (kspace.cuh) then reads back.  Here each CTA owns W
// columns kz in [kz0, kz0 + W) of one row j for all i, and per RK2 stage
//   1. copies the five components of that stage (W columns x N values each)
//      into shared memory with cp.async,
//   2. transforms every column along i (four-step FFT, N = L1 L2, in shared
//      memory, same routines as the plane kernel),
//   3. projects each k-point onto the two polarizations,
//      T_p = 2 (8 pi / a^2) dx^3 eps^p : S / 2 (fft_stresstensor's TT
//      projection, g2evolutionpert.cpp:203-313, in the polarization form of
//      kspace.cuh),
// keeping stage 0's T_p in registers; after stage 1 it takes both RK2 stages
// of h and l (evolve_perts/derivs, g2evolutionpert.cpp:406-431, 459-516) and
// writes the amplitudes.  Per k-point: 10 complex source values read once,
// 4 amplitudes read and written; the i-transformed sources never exist in HBM.
#pragma once

#include "kspace.cuh"
#include "planefft.cuh"
#include "sweep32.cuh"

namespace gabe {
namespace ksf {

// Per-N tile: W columns, four-step split N = L1 L2.  W N = 2048 k-points and
// 5 W N complex values (80 KiB) of shared memory per CTA at every N.
template <int N>
struct KsCfg;
template <>
struct KsCfg<512> {
    static constexpr int W = 4, L1 = 32, L2 = 16;
};
template <>
struct KsCfg<256> {
    static constexpr int W = 8, L1 = 16, L2 = 16;
};
template <>
struct KsCfg<128> {
    static constexpr int W = 16, L1 = 16, L2 = 8;
};
template <>
struct KsCfg<64> {
    static constexpr int W = 32, L1 = 8, L2 = 8;
};

constexpr int kKsThreads = 320;

template <int N>
struct KsGeom {
    static constexpr int W = KsCfg<N>::W, L1 = KsCfg<N>::L1, L2 = KsCfg<N>::L2;
    static constexpr int T = kKsThreads;
    static constexpr int NCOL = 5 * W;  // columns of one stage
    static constexpr int K = N * W;     // k-points per tile
    static constexpr int KPT = (K + T - 1) / T;
    // complex slot of (component qq, i, column w): W values per i, plus W
    // padding values after every L1 values of i (bank spread for the strided
    // passes)
    static constexpr int COMP = N * W + (N / L1) * W;
    static constexpr int SMEM_C = 5 * COMP + N;  // + twiddles
    static constexpr size_t SMEM_BYTES = (size_t)SMEM_C * sizeof(float2);
    __device__ static __forceinline__ int idx(int qq, int i, int w) { return qq * COMP + (i + (i / L1)) * W + w; }
    static_assert(L1 * L2 == N, "four-step split");
    static_assert((NCOL * L1) % T == 0 && (NCOL * L2) % T == 0, "FFT passes divide over the threads");
};

template <int N>
__global__ void __launch_bounds__(kKsThreads, 2) kspace_fused_kernel(KspaceArgs args) {
    using G = KsGeom<N>;
    constexpr int W = G::W, L1 = G::L1, L2 = G::L2, T = G::T, NCOL = G::NCOL, K = G::K, KPT = G::KPT;
    constexpr int nz = N / 2 + 1;
    constexpr size_t M = (size_t)N * N * nz;
    extern __shared__ __align__(16) float2 sm[];
    float2 *tw = sm + 5 * G::COMP;  // [k2][n1]: W_N^(n1 k2)
    const int tid = threadIdx.x;
    const int ngrp = (nz + W - 1) / W;

    for (int m = tid; m < N; m += T) {
        const int k2 = m / L1, n1 = m % L1;
        double sn, cs;
        sincospi(2.0 * (n1 * k2) / N, &sn, &cs);
        tw[m] = make_float2((float)cs, (float)-sn);
    }

    const LatticeConsts &c = args.c;
    const double *g4 = args.sc->gw[args.slot];
    const double a0 = g4[0], ad0 = g4[1], a1 = g4[2], ad1 = g4[3];
    const double norm0 = c.k2norm_c / a0 / a0, norm1 = c.k2norm_c / a1 / a1;
    const double om0 = c.eight_pi / a0 / a0, om1 = c.eight_pi / a1 / a1;
    const float c3H0 = (float)(3. * ad0 / a0), c3H1 = (float)(3. * ad1 / a1);
    const float src0 = (float)(2. * om0 * c.normmm), src1 = (float)(2. * om1 * c.normmm);
    const float hdt = (float)c.half_dt, dt = (float)c.dt;
    const float n0f = (float)norm0, n1f = (float)norm1;
    const float2 *S = static_cast<const float2 *>(args.S);
    float2 *Gm = static_cast<float2 *>(args.G);

    // persistent: tiles (row j, column group) in order, W columns each
    for (int tile = blockIdx.x; tile < N * ngrp; tile += gridDim.x) {
    const int j = tile / ngrp, kz0 = (tile % ngrp) * W;
    const int py = j <= N / 2 ? j : j - N;
    float2 t0[KPT][2];  // stage-0 projections of this thread's k-points
#pragma unroll
    for (int st = 0; st < 2; st++) {
        __syncthreads();  // previous stage's shared data consumed; twiddles ready
        // ---- copy the stage's five components: (qq, i, w), w fastest ----
        for (int t = tid; t < 5 * K; t += T) {
            const int w = t % W, r = t / W, i = r % N, qq = r / N;
            float2 *dst = sm + G::idx(qq, i, w);
            const int kz = kz0 + w;
            if (kz < nz)
                s32::cp_async8(dst, S + (size_t)(5 * st + qq) * M + ((size_t)i * N + j) * nz + kz);
            else
                *dst = make_float2(0.f, 0.f);
        }
        s32::cp_commit();
        s32::cp_wait<0>();
        __syncthreads();
        // ---- FFT along i, pass 1: L2-point FFTs over n2, twiddle ----
#pragma unroll
        for (int t0i = 0; t0i < NCOL * L1; t0i += T) {
            const int t = t0i + tid, w = t % W, r = t / W, n1 = r % L1, qq = r / L1;
            float2 x[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) x[n2] = sm[G::idx(qq, n1 + L1 * n2, w)];
            pfft::fft_reg<L2>(x);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++)
                sm[G::idx(qq, n1 + L1 * k2, w)] = k2 ? pfft::cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
        }
        __syncthreads();
        // ---- pass 2: L1-point FFTs over n1; slot k1 + L1 k2 then holds kx = k2 + L2 k1 ----
#pragma unroll
        for (int t0i = 0; t0i < NCOL * L2; t0i += T) {
            const int t = t0i + tid, w = t % W, r = t / W, k2 = r % L2, qq = r / L2;
            float2 y[L1];
#pragma unroll
            for (int n1 = 0; n1 < L1; n1++) y[n1] = sm[G::idx(qq, n1 + L1 * k2, w)];
            pfft::fft_reg<L1>(y);
#pragma unroll
            for (int k1 = 0; k1 < L1; k1++) sm[G::idx(qq, k1 + L1 * k2, w)] = y[k1];
        }
        __syncthreads();
        // ---- projection (and, after stage 1, the h/l update) per k-point ----
#pragma unroll
        for (int q = 0; q < KPT; q++) {
            const int t = q * T + tid;
            if (t >= K) break;
            const int w = t % W, kx = t / W, kz = kz0 + w;
            const int slot = kx / L2 + L1 * (kx % L2);
            const int px = kx <= N / 2 ? kx : kx - N;
            const float m2 = (float)(px * px + py * py + kz * kz);
            float2 tp = make_float2(0.f, 0.f), tx = make_float2(0.f, 0.f);
            if (kz < nz && m2 != 0.f) {
                // polarization basis (kspace.cuh pol_tensors, in FP32)
                const float inv = rsqrtf(m2);
                const float kx_ = px * inv, ky_ = py * inv, kz_ = kz * inv;
                // reference axis from the integer vector: the same choice as pol_tensors
                const int ax = abs(px), ay = abs(py), az = kz;
                const int rr = (ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2);
                const float kr = rr == 0 ? kx_ : (rr == 1 ? ky_ : kz_);
                float e1x = (rr == 0 ? 1.f : 0.f) - kr * kx_, e1y = (rr == 1 ? 1.f : 0.f) - kr * ky_,
                      e1z = (rr == 2 ? 1.f : 0.f) - kr * kz_;
                const float n1 = rsqrtf(e1x * e1x + e1y * e1y + e1z * e1z);
                e1x *= n1; e1y *= n1; e1z *= n1;
                const float e2x = ky_ * e1z - kz_ * e1y, e2y = kz_ * e1x - kx_ * e1z, e2z = kx_ * e1y - ky_ * e1x;
                // weights of (S11, S12, S13, S22, S23) in eps:S/2 with S33 = -S11 - S22
                const float ep33 = e1z * e1z - e2z * e2z, ex33 = 2.f * e1z * e2z;
                const float wp[5] = {0.5f * ((e1x * e1x - e2x * e2x) - ep33), e1x * e1y - e2x * e2y,
                                     e1x * e1z - e2x * e2z, 0.5f * ((e1y * e1y - e2y * e2y) - ep33),
                                     e1y * e1z - e2y * e2z};
                const float wx[5] = {0.5f * (2.f * e1x * e2x - ex33), e1x * e2y + e2x * e1y, e1x * e2z + e2x * e1z,
                                     0.5f * (2.f * e1y * e2y - ex33), e1y * e2z + e2y * e1z};
                const float f = st == 0 ? src0 : src1;
#pragma unroll
                for (int qq = 0; qq < 5; qq++) {
                    const float2 sv = sm[G::idx(qq, slot, w)];
                    tp.x += wp[qq] * sv.x;
                    tp.y += wp[qq] * sv.y;
                    tx.x += wx[qq] * sv.x;
                    tx.y += wx[qq] * sv.y;
                }
                tp.x *= f; tp.y *= f; tx.x *= f; tx.y *= f;
            }
            if (st == 0) {
                t0[q][0] = tp;
                t0[q][1] = tx;
            } else if (kz < nz && m2 != 0.f) {
                const size_t gi = ((size_t)kx * N + j) * nz + kz;
                const float kk0 = m2 * n0f, kk1 = m2 * n1f;
                const float2 T1[2] = {tp, tx};
#pragma unroll
                for (int p = 0; p < 2; p++) {
                    const float2 h0 = Gm[(size_t)p * M + gi], l0 = Gm[(size_t)(2 + p) * M + gi];
                    float2 hn, ln;
#pragma unroll
                    for (int ri = 0; ri < 2; ri++) {
                        const float hv = ri ? h0.y : h0.x, lv = ri ? l0.y : l0.x;
                        const float Ta = ri ? t0[q][p].y : t0[q][p].x, Tb = ri ? T1[p].y : T1[p].x;
                        // stage 1: evolve_perts(0, 1, dt/2)
                        const float ld0 = -kk0 * hv - c3H0 * lv + Ta;
                        const float h1 = hv + hdt * lv;
                        const float l1 = lv + hdt * ld0;
                        // stage 2: evolve_perts(1, 0, dt)
                        const float ld1 = -kk1 * h1 - c3H1 * l1 + Tb;
                        (ri ? hn.y : hn.x) = hv + dt * l1;
                        (ri ? ln.y : ln.x) = lv + dt * ld1;
                    }
                    Gm[(size_t)p * M + gi] = hn;
                    Gm[(size_t)(2 + p) * M + gi] = ln;
                }
            }
        }
    }
    }
}

}  // namespace ksf
}  // namespace gabe
