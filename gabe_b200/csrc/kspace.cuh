// Tensor-perturbation update in Fourier space: one pass per step.
//
// The reference, per step, calls evolve_perts twice (g2evolutionpert.cpp:
// 343-455): each call projects the transformed source onto its
// transverse-traceless part into T_gw[s] (fft_stresstensor, :203-321) and
// takes one RK2 stage of  hdot = l,  ldot = -k^2/a^2 h - 3 (adot/a) l
// + 2 (8 pi/a^2) T  (derivs, :459-516) with the continuum k^2 = |n|^2
// (2 pi/L)^2.  Both stages touch only their own k-point, so this kernel
// reads h0, l0 and the two transformed sources once, forms both projections
// in registers, takes both stages, and writes h0, l0 back: T_gw, h[1] and
// l[1] never exist in memory.
//
// Projection: T = dx^3 Lambda(k^) S with Lambda S = P S P - 1/2 P tr(P S),
// P = 1 - k^ k^T, evaluated as S - k u^T - u k^T + s k k^T
// - 1/2 (tr S - s) P with u = S k^, s = k^.u; for a traceless S this equals
// the reference's explicit formulas term by term (checked against them in
// the tests).  The k = 0 mode is set to zero as :319-321 does.
#pragma once

#include "common.cuh"

namespace gabe {

struct KspaceArgs {
    const void *S;   // complex half-spectra [12][N][N][N/2+1]
    void *h, *l;     // [12][N][N][N/2+1]
    const DevScalars *sc;
    LatticeConsts c;
};

template <typename T>
struct Cplx { T re, im; };

template <typename T>
__device__ __forceinline__ void tt_project(T kx, T ky, T kz, const T *S, T nm, T *out) {
    // S, out: 6 symmetric components 11,12,13,22,23,33 (one of re/im)
    const T S11 = S[0], S12 = S[1], S13 = S[2], S22 = S[3], S23 = S[4], S33 = S[5];
    const T u1 = S11 * kx + S12 * ky + S13 * kz;
    const T u2 = S12 * kx + S22 * ky + S23 * kz;
    const T u3 = S13 * kx + S23 * ky + S33 * kz;
    const T s = kx * u1 + ky * u2 + kz * u3;
    const T g = T(0.5) * ((S11 + S22 + S33) - s);
    out[0] = nm * (S11 - T(2) * kx * u1 + s * kx * kx - g * (T(1) - kx * kx));
    out[1] = nm * (S12 - kx * u2 - u1 * ky + (s + g) * kx * ky);
    out[2] = nm * (S13 - kx * u3 - u1 * kz + (s + g) * kx * kz);
    out[3] = nm * (S22 - T(2) * ky * u2 + s * ky * ky - g * (T(1) - ky * ky));
    out[4] = nm * (S23 - ky * u3 - u2 * kz + (s + g) * ky * kz);
    out[5] = nm * (S33 - T(2) * kz * u3 + s * kz * kz - g * (T(1) - kz * kz));
}

template <typename T>
__global__ void __launch_bounds__(256) kspace_kernel(KspaceArgs args) {
    const LatticeConsts &c = args.c;
    const int N = c.N, nz = N / 2 + 1;
    const size_t M = (size_t)N * N * nz;
    const DevScalars *sc = args.sc;
    const double a0 = sc->a[0], ad0 = sc->adot[0], a1 = sc->a[1], ad1 = sc->adot[1];
    // derivs() coefficients (g2evolutionpert.cpp:486-501) for both stages
    const double norm0 = c.k2norm_c / a0 / a0, norm1 = c.k2norm_c / a1 / a1;
    const double om0 = c.eight_pi / a0 / a0, om1 = c.eight_pi / a1 / a1;
    const T c3H0 = (T)(3. * ad0 / a0), c3H1 = (T)(3. * ad1 / a1);
    const T two_om0 = (T)(2. * om0), two_om1 = (T)(2. * om1);
    const T hdt = (T)c.half_dt, dt = (T)c.dt, nm = (T)c.normmm;
    const Cplx<T> *Sc = static_cast<const Cplx<T> *>(args.S);
    T *H = static_cast<T *>(args.h), *Lh = static_cast<T *>(args.l);

    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)gridDim.x * blockDim.x) {
        const int kzi = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = (int)(t % N), i = (int)(t / N);
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        const double m2 = ((double)px * px + (double)py * py) + (double)kzi * kzi;
        const T kk0 = (T)(m2 * norm0), kk1 = (T)(m2 * norm1);
        T T0[12], T1[12];
        if (m2 == 0.0) {
#pragma unroll
            for (int q = 0; q < 12; q++) { T0[q] = T(0); T1[q] = T(0); }
        } else {
            const double inv = 1.0 / sqrt(m2);
            const T kx = (T)(px * inv), ky = (T)(py * inv), kz = (T)(kzi * inv);
            T sr[6], si[6], tr[6], ti[6];
#pragma unroll
            for (int st = 0; st < 2; st++) {
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const Cplx<T> v = Sc[(size_t)(6 * st + q) * M + idx];
                    sr[q] = v.re;
                    si[q] = v.im;
                }
                tt_project(kx, ky, kz, sr, nm, tr);
                tt_project(kx, ky, kz, si, nm, ti);
                T *dst = st == 0 ? T0 : T1;
#pragma unroll
                for (int q = 0; q < 6; q++) { dst[2 * q] = tr[q]; dst[2 * q + 1] = ti[q]; }
            }
        }
#pragma unroll
        for (int q = 0; q < 12; q++) {
            const size_t g = (size_t)q * M + idx;
            const T h0 = H[g], l0 = Lh[g];
            // stage 1: evolve_perts(0, 1, dt/2)
            const T ld0 = -kk0 * h0 - c3H0 * l0 + two_om0 * T0[q];
            const T h1 = h0 + hdt * l0;
            const T l1 = l0 + hdt * ld0;
            // stage 2: evolve_perts(1, 0, dt)
            const T ld1 = -kk1 * h1 - c3H1 * l1 + two_om1 * T1[q];
            H[g] = h0 + dt * l1;
            Lh[g] = l0 + dt * ld1;
        }
    }
}

}  // namespace gabe
