// Tensor-perturbation update in Fourier space: one pass per step.
//
// The reference, per step, calls evolve_perts twice (g2evolutionpert.cpp:
// 343-455): each call projects the transformed source onto its
// transverse-traceless part T = dx^3 Lambda(k^) S (fft_stresstensor,
// :203-321) and takes one RK2 stage of  hdot = l,  ldot = -k^2/a^2 h
// - 3 (adot/a) l + 2 (8 pi/a^2) T  (derivs, :459-516) for all six
// components of h and l, with k^2 = |n|^2 (2 pi/L)^2.
//
// Storage.  h and l start at zero (g2main.cpp:58-95) and are driven only by
// T, which is transverse-traceless, through an equation whose coefficients
// depend on |k| alone -- so h_ij and l_ij stay TT and are fixed by two
// polarization amplitudes per k-point:  X_ij = sum_p eps^p_ij X_p  with
// eps^+ = e1 e1 - e2 e2, eps^x = e1 e2 + e2 e1 ({e1, e2, k^} orthonormal)
// and X_p = eps^p : X / 2.  The device keeps (h+, hx, l+, lx) -- 8 reals per
// k-point instead of 24 -- and converts to the reference's 12-component
// layout only at upload/download.  The source needs only five transformed
// components per stage (11, 12, 13, 22, 23): it is traceless in real space
// and eps^p is traceless, so S33 = -S11 - S22 gives eps^p : S exactly.
//
// Per k-point this kernel reads both stages' transformed sources and the
// four amplitudes once, forms T_p = dx^3 eps^p : S / 2 for both stages in
// registers, takes both RK2 stages and writes the amplitudes back; T_gw,
// h[1] and l[1] never exist in memory.  k = 0 carries no TT part (the
// reference zeroes T there, :319-321) and stays zero.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace gabe {

template <typename T>
struct Cplx {
    T re, im;
};

struct KspaceArgs {
    const void *S;   // complex half-spectra [10][N][N][N/2+1]: stage-0 11,12,13,22,23 then stage-1
    void *G;         // complex amplitudes [4][N][N][N/2+1]: h+, hx, l+, lx
    const DevScalars *sc;
    LatticeConsts c;
    int slot;        // which step's scalars (DevScalars::gw) to use
};

// Polarization tensors of the integer wave vector n (n != 0): the six
// components 11,12,13,22,23,33 of eps^+ and eps^x.
__host__ __device__ inline void pol_tensors(int px, int py, int pz, double ep[6], double ex[6]) {
    const double m = sqrt((double)px * px + (double)py * py + (double)pz * pz);
    const double kx = px / m, ky = py / m, kz = pz / m;
    // reference axis: the one least aligned with k
    const double ax = fabs(kx), ay = fabs(ky), az = fabs(kz);
    const int r = (ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2);
    const double kr = r == 0 ? kx : (r == 1 ? ky : kz);
    double e1x = (r == 0 ? 1.0 : 0.0) - kr * kx, e1y = (r == 1 ? 1.0 : 0.0) - kr * ky,
           e1z = (r == 2 ? 1.0 : 0.0) - kr * kz;
    const double n1 = 1.0 / sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    e1x *= n1; e1y *= n1; e1z *= n1;
    const double e2x = ky * e1z - kz * e1y, e2y = kz * e1x - kx * e1z, e2z = kx * e1y - ky * e1x;
    ep[0] = e1x * e1x - e2x * e2x; ep[1] = e1x * e1y - e2x * e2y; ep[2] = e1x * e1z - e2x * e2z;
    ep[3] = e1y * e1y - e2y * e2y; ep[4] = e1y * e1z - e2y * e2z; ep[5] = e1z * e1z - e2z * e2z;
    ex[0] = 2. * e1x * e2x; ex[1] = e1x * e2y + e2x * e1y; ex[2] = e1x * e2z + e2x * e1z;
    ex[3] = 2. * e1y * e2y; ex[4] = e1y * e2z + e2y * e1z; ex[5] = 2. * e1z * e2z;
}

// The same in FP32 (for the FP32 path's k-space update): the reference axis
// is chosen by comparing the integer components, which orders them exactly as
// the FP64 form's |k_i| / |n| do, so both forms take the same basis; e1, e2
// then carry FP32 rounding (~1e-7 relative).
__device__ inline void pol_tensors32(int px, int py, int pz, float ep[6], float ex[6]) {
    const float inv = rsqrtf((float)(px * px + py * py + pz * pz));
    const float kx = px * inv, ky = py * inv, kz = pz * inv;
    const int ax = abs(px), ay = abs(py), az = abs(pz);
    const int r = (ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2);
    const float kr = r == 0 ? kx : (r == 1 ? ky : kz);
    float e1x = (r == 0 ? 1.f : 0.f) - kr * kx, e1y = (r == 1 ? 1.f : 0.f) - kr * ky, e1z = (r == 2 ? 1.f : 0.f) - kr * kz;
    const float n1 = rsqrtf(e1x * e1x + e1y * e1y + e1z * e1z);
    e1x *= n1; e1y *= n1; e1z *= n1;
    const float e2x = ky * e1z - kz * e1y, e2y = kz * e1x - kx * e1z, e2z = kx * e1y - ky * e1x;
    ep[0] = e1x * e1x - e2x * e2x; ep[1] = e1x * e1y - e2x * e2y; ep[2] = e1x * e1z - e2x * e2z;
    ep[3] = e1y * e1y - e2y * e2y; ep[4] = e1y * e1z - e2y * e2z; ep[5] = e1z * e1z - e2z * e2z;
    ex[0] = 2.f * e1x * e2x; ex[1] = e1x * e2y + e2x * e1y; ex[2] = e1x * e2z + e2x * e1z;
    ex[3] = 2.f * e1y * e2y; ex[4] = e1y * e2z + e2y * e1z; ex[5] = 2.f * e1z * e2z;
}

// eps : S / 2 for a symmetric traceless S given by (S11, S12, S13, S22, S23).
template <typename T>
__device__ __forceinline__ T pol_contract(const T *w, const T *S) {
    return w[0] * S[0] + w[1] * S[1] + w[2] * S[2] + w[3] * S[3] + w[4] * S[4];
}

// derivs() coefficients (g2evolutionpert.cpp:486-501) of both RK2 stages of
// one step, from the scale factor and its derivative at the two stages.
template <typename T>
struct KsCoef {
    double norm0, norm1;  // k^2 / a^2 per |n|^2
    T c3H0, c3H1, src0, src1, hdt, dt;
};

template <typename T>
__device__ __forceinline__ KsCoef<T> ks_coef(const LatticeConsts &c, const double *g4) {
    const double a0 = g4[0], ad0 = g4[1], a1 = g4[2], ad1 = g4[3];
    KsCoef<T> k;
    k.norm0 = c.k2norm_c / a0 / a0;
    k.norm1 = c.k2norm_c / a1 / a1;
    const double om0 = c.eight_pi / a0 / a0, om1 = c.eight_pi / a1 / a1;
    k.c3H0 = (T)(3. * ad0 / a0);
    k.c3H1 = (T)(3. * ad1 / a1);
    k.src0 = (T)(2. * om0 * c.normmm);
    k.src1 = (T)(2. * om1 * c.normmm);
    k.hdt = (T)c.half_dt;
    k.dt = (T)c.dt;
    return k;
}

// Both RK2 stages of the amplitudes g[4] (h+, hx, l+, lx) of the k-point
// with integer wave vector (px, py, kzi), driven by its transformed
// sources s[10] (stage-0 11,12,13,22,23, then stage 1); g is updated in
// place.  k = 0 has no TT part and is left as it is.
// P: precision of the polarization tensors (double, or float for POL32).
template <typename T, bool POL32 = false>
__device__ __forceinline__ void kspace_update_vals(const KsCoef<T> &kc, int px, int py, int kzi, const Cplx<T> (&s)[10],
                                                   Cplx<T> (&g)[4]) {
    const double m2 = ((double)px * px + (double)py * py) + (double)kzi * kzi;
    if (m2 == 0.0) return;  // no TT mode at k = 0; its amplitudes stay zero
    using P = typename std::conditional<POL32, float, double>::type;
    P ep[6], ex[6];
    if constexpr (POL32) pol_tensors32(px, py, kzi, ep, ex);
    else pol_tensors(px, py, kzi, ep, ex);
    // weights of (S11, S12, S13, S22, S23) in eps:S/2 with S33 = -S11-S22
    const P half = (P)0.5;
    const T wp[5] = {(T)(half * (ep[0] - ep[5])), (T)ep[1], (T)ep[2], (T)(half * (ep[3] - ep[5])), (T)ep[4]};
    const T wx[5] = {(T)(half * (ex[0] - ex[5])), (T)ex[1], (T)ex[2], (T)(half * (ex[3] - ex[5])), (T)ex[4]};
    const T kk0 = (T)(m2 * kc.norm0), kk1 = (T)(m2 * kc.norm1);
    T Tp[2][2][2];  // [stage][pol][re/im], already times 2 (8 pi/a^2) dx^3
#pragma unroll
    for (int st = 0; st < 2; st++) {
        T sr[5], si[5];
#pragma unroll
        for (int q = 0; q < 5; q++) { sr[q] = s[5 * st + q].re; si[q] = s[5 * st + q].im; }
        const T f = st == 0 ? kc.src0 : kc.src1;
        Tp[st][0][0] = f * pol_contract(wp, sr);
        Tp[st][0][1] = f * pol_contract(wp, si);
        Tp[st][1][0] = f * pol_contract(wx, sr);
        Tp[st][1][1] = f * pol_contract(wx, si);
    }
#pragma unroll
    for (int p = 0; p < 2; p++) {
        Cplx<T> hn, ln;
#pragma unroll
        for (int ri = 0; ri < 2; ri++) {
            const T h0 = ri ? g[p].im : g[p].re, l0 = ri ? g[2 + p].im : g[2 + p].re;
            // stage 1: evolve_perts(0, 1, dt/2)
            const T ld0 = -kk0 * h0 - kc.c3H0 * l0 + Tp[0][p][ri];
            const T h1 = h0 + kc.hdt * l0;
            const T l1 = l0 + kc.hdt * ld0;
            // stage 2: evolve_perts(1, 0, dt)
            const T ld1 = -kk1 * h1 - kc.c3H1 * l1 + Tp[1][p][ri];
            (ri ? hn.im : hn.re) = h0 + kc.dt * l1;
            (ri ? ln.im : ln.re) = l0 + kc.dt * ld1;
        }
        g[p] = hn;
        g[2 + p] = ln;
    }
}

// The same for the k-point stored at element idx of arrays of M points:
// sources Sc [10][M], amplitudes G [4][M].
template <typename T>
__device__ __forceinline__ void kspace_update(const KsCoef<T> &kc, int px, int py, int kzi, size_t M,
                                              const Cplx<T> *Sc, Cplx<T> *G, size_t idx) {
    Cplx<T> s[10], g[4];
#pragma unroll
    for (int q = 0; q < 10; q++) s[q] = Sc[(size_t)q * M + idx];
#pragma unroll
    for (int q = 0; q < 4; q++) g[q] = G[(size_t)q * M + idx];
    if (px == 0 && py == 0 && kzi == 0) return;
    kspace_update_vals<T>(kc, px, py, kzi, s, g);
#pragma unroll
    for (int q = 0; q < 4; q++) G[(size_t)q * M + idx] = g[q];
}

// k-point idx of the half spectrum [N][N][N/2+1] (M points).
template <typename T>
__device__ __forceinline__ void kspace_point(const KsCoef<T> &kc, int N, size_t M, const Cplx<T> *Sc, Cplx<T> *G,
                                             size_t idx) {
    const int nz = N / 2 + 1;
    const int kzi = (int)(idx % nz);
    const size_t t = idx / nz;
    const int j = (int)(t % N), i = (int)(t / N);
    const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
    kspace_update<T>(kc, px, py, kzi, M, Sc, G, idx);
}

template <typename T>
__global__ void __launch_bounds__(256) kspace_kernel(KspaceArgs args) {
    const LatticeConsts &c = args.c;
    const int N = c.N;
    const size_t M = (size_t)N * N * (N / 2 + 1);
    const KsCoef<T> kc = ks_coef<T>(c, args.sc->gw[args.slot]);
    const Cplx<T> *Sc = static_cast<const Cplx<T> *>(args.S);
    Cplx<T> *G = static_cast<Cplx<T> *>(args.G);
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)gridDim.x * blockDim.x)
        kspace_point<T>(kc, N, M, Sc, G, idx);
}

// Element of the amplitude arrays that holds k-point (i, j, kz) of the half
// spectrum: [i][j][kz] (the library r2c's order), or [kz][j][i] for the
// transposed transform of fftt.cuh (gt = 1).
__host__ __device__ inline size_t g_index(int i, int j, int kz, int N, int gt) {
    return gt ? ((size_t)kz * N + j) * N + i : ((size_t)i * N + j) * (N / 2 + 1) + kz;
}

// ---------------------------------------------------------------------------
// conversions between the reference's 12-component layout (FP64 host data,
// staged in device memory as [12][cnt]) and the amplitudes, for k-points
// m0 .. m0+cnt-1 of the half spectrum.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void gw_pack_kernel(const double *src, size_t cnt, size_t m0, int N, size_t M, Cplx<T> *G, int which,
                               double *norms /* [2]: |X|^2, |X - TT(X)|^2 */, int gt) {
    const int nz = N / 2 + 1;
    double nrm = 0., res = 0.;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
        const size_t idx = m0 + q;
        const int kzi = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = (int)(t % N), i = (int)(t / N);
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        double X[2][6];  // [re/im][component]
#pragma unroll
        for (int c6 = 0; c6 < 6; c6++) {
            X[0][c6] = src[(size_t)(2 * c6) * cnt + q];
            X[1][c6] = src[(size_t)(2 * c6 + 1) * cnt + q];
        }
        Cplx<T> ap = {0, 0}, ax = {0, 0};
        double ep[6] = {0, 0, 0, 0, 0, 0}, ex[6] = {0, 0, 0, 0, 0, 0};
        double A[2][2] = {{0, 0}, {0, 0}};  // [pol][re/im]
        if (px || py || kzi) {
            pol_tensors(px, py, kzi, ep, ex);
            const double w[6] = {1, 2, 2, 1, 2, 1};  // eps:X over all 9 entries
#pragma unroll
            for (int ri = 0; ri < 2; ri++) {
                double sp = 0., sx = 0.;
#pragma unroll
                for (int c6 = 0; c6 < 6; c6++) {
                    sp += w[c6] * ep[c6] * X[ri][c6];
                    sx += w[c6] * ex[c6] * X[ri][c6];
                }
                A[0][ri] = 0.5 * sp;
                A[1][ri] = 0.5 * sx;
            }
            ap = {(T)A[0][0], (T)A[0][1]};
            ax = {(T)A[1][0], (T)A[1][1]};
        }
        const double w9[6] = {1, 2, 2, 1, 2, 1};
#pragma unroll
        for (int ri = 0; ri < 2; ri++)
#pragma unroll
            for (int c6 = 0; c6 < 6; c6++) {
                const double r = X[ri][c6] - (ep[c6] * A[0][ri] + ex[c6] * A[1][ri]);
                nrm += w9[c6] * X[ri][c6] * X[ri][c6];
                res += w9[c6] * r * r;
            }
        const size_t gi = g_index(i, j, kzi, N, gt);
        G[(size_t)(2 * which) * M + gi] = ap;
        G[(size_t)(2 * which + 1) * M + gi] = ax;
    }
    // block sums then one atomic pair per block (a check, order is irrelevant)
    __shared__ double sred[8 * 2];
    double v[2] = {nrm, res};
    block_reduce<2>(v, sred);
    if (threadIdx.x == 0) {
        atomicAdd(norms, v[0]);
        atomicAdd(norms + 1, v[1]);
    }
}

template <typename T>
__global__ void gw_unpack_kernel(const Cplx<T> *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst,
                                 int gt) {
    const int nz = N / 2 + 1;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
        const size_t idx = m0 + q;
        const int kzi = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = (int)(t % N), i = (int)(t / N);
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        double ep[6] = {0, 0, 0, 0, 0, 0}, ex[6] = {0, 0, 0, 0, 0, 0};
        if (px || py || kzi) pol_tensors(px, py, kzi, ep, ex);
        const size_t gi = g_index(i, j, kzi, N, gt);
        const Cplx<T> ap = G[(size_t)(2 * which) * M + gi], ax = G[(size_t)(2 * which + 1) * M + gi];
#pragma unroll
        for (int c6 = 0; c6 < 6; c6++) {
            dst[(size_t)(2 * c6) * cnt + q] = ep[c6] * (double)ap.re + ex[c6] * (double)ax.re;
            dst[(size_t)(2 * c6 + 1) * cnt + q] = ep[c6] * (double)ap.im + ex[c6] * (double)ax.im;
        }
    }
}

}  // namespace gabe
