// FP32 sweep A with the GW sources leaving the kernel transformed along k.
//
// The reference transforms each source array with a 3-D r2c
// (fft_stresstensor, g2evolutionpert.cpp:183-195); its first pass, along k,
// needs whole rows.  Here a block owns two whole rows (j0, j0+1) of every
// plane of its chunk, so the source rows it computes are complete in shared
// memory and are transformed before they are written: the sources reach HBM
// once, as half spectra along k, and the GW chain only runs the passes along
// j and i (fft3d.cuh col_fft_kernel).  This removes one read and one write
// of the ten source arrays per step.
//
// Per plane:
//   * the per-site update of sweep A (sweep32.cuh site_a32: energies as FP32
//     moments folded into FP64, sources of both stages) for the block's
//     2 N sites, two per thread, from a ring of S plane slots filled by
//     cp.async (rows j0-1 .. j0+2 of the four input arrays, each row with
//     its periodic k neighbours);
//   * the ten source rows of each of the two rows go to a shared buffer in
//     the row kernel's layout, and the pair (row j0, row j0+1) of every
//     component is transformed as one complex row exactly as
//     f3d::row_r2c_kernel does (same four-step split, twiddles, order of
//     operations and Hermitian separation), so the written half spectra are
//     bit for bit those of the separate row pass.
#pragma once

#include "fft3d.cuh"

namespace gabe {
namespace s32 {

template <int N>
struct RowsGeom {
    static constexpr int T = N;                 // threads: N/2 pairs of sites per row, two rows
    static constexpr int TK2 = N / 2, PK = N + 4, ROWS = 4;  // ring rows j0-1, j0, j0+1, j0+2
    static constexpr int ARR = ROWS * PK, SLOT = 4 * ARR;
    static constexpr int S = 5;                 // ring slots: two planes in flight
    static constexpr int NP = 2 * kSrc;         // components = row pairs transformed per plane
    static constexpr int FBUF = 2 * NP * N;     // source rows [component][row][N], pair-swizzled
    static constexpr size_t SMEM_BYTES = (size_t)(S * SLOT + FBUF + 2 * N) * sizeof(float);
    static constexpr int MINB = 512 / T;        // blocks per SM the 128-register budget allows
};

template <int N>
__global__ void __launch_bounds__(RowsGeom<N>::T, RowsGeom<N>::MINB) sweep32_rows_kernel(StencilArgs args) {
    using G = RowsGeom<N>;
    using RG = f3d::RowGeom<N>;
    constexpr int MODE = MODE_A_GW;
    constexpr int T = G::T, TK2 = G::TK2, PK = G::PK, S = G::S, NP = G::NP;
    constexpr int L1 = RG::L1, L2 = RG::L2, RP = N + 2, NH = N / 2 + 1, NN = N * N;
    constexpr int NT2 = (NP * L2 + T - 1) / T;
    extern __shared__ __align__(16) float smem[];
    float *ring = smem;
    float *fb = smem + S * G::SLOT;
    float2 *tw = reinterpret_cast<float2 *>(fb + G::FBUF);
    __shared__ double sred[(T / 32) * kNV];
    __shared__ int sflag;

    const LatticeConsts &c = args.c;
    const int tid = threadIdx.x, tx = tid % TK2, r = tid / TK2;
    const int j0 = 2 * blockIdx.x;
    const int i0 = blockIdx.y * args.ci, i1 = min(i0 + args.ci, N);
    const int n3 = N * N * N;
    const float *X = static_cast<const float *>(args.X), *D = static_cast<const float *>(args.D);
    const float *src[4] = {X, X + n3, D, D + n3};
    float *Sg = static_cast<float *>(args.S);
    f3d::twiddles<N>(tw);

    const int k = 2 * tx, j = j0 + r;
    const int jm = wrapi(j0 - 1, N), jp = wrapi(j0 + 2, N);
    const int o_own = j * N + k, so_own = (r + 1) * PK + 2 + 2 * tx;
    // every thread also copies one pair of a halo row (r = 0: row j0-1, r = 1: row j0+2)
    const int h_go = (r ? jp : jm) * N + k, h_so = (r ? 3 * PK : 0) + 2 + 2 * tx;
    // threads 0..3: the periodic k neighbours of the own rows (column 1 = k N-1, column N+2 = k 0)
    int kh_go = -1, kh_so = 0;
    if (tid < 4) {
        const int rr = tid >> 1, e = tid & 1;
        kh_go = (j0 + rr) * N + (e ? 0 : N - 1);
        kh_so = (rr + 1) * PK + (e ? N + 2 : 1);
    }
    auto issue = [&](int p, int sl) {  // plane p (wrapped) into slot sl
        float *slot = ring + sl * G::SLOT;
        const int pb = wrapi(p, N) * NN;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            float *sa = slot + a * G::ARR;
            const float *g = src[a] + pb;
            cp_async8(sa + so_own, g + o_own);
            cp_async8(sa + h_so, g + h_go);
            if (kh_go >= 0) cp_async4(sa + kh_so, g + kh_go);
        }
    };
    auto next_slot = [](int sl) { return sl + 1 == S ? 0 : sl + 1; };

    const Site32 s = site32_consts<MODE>(c, args.sc);
    double acc[kNV];
#pragma unroll
    for (int q = 0; q < kNV; q++) acc[q] = 0.;
    Moments mom;
    zero(mom);
    int ngroup = 0;

#pragma unroll
    for (int q = 0; q < S - 1; q++) {
        const int p = i0 - 1 + q;
        if (p <= i1) issue(p, q);
        cp_commit();
    }
    int s_pr = 0, s_cu = 1, s_nx = 2, s_is = S - 1;
    float2 pr[4], cu[4];
    for (int i = i0; i < i1; i++) {
        cp_wait<S - 4>();
        __syncthreads();  // plane i+1 landed; the previous plane's transform is fully consumed
        if (i + S - 2 <= i1) issue(i + S - 2, s_is);
        cp_commit();
        {
            const float *sc = ring + s_cu * G::SLOT;
            const float *sn = ring + s_nx * G::SLOT;
            if (i == i0) {
                const float *sp = ring + s_pr * G::SLOT;
#pragma unroll
                for (int a = 0; a < 4; a++) {
                    pr[a] = *reinterpret_cast<const float2 *>(sp + a * G::ARR + so_own);
                    cu[a] = *reinterpret_cast<const float2 *>(sc + a * G::ARR + so_own);
                }
            }
            Nb7<float> nb[4][2];
            float2 nx[4];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const int ao = a * G::ARR + so_own;
                nx[a] = *reinterpret_cast<const float2 *>(sn + ao);
                const float2 up = *reinterpret_cast<const float2 *>(sc + ao + PK);
                const float2 dn = *reinterpret_cast<const float2 *>(sc + ao - PK);
                const float lm = sc[ao - 1], rp = sc[ao + 2];
                // reference neighbour order: centre, i+1, i-1, j+1, j-1, k+1, k-1
                nb[a][0] = Nb7<float>{{cu[a].x, nx[a].x, pr[a].x, up.x, dn.x, cu[a].y, lm}};
                nb[a][1] = Nb7<float>{{cu[a].y, nx[a].y, pr[a].y, up.y, dn.y, rp, cu[a].x}};
            }
            float s0[2][kSrc] = {}, s1[2][kSrc] = {};
#pragma unroll
            for (int v = 0; v < 2; v++) site_a32<MODE>(c, s, nb[0][v], nb[1][v], nb[2][v], nb[3][v], mom, s0[v], s1[v]);
            if (++ngroup == kGroup || i == i1 - 1) {
                fold<MODE>(s.mt, s.q3f, 2 * ngroup, mom, acc);
                ngroup = 0;
            }
            // source rows into the transform buffer: component q (stage 0) and kSrc + q (stage 1)
            const int fo = r * N + RG::phys(k);
#pragma unroll
            for (int q = 0; q < kSrc; q++) {
                *reinterpret_cast<float2 *>(fb + (2 * q) * N + fo) = make_float2(s0[0][q], s0[1][q]);
                *reinterpret_cast<float2 *>(fb + (2 * (kSrc + q)) * N + fo) = make_float2(s1[0][q], s1[1][q]);
            }
#pragma unroll
            for (int a = 0; a < 4; a++) {
                pr[a] = cu[a];
                cu[a] = nx[a];
            }
        }
        __syncthreads();  // all source rows of plane i are in the buffer
        // four-step pass 1: L2-point FFTs over n2 (stride L1), twiddle W_N^(n1 k2), in place
#pragma unroll
        for (int t0 = 0; t0 < NP * L1; t0 += T) {
            const int t = t0 + tid, p = t / L1, n1 = t % L1;
            if (t >= NP * L1) break;
            float *re = fb + 2 * p * N, *im = re + N;
            float2 x[L2];
#pragma unroll
            for (int n2 = 0; n2 < L2; n2++) {
                const int a = RG::phys(n1 + L1 * n2);
                x[n2] = make_float2(re[a], im[a]);
            }
            pfft::fft_reg<L2>(x);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) {
                const float2 y = k2 ? pfft::cmul(x[k2], tw[k2 * L1 + n1]) : x[k2];
                const int a = RG::phys(n1 + L1 * k2);
                re[a] = y.x;
                im[a] = y.y;
            }
        }
        __syncthreads();
        // pass 2: L1-point FFTs over n1, back in natural order k = k2 + L2 k1
        {
            float2 y[NT2][L1];
#pragma unroll
            for (int q = 0; q < NT2; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                if (t < NP * L2) {
                    const float *re = fb + 2 * p * N, *im = re + N;
#pragma unroll
                    for (int n1 = 0; n1 < L1; n1++) {
                        const int a = RG::phys(n1 + L1 * k2);
                        y[q][n1] = make_float2(re[a], im[a]);
                    }
                    pfft::fft_reg<L1>(y[q]);
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < NT2; q++) {
                const int t = q * T + tid, p = t / L2, k2 = t % L2;
                if (t < NP * L2) {
                    float *re = fb + 2 * p * N, *im = re + N;
#pragma unroll
                    for (int k1 = 0; k1 < L1; k1++) {
                        const int a = RG::phys(k2 + L2 * k1);
                        re[a] = y[q][k1].x;
                        im[a] = y[q][k1].y;
                    }
                }
            }
        }
        __syncthreads();
        // separate each pair into rows j0 and j0+1: N/2+1 complex values each, in place in
        // the N+2 reals of the source row
        for (int t = tid; t < NP * NH; t += T) {
            const int p = t / NH, kk = t % NH, km = (N - kk) & (N - 1);
            const float *re = fb + 2 * p * N, *im = re + N;
            const int ak = RG::phys(kk & (N - 1)), am = RG::phys(km);
            const float zr = re[ak], zi = im[ak], mr = re[am], mi = im[am];
            float *g = Sg + ((size_t)(p * N + i) * N + j0) * RP;
            __stcs(reinterpret_cast<float2 *>(g) + kk, make_float2(0.5f * (zr + mr), 0.5f * (zi - mi)));
            __stcs(reinterpret_cast<float2 *>(g + RP) + kk, make_float2(0.5f * (zi + mi), 0.5f * (mr - zr)));
        }
        s_pr = s_cu;
        s_cu = s_nx;
        s_nx = next_slot(s_nx);
        s_is = next_slot(s_is);
    }
    cp_wait<0>();

    const int bid = blockIdx.x + gridDim.x * blockIdx.y;
    block_reduce<kNV>(acc, sred);
    if (tid == 0)
        for (int q = 0; q < kNV; q++) args.partials[(size_t)bid * kNV + q] = acc[q];
    if (!last_block_done(args.counter, &sflag)) return;
    double tot[kNV];
    sum_partials<kNV>(args.partials, gridDim.x * gridDim.y, tot, sred);
    if (tid == 0) {
        finish_a<float, MODE>(c, args.sc, tot, args.slot);
        *args.counter = 0u;
    }
}

}  // namespace s32
}  // namespace gabe
