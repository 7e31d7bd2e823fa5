// FP32 stencil sweeps with a cp.async plane pipeline.
//
// Same sweeps as sweep_kernel (stencil.cuh: sweep A with the GW sources,
// sweep B, mode E0) and the same per-site arithmetic, with a data path built
// for HBM bandwidth rather than registers:
//
//   * a block owns a TK x TJ column tile (TK = 2 TK2 along k, two sites per
//     thread, 8-byte accesses) and marches along i over `ci` planes;
//   * every plane of the four input arrays (f phi, f chi, fdot phi, fdot chi)
//     -- the thread's own pair of sites plus the one-point j/k halo -- is
//     copied global -> shared with cp.async into a ring of S plane slots, S-3
//     planes ahead of the plane being computed, so each thread keeps three
//     planes of 8-byte loads in flight without holding them in registers;
//   * one barrier per plane: the slot of plane i-2 is refilled (plane i+S-2)
//     only after every thread has left plane i-1.
// Each input value crosses HBM once per sweep (halo points are re-read from
// L2 by the neighbouring tiles).
#pragma once

#include "stencil.cuh"

namespace gabe {
namespace s32 {

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
// 16 bytes, cached in L2 only.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}

// Shared-memory plane slot: [4 arrays][TJ + 2 rows][PK columns]; column C0-1
// is the k0-1 halo, columns C0 .. C0+TK-1 the tile, column C0+TK the k0+TK
// halo.  Narrow (W16 false): C0 = 2, PK = TK + 4, every thread's pair on an
// 8-byte boundary, one 8-byte copy per thread.  Wide (W16): C0 = 4,
// PK = TK + 8, rows 16-byte multiples, so the pairs of threads 2m and 2m+1
// land as one 16-byte copy (L2 only).  The single-lattice and ensemble
// sweeps use the wide slots (at 512^3 sweep A 1.81 ms against 1.83 narrow,
// sweep B 0.835 with five wide slots against 0.87 with six narrow ones).
template <int TK2, int TJ, bool W16 = false>
struct Ring {
    static constexpr int TK = 2 * TK2, PK = TK + (W16 ? 8 : 4), ROWS = TJ + 2, C0 = W16 ? 4 : 2;
    static constexpr int ARR = ROWS * PK, SLOT = 4 * ARR;
};

// Per-launch constants of the FP32 site update (stage scalars as floats,
// homogeneous trajectory).
struct Site32 {
    MeanTraj mt;
    MeanF m0, m1;
    float ia02f, ia12f, c3H0f, c3H1f, hf, dtf, inv_dx2f, qsf, q3f;  // qsf = dn / 4
};

template <int MODE>
__device__ __forceinline__ Site32 site32_consts(const LatticeConsts &c, const DevScalars *scp) {
    Site32 s{};
    const double h = c.half_dt, a0 = scp->a[0];
    s.mt = mean_traj(c, scp);
    s.m0 = mean_f(c, s.mt.fb0);
    s.m1 = mean_f(c, s.mt.fb1);
    s.ia02f = (float)(1.0 / (a0 * a0));
    s.hf = (float)h;
    s.dtf = (float)c.dt;
    s.inv_dx2f = (float)(1.0 / c.inv_dx2_div);
    s.qsf = (float)(0.25 * c.dn);
    s.q3f = (float)(-h * 3. / a0);
    if constexpr (MODE == MODE_B) {
        const double ad0 = scp->adot[0], a1 = scp->a[1], ad1 = scp->adot[1];
        s.ia12f = (float)(1.0 / (a1 * a1));
        s.c3H0f = (float)((3. * ad0) / a0);
        s.c3H1f = (float)((3. * ad1) / a1);
    }
    return s;
}

// Potential of the site functions: MODEL >= 0 fixes it at compile time (the
// single-lattice sweeps, one instantiation per model, no branch per site),
// -1 reads it from the lattice constants (the ensemble's mixed batches).
template <int MODEL>
__device__ __forceinline__ int site_model(const LatticeConsts &c) {
    return MODEL >= 0 ? MODEL : c.model;
}

// One site of sweep A / E0: adds to the moments, fills the sources.
template <int MODE, int MODEL = -1>
__device__ __forceinline__ void site_a32(const LatticeConsts &c, const Site32 &s, const Nb7<float> &fp,
                                         const Nb7<float> &fc, const Nb7<float> &dp, const Nb7<float> &dc,
                                         Moments &m, float (&s0)[kSrc], float (&s1)[kSrc]) {
    const int model = site_model<MODEL>(c);
    const Nb7<float> *f0[2] = {&fp, &fc}, *d0[2] = {&dp, &dc};
    float f1c[2];
    float P0[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, P1[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const Nb7<float> &ff = *f0[f], &dd = *d0[f];
        const float lap0 = lap32(ff, s.inv_dx2f);
        const float d = dd.v[0];
        m.a[f] += d;
        m.b = fmaf(d, d, m.b);
        m.g0 = fmaf(ff.v[0], lap0, m.g0);
        if constexpr (MODE != MODE_E0) {
            const Nb7<float> f1 = axpy7(ff, s.hf, dd);
            f1c[f] = f1.v[0];
            const float Pd = d + s.hf * (lap0 * s.ia02f - dv_diff32(s.m0, model, f, fp.v[0], fc.v[0]));
            m.c[f] += Pd;
            m.e = fmaf(Pd, Pd, m.e);
            m.f = fmaf(Pd, d, m.f);
            m.g1 = fmaf(f1.v[0], lap32(f1, s.inv_dx2f), m.g1);
            if constexpr (MODE == MODE_A_GW) {
                grad_prod_add(ff, P0);
                grad_prod_add(f1, P1);
            }
        }
    }
    if constexpr (MODE == MODE_A_GW) {
        source_from_prod(s.qsf, P0, s0);
        source_from_prod(s.qsf, P1, s1);
    }
    m.v0 += v_diff32(s.m0, model, fp.v[0], fc.v[0]);
    if constexpr (MODE != MODE_E0) m.v1 += v_diff32(s.m1, model, f1c[0], f1c[1]);
}

// One site of sweep B: the new field and momentum of both fields.
template <int MODEL = -1>
__device__ __forceinline__ void site_b32(const LatticeConsts &c, const Site32 &s, const Nb7<float> &fp,
                                         const Nb7<float> &fc, const Nb7<float> &dp, const Nb7<float> &dc,
                                         float (&xo)[2], float (&dout)[2]) {
    const int model = site_model<MODEL>(c);
    const Nb7<float> *f0[2] = {&fp, &fc}, *d0[2] = {&dp, &dc};
    const Nb7<float> f1[2] = {axpy7(fp, s.hf, dp), axpy7(fc, s.hf, dc)};
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const Nb7<float> &ff = *f0[f], &dd = *d0[f];
        const float lap0 = lap32(ff, s.inv_dx2f);
        const float dd0 = lap0 * s.ia02f - dv_diff32(s.m0, model, f, fp.v[0], fc.v[0]) - s.c3H0f * dd.v[0];
        const float d1c = dd.v[0] + s.hf * dd0;
        const float lap1 = lap32(f1[f], s.inv_dx2f);
        const float dd1 = lap1 * s.ia12f - dv_diff32(s.m1, model, f, f1[0].v[0], f1[1].v[0]) - s.c3H1f * d1c;
        xo[f] = ff.v[0] + s.dtf * d1c;
        dout[f] = dd.v[0] + s.dtf * dd1;
    }
}

// Threads per SM the register budget is sized for: sweep A with sources holds
// the most live values and runs two 256-thread blocks per SM without spills;
// the others fit three.
template <int MODE>
constexpr int sweep32_threads_per_sm() {
    return (MODE == MODE_A_GW || MODE == MODE_A) ? 512 : 768;
}

// Pointers and bounds of one column tile of one lattice.
struct Tile32 {
    const float *X, *D;  // fields and momenta of the current state, [2][N^3]
    float *Xo, *Do;      // new fields and momenta (sweep B)
    float *S;            // GW sources [10][N][N][N+2] (sweep A with sources; a slab: its own planes)
    int k0, j0, i0, i1;
    int planes;          // planes per field in X, D, Xo, Do (slab, no wrap along i); 0 = N, periodic
};

// The plane march of one TK x TJ tile over planes i0 .. i1-1 by a block of NT
// threads (NT >= TK2 TJ; threads beyond TK2 TJ only take part in the
// barriers).  Sweep A / E0 add the tile's folded sums to acc (per-thread
// partials, zero on idle threads); sweep B writes the new state.
template <int TK2, int TJ, int MODE, int S, int NT, int MODEL = -1, bool W16 = false>
__device__ __forceinline__ void march32(const LatticeConsts &c, const Site32 &s, const Tile32 &t, float *ring,
                                        double (&acc)[kNV]) {
    using Rg = Ring<TK2, TJ, W16>;
    constexpr int TK = Rg::TK, PK = Rg::PK, C0 = Rg::C0;
    static_assert(S >= 4, "ring needs planes i-1, i, i+1 and one in flight");
    static_assert(!W16 || TK2 % 2 == 0, "wide slots copy the pairs of threads 2m and 2m+1 of one row together");
    static_assert(TK2 * TJ >= 2 * TK2 + 2 * TJ, "enough threads for the halo copies");
    static_assert(NT >= TK2 * TJ, "block smaller than the tile");
    const int N = c.N;
    const int n3 = (t.planes ? t.planes : N) * N * N;  // < 2^31 for N <= 1024
    const int tid = threadIdx.x;
    const bool act = NT == TK2 * TJ || tid < TK2 * TJ;
    const int tx = tid % TK2, ty = tid / TK2;
    const int k0 = t.k0, j0 = t.j0, i0 = t.i0, i1 = t.i1;
    const int j = j0 + ty, k = k0 + 2 * tx;
    const float *src[4] = {t.X, t.X + n3, t.D, t.D + n3};

    // element offsets of the own pair and the halo points within a plane;
    // planes are p N^2
    const int NN = N * N;
    const int jm = wrapi(j0 - 1, N), jp = wrapi(j0 + TJ, N), km = wrapi(k0 - 1, N), kp = wrapi(k0 + TK, N);
    const int o_own = j * N + k;
    const int so_own = (ty + 1) * PK + C0 + 2 * tx;  // shared offset of the own pair within an array
    // halo duty, one copy per array: threads 0 .. 2 TK2 - 1 copy pairs of the
    // j0-1 and j0+TJ rows, the next 2 TJ threads single points of the k0-1 and
    // k0+TK columns
    int h_kind = 0, h_so = 0, h_go = 0;  // 0 none, 8 pair, 4 point
    if (tid < 2 * TK2) {
        const int r = tid / TK2, q = tid % TK2;
        h_kind = 8;
        h_so = (r ? (TJ + 1) * PK : 0) + C0 + 2 * q;
        h_go = (r ? jp : jm) * N + k0 + 2 * q;
    } else if (tid < 2 * TK2 + 2 * TJ) {
        const int r = (tid - 2 * TK2) / TJ, q = (tid - 2 * TK2) % TJ;
        h_kind = 4;
        h_so = (q + 1) * PK + (r ? TK + C0 : C0 - 1);
        h_go = (j0 + q) * N + (r ? kp : km);
    }
    auto issue = [&](int p, int sl) {  // plane p (wrapped) into slot sl
        if (!act) return;
        float *slot = ring + sl * Rg::SLOT;
        const int pb = (t.planes ? p : wrapi(p, N)) * NN;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            float *sa = slot + a * Rg::ARR;
            const float *g = src[a] + pb;
            if constexpr (W16) {
                // the pairs of threads 2m and 2m+1 as one 16-byte copy (k0 + 4m is 16-byte aligned)
                if ((tx & 1) == 0) cp_async16(sa + so_own, g + o_own);
            } else {
                cp_async8(sa + so_own, g + o_own);
            }
            // the energies-only sweep reads the momenta at the own sites only
            if (MODE == MODE_E0 && a >= 2) continue;
            if (h_kind == 8) cp_async8(sa + h_so, g + h_go);
            else if (h_kind == 4) cp_async4(sa + h_so, g + h_go);
        }
    };
    auto next_slot = [](int sl) { return sl + 1 == S ? 0 : sl + 1; };

    Moments mom;
    zero(mom);
    int ngroup = 0;  // planes in the current moment group

    // prologue: planes i0-1 .. i0+S-3 (one commit group each) into slots 0 .. S-2
#pragma unroll
    for (int q = 0; q < S - 1; q++) {
        const int p = i0 - 1 + q;
        if (p <= i1) issue(p, q);
        cp_commit();
    }
    // slots of planes i-1, i, i+1 and of the plane issued next (i+S-2)
    int s_pr = 0, s_cu = 1, s_nx = 2, s_is = S - 1;
    float2 pr[4], cu[4];  // own pair of planes i-1 and i
    // sources [10][planes][N][N+2]: the whole lattice, or a slab's own planes (plane i at i - 1)
    const int splanes = t.planes ? t.planes - 2 : N, sfirst = t.planes ? 1 : 0;
    const int sstride = splanes * N * (N + 2);  // one source component
    const int so_row = j * (N + 2) + k;
    for (int i = i0; i < i1; i++) {
        cp_wait<S - 4>();  // planes up to i+1 have landed (this thread's copies)
        __syncthreads();   // ... and everybody's; every thread has left plane i-1
        if (i + S - 2 <= i1) issue(i + S - 2, s_is);  // into the slot of plane i-2
        cp_commit();

        if (act) {
            const float *sc = ring + s_cu * Rg::SLOT;
            const float *sn = ring + s_nx * Rg::SLOT;
            if (i == i0) {
                const float *sp = ring + s_pr * Rg::SLOT;
#pragma unroll
                for (int a = 0; a < 4; a++) {
                    pr[a] = *reinterpret_cast<const float2 *>(sp + a * Rg::ARR + so_own);
                    cu[a] = *reinterpret_cast<const float2 *>(sc + a * Rg::ARR + so_own);
                }
            }
            Nb7<float> nb[4][2];  // [array][site]
            float2 nx[4];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const int ao = a * Rg::ARR + so_own;
                nx[a] = *reinterpret_cast<const float2 *>(sn + ao);
                const float2 up = *reinterpret_cast<const float2 *>(sc + ao + PK);
                const float2 dn = *reinterpret_cast<const float2 *>(sc + ao - PK);
                const float lm = sc[ao - 1], rp = sc[ao + 2];
                // reference neighbour order: centre, i+1, i-1, j+1, j-1, k+1, k-1
                nb[a][0] = Nb7<float>{{cu[a].x, nx[a].x, pr[a].x, up.x, dn.x, cu[a].y, lm}};
                nb[a][1] = Nb7<float>{{cu[a].y, nx[a].y, pr[a].y, up.y, dn.y, rp, cu[a].x}};
            }
            if constexpr (MODE == MODE_B) {
                float xo[2][2], dout[2][2];  // [site][field]
#pragma unroll
                for (int v = 0; v < 2; v++) {
                    site_b32<MODEL>(c, s, nb[0][v], nb[1][v], nb[2][v], nb[3][v], xo[v], dout[v]);
                }
                const int gx = i * NN + o_own;
                __stcs(reinterpret_cast<float2 *>(t.Xo + gx), make_float2(xo[0][0], xo[1][0]));
                __stcs(reinterpret_cast<float2 *>(t.Xo + n3 + gx), make_float2(xo[0][1], xo[1][1]));
                __stcs(reinterpret_cast<float2 *>(t.Do + gx), make_float2(dout[0][0], dout[1][0]));
                __stcs(reinterpret_cast<float2 *>(t.Do + n3 + gx), make_float2(dout[0][1], dout[1][1]));
            } else {
                float s0[2][kSrc] = {}, s1[2][kSrc] = {};
#pragma unroll
                for (int v = 0; v < 2; v++) {
                    site_a32<MODE, MODEL>(c, s, nb[0][v], nb[1][v], nb[2][v], nb[3][v], mom, s0[v], s1[v]);
                }
                if (++ngroup == kGroup || i == i1 - 1) {
                    fold<MODE>(s.mt, s.q3f, 2 * ngroup, mom, acc);
                    ngroup = 0;
                }
                if constexpr (MODE == MODE_A_GW) {
                    float *g = t.S + ((i - sfirst) * (N * (N + 2)) + so_row);
#pragma unroll
                    for (int q = 0; q < kSrc; q++, g += sstride)
                        __stcs(reinterpret_cast<float2 *>(g), make_float2(s0[0][q], s0[1][q]));
#pragma unroll
                    for (int q = 0; q < kSrc; q++, g += sstride)
                        __stcs(reinterpret_cast<float2 *>(g), make_float2(s1[0][q], s1[1][q]));
                }
            }
#pragma unroll
            for (int a = 0; a < 4; a++) {
                pr[a] = cu[a];
                cu[a] = nx[a];
            }
        }
        s_pr = s_cu;
        s_cu = s_nx;
        s_nx = next_slot(s_nx);
        s_is = next_slot(s_is);
    }
    cp_wait<0>();
    __syncthreads();  // the ring may be refilled by the block's next tile
}

template <int TK2, int TJ, int MODE, int S, int MODEL = -1, bool W16 = false>
__global__ void __launch_bounds__(TK2 *TJ, (sweep32_threads_per_sm<MODE>() + TK2 * TJ - 1) / (TK2 * TJ))
    sweep32_kernel(StencilArgs args) {
    extern __shared__ __align__(16) float ring[];  // S slots
    __shared__ double sred[((TK2 * TJ + 31) / 32) * kNV];
    __shared__ int sflag;

    const LatticeConsts &c = args.c;
    const int N = c.N;
    const int tid = threadIdx.x;
    Tile32 t;
    t.X = static_cast<const float *>(args.X);
    t.D = static_cast<const float *>(args.D);
    t.Xo = static_cast<float *>(args.Xo);
    t.Do = static_cast<float *>(args.Do);
    t.S = static_cast<float *>(args.S);
    t.k0 = blockIdx.x * 2 * TK2;
    t.j0 = blockIdx.y * TJ;
    t.planes = args.planes;
    const int first = args.planes ? 1 : 0, end = args.planes ? args.planes - 1 : N;  // own planes
    t.i0 = first + blockIdx.z * args.ci;
    t.i1 = min(t.i0 + args.ci, end);

    const Site32 s = site32_consts<MODE>(c, args.sc);
    double acc[kNV];
#pragma unroll
    for (int q = 0; q < kNV; q++) acc[q] = 0.;
    march32<TK2, TJ, MODE, S, TK2 * TJ, MODEL, W16>(c, s, t, ring, acc);

    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if constexpr (MODE != MODE_B) {
        block_reduce<kNV>(acc, sred);
        if (tid == 0)
            for (int q = 0; q < kNV; q++) args.partials[(size_t)bid * kNV + q] = acc[q];
    }
    if (!last_block_done(args.counter, &sflag)) return;
    if constexpr (MODE != MODE_B) {
        double tot[kNV];
        sum_partials<kNV>(args.partials, gridDim.x * gridDim.y * gridDim.z, tot, sred);
        if (tid == 0) {
            if (args.sums_out)
                for (int q = 0; q < kNV; q++) args.sums_out[q] = tot[q];
            else
                finish_a<float, MODE>(c, args.sc, tot, args.slot);
            *args.counter = 0u;
        }
    } else if (tid == 0) {
        finish_b<float>(c, args.sc);
        *args.counter = 0u;
    }
}

}  // namespace s32
}  // namespace gabe
