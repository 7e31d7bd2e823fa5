// Fused RK2 stencil sweeps for the GABE step (expansion_type 1,
// g2functions.cpp:234-271).
//
// The reference makes, per step, two field-update sweeps plus two
// calcEnergy() calls of three sweeps each, and (with GWs) two source sweeps.
// Its Friedmann update needs the full-volume energy of the stage-1 state
// before stage 2 can start (g2functions.cpp:250-252), and the end-of-step
// energy before the next step (:268-270).  Two sweeps per step is therefore
// the minimum, and these two kernels are those sweeps:
//
//   stage1: reads f0, fdot0 (7-point stencils); derives f1 = f0 + dt/2 fdot0
//           and fdot1 (never stored); reduces the stage-1 energies
//           (calcEnergy(1)); writes the GW sources of f0 and f1
//           (g2evolutionpert.cpp:48-132, 165-180) when calc_gws.  Its last
//           block forms a[1], adot[1] (adf).
//   stage2: reads f0, fdot0 again; recomputes fdot1 on a one-point halo in
//           shared memory (f0 staged with a two-point halo), writes
//           f0' = f0 + dt fdot1 and fdot0' = fdot0 + dt fddot(f1), and reduces
//           the end-of-step energies from f0', whose Laplacian needs fdot1
//           on the halo.  Its last block forms a[0], adot[0].
//
// Blocks march along i (slowest axis) over a chunk of `ci` planes, holding a
// ring of planes per array in shared memory; (j,k) tiles are blockDim.y x
// blockDim.x with k on the warp lanes for coalesced rows.  Periodic wrap is
// applied when staging planes.  The FP64 instantiation keeps the reference's
// operation order (compiled without FMA contraction); the FP32 one evolves
// fluctuations about the FP64 homogeneous trajectory (see common.cuh).
#pragma once

#include "common.cuh"

namespace gabe {

struct StencilArgs {
    const void *X;       // fields in  [2][N^3]
    const void *D;       // momenta in [2][N^3]
    void *Xo;            // fields out   (stage2)
    void *Do;            // momenta out  (stage2)
    void *S;             // GW sources [12][N][N][N+2] (stage1, calc_gws)
    double *partials;    // [nblocks][3]
    unsigned int *counter;
    DevScalars *sc;
    LatticeConsts c;
    int ci;              // planes per block along i
    int gws;
};

// Stage one plane of `src` (one field, N^3) with halo H into dst
// ((TJ+2H) x (TK+2H), row stride TK+2H).
template <typename T>
__device__ __forceinline__ void stage_plane(T *dst, const T *__restrict__ src, int N, int i, int j0, int k0, int H) {
    const int TK = blockDim.x, TJ = blockDim.y;
    const int C = TK + 2 * H, R = TJ + 2 * H;
    const T *plane = src + (size_t)wrapi(i, N) * N * N;
    for (int r = threadIdx.y; r < R; r += TJ) {
        const T *row = plane + (size_t)wrapi(j0 - H + r, N) * N;
        for (int c = threadIdx.x; c < C; c += TK) dst[r * C + c] = __ldg(row + wrapi(k0 - H + c, N));
    }
}

__device__ __forceinline__ int ring(int p, int n) { int m = p % n; return m < 0 ? m + n : m; }

// 7-point neighbourhood, reference order: centre, i+1, i-1, j+1, j-1, k+1, k-1.
template <typename T>
struct Nb7 {
    T v[7];
};

template <typename T>
__device__ __forceinline__ Nb7<T> gather7(const T *pm, const T *pc, const T *pp, int o, int C) {
    Nb7<T> n;
    n.v[0] = pc[o]; n.v[1] = pp[o]; n.v[2] = pm[o];
    n.v[3] = pc[o + C]; n.v[4] = pc[o - C]; n.v[5] = pc[o + 1]; n.v[6] = pc[o - 1];
    return n;
}

// laplacian() of g2functions.cpp:35-43 in its operation order.
__device__ __forceinline__ double lap64(const Nb7<double> &f, double dx2) {
    return (f.v[1] + f.v[2] + f.v[3] + f.v[4] + f.v[5] + f.v[6] - 6. * f.v[0]) / dx2;
}
__device__ __forceinline__ float lap32(const Nb7<float> &f, float inv_dx2) {
    return (((f.v[1] + f.v[2]) + (f.v[3] + f.v[4])) + (f.v[5] + f.v[6]) - 6.f * f.v[0]) * inv_dx2;
}

// GW source components 11,12,13,22,23,33 of one field added into s
// (jtg_stresstensor, g2evolutionpert.cpp:48-132, operation order kept).
__device__ __forceinline__ void source_add64(const LatticeConsts &c, const Nb7<double> &f, double *s) {
    const double d1 = (f.v[1] - f.v[2]) / 2;
    const double d2 = (f.v[3] - f.v[4]) / 2;
    const double d3 = (f.v[5] - f.v[6]) / 2;
    const double c13 = c.c13, c23 = c.c23, dn = c.dn;
    s[0] += c23 * d1 * d1 - c13 * d2 * d2 - c13 * d3 * d3;
    s[1] += dn * d1 * d2;
    s[2] += (dn * d1 * d3);
    s[3] += -c13 * d1 * d1 + c23 * d2 * d2 - c13 * d3 * d3;
    s[4] += (dn * d2 * d3);
    s[5] += -c13 * d1 * d1 - c13 * d2 * d2 + c23 * d3 * d3;
}
__device__ __forceinline__ void source_add32(float dn, const Nb7<float> &f, float *s) {
    const float d1 = 0.5f * (f.v[1] - f.v[2]);
    const float d2 = 0.5f * (f.v[3] - f.v[4]);
    const float d3 = 0.5f * (f.v[5] - f.v[6]);
    const float t = (1.f / 3.f) * (d1 * d1 + d2 * d2 + d3 * d3);
    s[0] += dn * (d1 * d1 - t);
    s[1] += dn * d1 * d2;
    s[2] += dn * d1 * d3;
    s[3] += dn * (d2 * d2 - t);
    s[4] += dn * d2 * d3;
    s[5] += dn * (d3 * d3 - t);
}

template <typename T>
__device__ __forceinline__ void store_sources(T *S, int N, int i, int j, int k, const T *s0, const T *s1) {
    const size_t slot = (size_t)N * N * (N + 2);
    const size_t o = ((size_t)i * N + j) * (N + 2) + k;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        S[q * slot + o] = s0[q];
        S[(6 + q) * slot + o] = s1[q];
    }
}

// Homogeneous-trajectory values for the FP32 path at the three stages of a
// step (start, midpoint, end), computed identically by every thread.
struct MeanTraj {
    double fb0[2], dfb0[2], fb1[2], dfb1[2], fbn[2], dfbn[2];
};
__device__ __forceinline__ MeanTraj mean_traj(const LatticeConsts &c, const DevScalars *sc, bool need_end) {
    MeanTraj m;
    const double h = c.half_dt, dt = c.dt;
    const double a0 = sc->a[0], c3H0 = (3. * sc->adot[0]) / a0;
    for (int f = 0; f < 2; f++) { m.fb0[f] = sc->fbar[f]; m.dfb0[f] = sc->dfbar[f]; }
    for (int f = 0; f < 2; f++) {
        m.fb1[f] = m.fb0[f] + h * m.dfb0[f];
        m.dfb1[f] = m.dfb0[f] + h * (-dv_h(c.model, c.mc, f, m.fb0[0], m.fb0[1]) - c3H0 * m.dfb0[f]);
    }
    if (need_end) {
        const double a1 = sc->a[1], c3H1 = (3. * sc->adot[1]) / a1;
        for (int f = 0; f < 2; f++) {
            m.fbn[f] = m.fb0[f] + dt * m.dfb1[f];
            m.dfbn[f] = m.dfb0[f] + dt * (-dv_h(c.model, c.mc, f, m.fb1[0], m.fb1[1]) - c3H1 * m.dfb1[f]);
        }
    }
    return m;
}

__device__ __forceinline__ MeanF mean_f(const LatticeConsts &c, const double *fb) {
    MeanF m;
    m.pb = (float)fb[0];
    m.cb = (float)fb[1];
    m.q0 = (float)c.mc[0];
    m.q1 = (float)c.mc[1];
    m.q2 = (float)c.mc[2];
    m.q3 = (float)c.mc[3];
    return m;
}

// ---------------------------------------------------------------------------
// stage 1
// ---------------------------------------------------------------------------
template <typename T, bool GWS>
__global__ void __launch_bounds__(256) stage1_kernel(StencilArgs args) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sred[8 * 3];
    __shared__ int sflag;
    T *sm = reinterpret_cast<T *>(smem_raw);
    const LatticeConsts &c = args.c;
    const int N = c.N;
    const int TK = blockDim.x, TJ = blockDim.y, tx = threadIdx.x, ty = threadIdx.y;
    const int C1 = TK + 2, P1 = C1 * (TJ + 2);
    T *F0 = sm;           // [fld*3 + slot][P1]
    T *D0 = sm + 6 * P1;  // [fld*3 + slot][P1]
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int i0 = blockIdx.z * args.ci, i1 = min(i0 + args.ci, N);
    const size_t n3 = (size_t)N * N * N;
    const T *X = static_cast<const T *>(args.X), *D = static_cast<const T *>(args.D);
    const DevScalars *scp = args.sc;
    const double a0 = scp->a[0], ad0 = scp->adot[0];
    const double h = c.half_dt;
    const double c3H0 = (3. * ad0) / a0;

    MeanTraj mt;
    MeanF m0, m1;
    float ia02f = 0.f, c3H0f = 0.f, hf = 0.f, inv_dx2f = 0.f, dnf = 0.f;
    if constexpr (sizeof(T) == 4) {
        mt = mean_traj(c, scp, false);
        m0 = mean_f(c, mt.fb0);
        m1 = mean_f(c, mt.fb1);
        ia02f = (float)(1.0 / (a0 * a0));
        c3H0f = (float)c3H0;
        hf = (float)h;
        inv_dx2f = (float)(1.0 / c.inv_dx2_div);
        dnf = (float)c.dn;
    }

    double kin = 0., pot = 0., grad = 0.;
    for (int p = i0 - 1; p <= i0; p++)
        for (int f = 0; f < 2; f++) {
            stage_plane(F0 + (f * 3 + ring(p, 3)) * P1, X + f * n3, N, p, j0, k0, 1);
            stage_plane(D0 + (f * 3 + ring(p, 3)) * P1, D + f * n3, N, p, j0, k0, 1);
        }
    const int o = (ty + 1) * C1 + (tx + 1);
    for (int i = i0; i < i1; i++) {
        for (int f = 0; f < 2; f++) {
            stage_plane(F0 + (f * 3 + ring(i + 1, 3)) * P1, X + f * n3, N, i + 1, j0, k0, 1);
            stage_plane(D0 + (f * 3 + ring(i + 1, 3)) * P1, D + f * n3, N, i + 1, j0, k0, 1);
        }
        __syncthreads();
        const int sm_ = ring(i - 1, 3), sc_ = ring(i, 3), sp_ = ring(i + 1, 3);
        Nb7<T> f0[2], d0[2], f1[2];
        for (int f = 0; f < 2; f++) {
            f0[f] = gather7(F0 + (f * 3 + sm_) * P1, F0 + (f * 3 + sc_) * P1, F0 + (f * 3 + sp_) * P1, o, C1);
            d0[f] = gather7(D0 + (f * 3 + sm_) * P1, D0 + (f * 3 + sc_) * P1, D0 + (f * 3 + sp_) * P1, o, C1);
        }
        T s0[6] = {0, 0, 0, 0, 0, 0}, s1[6] = {0, 0, 0, 0, 0, 0};
        if constexpr (sizeof(T) == 8) {
            for (int f = 0; f < 2; f++) {
                const double lap0 = lap64(f0[f], c.inv_dx2_div);
                const double dd0 = lap0 / a0 / a0 - dv64(c, f, f0[0].v[0], f0[1].v[0]) - c3H0 * d0[f].v[0];
                const double d1c = d0[f].v[0] + h * dd0;
#pragma unroll
                for (int q = 0; q < 7; q++) f1[f].v[q] = f0[f].v[q] + h * d0[f].v[q];
                const double lap1 = lap64(f1[f], c.inv_dx2_div);
                kin += d1c * d1c;
                grad -= f1[f].v[0] * lap1;
                if constexpr (GWS) {
                    source_add64(c, f0[f], s0);
                    source_add64(c, f1[f], s1);
                }
            }
            pot += pot64(c, f1[0].v[0], f1[1].v[0]);
        } else {
            for (int f = 0; f < 2; f++) {
                const float lap0 = lap32(f0[f], inv_dx2f);
                const float dd0 = lap0 * ia02f - dv_diff32(m0, c.model, f, f0[0].v[0], f0[1].v[0]) - c3H0f * d0[f].v[0];
                const float d1c = d0[f].v[0] + hf * dd0;
#pragma unroll
                for (int q = 0; q < 7; q++) f1[f].v[q] = f0[f].v[q] + hf * d0[f].v[q];
                const float lap1 = lap32(f1[f], inv_dx2f);
                const double dtot = mt.dfb1[f] + (double)d1c;
                kin += dtot * dtot;
                grad -= (double)(f1[f].v[0] * lap1);
                if constexpr (GWS) {
                    source_add32(dnf, f0[f], s0);
                    source_add32(dnf, f1[f], s1);
                }
            }
            pot += (double)v_diff32(m1, c.model, f1[0].v[0], f1[1].v[0]);
        }
        if constexpr (GWS) store_sources(static_cast<T *>(args.S), N, i, j0 + ty, k0 + tx, s0, s1);
        __syncthreads();
    }

    double v[3] = {kin, pot, grad};
    block_reduce<3>(v, sred);
    const int tid = tx + TK * ty;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid == 0)
        for (int q = 0; q < 3; q++) args.partials[(size_t)bid * 3 + q] = v[q];
    if (!last_block_done(args.counter, &sflag)) return;
    double tot[3];
    sum_partials<3>(args.partials, gridDim.x * gridDim.y * gridDim.z, tot, sred);
    if (tid == 0) {
        DevScalars *s = args.sc;
        const double a1 = a0 + h * ad0; /* g2functions.cpp:250 */
        double ek = tot[0] / c.gridsize / 2.;
        double ep = tot[1] / c.gridsize;
        double eg = tot[2] / c.gridsize / 2. / a1 / a1;
        if constexpr (sizeof(T) == 4) {
            MeanTraj m = mean_traj(c, s, false);
            ep += pot_h(c.model, c.mc, m.fb1[0], m.fb1[1]);
        }
        const double rho = ek + ep + eg;
        s->a[1] = a1;
        s->edkin[1] = ek;
        s->edpot[1] = ep;
        s->edgrad[1] = eg;
        s->edrho[1] = rho;
        s->adot[1] = sqrt(c.eight_pi_3 * rho) * a1; /* adf(1), :252 */
        if (!isfinite(rho)) s->status |= ST_NONFINITE;
        *args.counter = 0u;
    }
}

// ---------------------------------------------------------------------------
// stage 2
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void fdot1_region(const LatticeConsts &c, T *F0, T *D0, T *D1, int p, int P1, int P2,
                                             int C1, int C2, double a0, double c3H0, const MeanF &m0, float ia02f,
                                             float c3H0f, float hf, float inv_dx2f) {
    // fdot1 = fdot0 + dt/2 * fddot(f0) on the (TJ+2) x (TK+2) region of plane p
    const int TK = blockDim.x, TJ = blockDim.y;
    const int R1 = TJ + 2;
    const int sm4 = ring(p - 1, 4), sc4 = ring(p, 4), sp4 = ring(p + 1, 4), s3 = ring(p, 3);
    for (int r = threadIdx.y; r < R1; r += TJ)
        for (int cc = threadIdx.x; cc < C1; cc += TK) {
            const int o2 = (r + 1) * C2 + (cc + 1), o1 = r * C1 + cc;
            Nb7<T> g[2];
            for (int f = 0; f < 2; f++)
                g[f] = gather7(F0 + (f * 4 + sm4) * P2, F0 + (f * 4 + sc4) * P2, F0 + (f * 4 + sp4) * P2, o2, C2);
            for (int f = 0; f < 2; f++) {
                const T d0 = D0[(f * 3 + s3) * P1 + o1];
                if constexpr (sizeof(T) == 8) {
                    const double lap0 = lap64(g[f], c.inv_dx2_div);
                    const double dd0 = lap0 / a0 / a0 - dv64(c, f, g[0].v[0], g[1].v[0]) - c3H0 * d0;
                    D1[(f * 3 + s3) * P1 + o1] = d0 + c.half_dt * dd0;
                } else {
                    const float lap0 = lap32(g[f], inv_dx2f);
                    const float dd0 = lap0 * ia02f - dv_diff32(m0, c.model, f, g[0].v[0], g[1].v[0]) - c3H0f * d0;
                    D1[(f * 3 + s3) * P1 + o1] = d0 + hf * dd0;
                }
            }
        }
}

template <typename T>
__global__ void __launch_bounds__(256) stage2_kernel(StencilArgs args) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sred[8 * 3];
    __shared__ int sflag;
    T *sm = reinterpret_cast<T *>(smem_raw);
    const LatticeConsts &c = args.c;
    const int N = c.N;
    const int TK = blockDim.x, TJ = blockDim.y, tx = threadIdx.x, ty = threadIdx.y;
    const int C1 = TK + 2, P1 = C1 * (TJ + 2);
    const int C2 = TK + 4, P2 = C2 * (TJ + 4);
    T *F0 = sm;               // [fld*4 + slot][P2]   halo 2
    T *D0 = F0 + 8 * P2;      // [fld*3 + slot][P1]   halo 1
    T *D1 = D0 + 6 * P1;      // [fld*3 + slot][P1]   halo 1 (computed)
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int i0 = blockIdx.z * args.ci, i1 = min(i0 + args.ci, N);
    const size_t n3 = (size_t)N * N * N;
    const T *X = static_cast<const T *>(args.X), *D = static_cast<const T *>(args.D);
    T *Xo = static_cast<T *>(args.Xo), *Do = static_cast<T *>(args.Do);
    const DevScalars *scp = args.sc;
    const double a0 = scp->a[0], ad0 = scp->adot[0], a1 = scp->a[1], ad1 = scp->adot[1];
    const double h = c.half_dt, dt = c.dt;
    const double c3H0 = (3. * ad0) / a0, c3H1 = (3. * ad1) / a1;

    MeanTraj mt;
    MeanF m0, m1, mn;
    float ia02f = 0.f, ia12f = 0.f, c3H0f = 0.f, c3H1f = 0.f, hf = 0.f, dtf = 0.f, inv_dx2f = 0.f;
    if constexpr (sizeof(T) == 4) {
        mt = mean_traj(c, scp, true);
        m0 = mean_f(c, mt.fb0);
        m1 = mean_f(c, mt.fb1);
        mn = mean_f(c, mt.fbn);
        ia02f = (float)(1.0 / (a0 * a0));
        ia12f = (float)(1.0 / (a1 * a1));
        c3H0f = (float)c3H0;
        c3H1f = (float)c3H1;
        hf = (float)h;
        dtf = (float)dt;
        inv_dx2f = (float)(1.0 / c.inv_dx2_div);
    }

    for (int p = i0 - 2; p <= i0 + 1; p++)
        for (int f = 0; f < 2; f++) stage_plane(F0 + (f * 4 + ring(p, 4)) * P2, X + f * n3, N, p, j0, k0, 2);
    for (int p = i0 - 1; p <= i0; p++)
        for (int f = 0; f < 2; f++) stage_plane(D0 + (f * 3 + ring(p, 3)) * P1, D + f * n3, N, p, j0, k0, 1);
    __syncthreads();
    fdot1_region<T>(c, F0, D0, D1, i0 - 1, P1, P2, C1, C2, a0, c3H0, m0, ia02f, c3H0f, hf, inv_dx2f);
    fdot1_region<T>(c, F0, D0, D1, i0, P1, P2, C1, C2, a0, c3H0, m0, ia02f, c3H0f, hf, inv_dx2f);

    double kin = 0., pot = 0., grad = 0.;
    const int o1 = (ty + 1) * C1 + (tx + 1), o2 = (ty + 2) * C2 + (tx + 2);
    const int j = j0 + ty, k = k0 + tx;
    for (int i = i0; i < i1; i++) {
        __syncthreads();
        for (int f = 0; f < 2; f++) {
            stage_plane(F0 + (f * 4 + ring(i + 2, 4)) * P2, X + f * n3, N, i + 2, j0, k0, 2);
            stage_plane(D0 + (f * 3 + ring(i + 1, 3)) * P1, D + f * n3, N, i + 1, j0, k0, 1);
        }
        __syncthreads();
        fdot1_region<T>(c, F0, D0, D1, i + 1, P1, P2, C1, C2, a0, c3H0, m0, ia02f, c3H0f, hf, inv_dx2f);
        __syncthreads();

        const int m4 = ring(i - 1, 4), c4 = ring(i, 4), p4 = ring(i + 1, 4);
        const int m3 = ring(i - 1, 3), c3 = ring(i, 3), p3 = ring(i + 1, 3);
        Nb7<T> f0[2], d0[2], d1[2], f1[2], fn[2];
        for (int f = 0; f < 2; f++) {
            f0[f] = gather7(F0 + (f * 4 + m4) * P2, F0 + (f * 4 + c4) * P2, F0 + (f * 4 + p4) * P2, o2, C2);
            d0[f] = gather7(D0 + (f * 3 + m3) * P1, D0 + (f * 3 + c3) * P1, D0 + (f * 3 + p3) * P1, o1, C1);
            d1[f] = gather7(D1 + (f * 3 + m3) * P1, D1 + (f * 3 + c3) * P1, D1 + (f * 3 + p3) * P1, o1, C1);
        }
        const size_t gx = ((size_t)i * N + j) * N + k;
        if constexpr (sizeof(T) == 8) {
            for (int f = 0; f < 2; f++)
#pragma unroll
                for (int q = 0; q < 7; q++) {
                    f1[f].v[q] = f0[f].v[q] + h * d0[f].v[q];
                    fn[f].v[q] = f0[f].v[q] + dt * d1[f].v[q]; /* g2functions.cpp:259 */
                }
            for (int f = 0; f < 2; f++) {
                const double lap1 = lap64(f1[f], c.inv_dx2_div);
                const double dd1 = lap1 / a1 / a1 - dv64(c, f, f1[0].v[0], f1[1].v[0]) - c3H1 * d1[f].v[0];
                const double dnew = d0[f].v[0] + dt * dd1; /* :260 */
                const double lapn = lap64(fn[f], c.inv_dx2_div);
                Xo[f * n3 + gx] = fn[f].v[0];
                Do[f * n3 + gx] = dnew;
                kin += dnew * dnew;
                grad -= fn[f].v[0] * lapn;
            }
            pot += pot64(c, fn[0].v[0], fn[1].v[0]);
        } else {
            for (int f = 0; f < 2; f++)
#pragma unroll
                for (int q = 0; q < 7; q++) {
                    f1[f].v[q] = f0[f].v[q] + hf * d0[f].v[q];
                    fn[f].v[q] = f0[f].v[q] + dtf * d1[f].v[q];
                }
            for (int f = 0; f < 2; f++) {
                const float lap1 = lap32(f1[f], inv_dx2f);
                const float dd1 = lap1 * ia12f - dv_diff32(m1, c.model, f, f1[0].v[0], f1[1].v[0]) - c3H1f * d1[f].v[0];
                const float dnew = d0[f].v[0] + dtf * dd1;
                const float lapn = lap32(fn[f], inv_dx2f);
                Xo[f * n3 + gx] = fn[f].v[0];
                Do[f * n3 + gx] = dnew;
                const double dtot = mt.dfbn[f] + (double)dnew;
                kin += dtot * dtot;
                grad -= (double)(fn[f].v[0] * lapn);
            }
            pot += (double)v_diff32(mn, c.model, fn[0].v[0], fn[1].v[0]);
        }
    }

    double v[3] = {kin, pot, grad};
    block_reduce<3>(v, sred);
    const int tid = tx + TK * ty;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid == 0)
        for (int q = 0; q < 3; q++) args.partials[(size_t)bid * 3 + q] = v[q];
    if (!last_block_done(args.counter, &sflag)) return;
    double tot[3];
    sum_partials<3>(args.partials, gridDim.x * gridDim.y * gridDim.z, tot, sred);
    if (tid == 0) {
        DevScalars *s = args.sc;
        const double an = a0 + dt * ad1; /* g2functions.cpp:268 */
        double ek = tot[0] / c.gridsize / 2.;
        double ep = tot[1] / c.gridsize;
        double eg = tot[2] / c.gridsize / 2. / an / an;
        if constexpr (sizeof(T) == 4) {
            MeanTraj m = mean_traj(c, s, true);
            ep += pot_h(c.model, c.mc, m.fbn[0], m.fbn[1]);
            for (int f = 0; f < 2; f++) { s->fbar[f] = m.fbn[f]; s->dfbar[f] = m.dfbn[f]; }
        }
        const double rho = ek + ep + eg;
        s->a[0] = an;
        s->edkin[0] = ek;
        s->edpot[0] = ep;
        s->edgrad[0] = eg;
        s->edrho[0] = rho;
        s->adot[0] = sqrt(c.eight_pi_3 * rho) * an; /* adf(0), :270 */
        s->step += 1;
        if (!isfinite(rho)) s->status |= ST_NONFINITE;
        *args.counter = 0u;
    }
}

}  // namespace gabe
