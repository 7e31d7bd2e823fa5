// Fused RK2 stencil sweeps for the GABE step (expansion_type 1,
// g2functions.cpp:234-271).
//
// The reference makes, per step, two field-update sweeps, two calcEnergy()
// calls of three sweeps each and (with GWs) two source sweeps.  Its
// Friedmann update needs the full-volume energy of the stage-1 state before
// stage 2 (g2functions.cpp:250-252) and of the end state before the next
// step (:268-270), so two sweeps per step is the minimum.  They are:
//
//   sweep A (mode A / A_GW): reads f0, fdot0 with 7-point neighbourhoods and
//     reduces, in one pass,
//       E0 = calcEnergy(0) of (f0, fdot0) -> adot0 = adf(0) (:268-270 of the
//            previous step; skipped right after an upload, where adot0 is the
//            caller's, g2init.cpp:29),
//       the stage-1 energies: pot1 and grad1 depend only on
//            f1 = f0 + dt/2 fdot0; fdot1 = P + adot0 Q is affine in adot0, so
//            kin1 = sum P^2 + 2 adot0 sum PQ + adot0^2 sum Q^2 is formed from
//            three sums without knowing adot0 during the sweep,
//     and writes the GW sources of f0 and f1 (g2evolutionpert.cpp:48-132,
//     165-180).  Its last block forms adot0, a[1], adot[1] (:250-252).
//   sweep B: reads f0, fdot0 again, forms fdot1 and f1 at the 7 points,
//     writes f0' = f0 + dt fdot1 and fdot0' = fdot0 + dt fddot(f1)
//     (:254-262).  Its last block advances a[0] (:268).
//   mode E0: sweep A's E0 part alone, for energies asked for between steps.
//
// Both sweeps are radius-1 stencils: in the FP64 kernels here each thread
// owns a (j,k) column of a TJ x TK tile and marches along i over `ci` planes,
// keeping the i-1, i, i+1 values of its column in registers (plus i+2
// prefetched), and the (j,k) neighbours of plane i in a double-buffered
// shared-memory tile with a one-point halo, so each value is read from HBM
// once per sweep and there is one barrier per plane.  They keep the
// reference's operation order (compiled without FMA contraction).  The FP32
// sweeps (sweep32.cuh) evolve fluctuations about the FP64 homogeneous
// trajectory with the per-site helpers and moment folding defined here.
#pragma once

#include "common.cuh"

namespace gabe {

enum SweepMode : int { MODE_A = 0, MODE_A_GW = 1, MODE_E0 = 2, MODE_B = 3 };

struct StencilArgs {
    const void *X;       // fields in  [2][N^3]
    const void *D;       // momenta in [2][N^3]
    void *Xo;            // fields out   (sweep B)
    void *Do;            // momenta out  (sweep B)
    void *S;             // GW sources [10][N][N][N+2] (sweep A with GWs)
    double *partials;    // [nblocks][8]
    unsigned int *counter;
    DevScalars *sc;
    LatticeConsts c;
    int ci;              // planes per block along i
    int slot;            // source buffer / GW scalar slot of this step
    // Slab of a lattice split along i (slab.cu): X, D, Xo, Do hold `planes`
    // planes per field -- own planes 1 .. planes-2 between two halo planes --
    // addressed without wrap along i.  0: the whole periodic lattice.
    int planes;
    // Slab: the last block writes the block-summed totals (kNV doubles) here
    // instead of finishing the stage; the caller adds the totals of all
    // slabs and finishes with slab_finish_kernel.
    double *sums_out;
};

constexpr int kNV = 8;  // reduced values: kin0 pot0 grad0 | pot1 grad1 PP PQ QQ

// 7-point neighbourhood, reference order: centre, i+1, i-1, j+1, j-1, k+1, k-1.
template <typename T>
struct Nb7 {
    T v[7];
};

// laplacian() of g2functions.cpp:35-43 in its operation order.
__device__ __forceinline__ double lap64(const Nb7<double> &f, double dx2) {
    return (f.v[1] + f.v[2] + f.v[3] + f.v[4] + f.v[5] + f.v[6] - 6. * f.v[0]) / dx2;
}
__device__ __forceinline__ float lap32(const Nb7<float> &f, float inv_dx2) {
    return fmaf(-6.f, f.v[0], ((f.v[1] + f.v[2]) + (f.v[3] + f.v[4])) + (f.v[5] + f.v[6])) * inv_dx2;
}

// GW source components 11,12,13,22,23 of one field added into s
// (jtg_stresstensor, g2evolutionpert.cpp:48-132, operation order kept).  The
// source is traceless, so component 33 (= -11 - 22) is never stored: the
// k-space update needs only the five (kspace.cuh).
constexpr int kSrc = 5;
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
}
// FP32 form: the products of the undivided central differences e_i =
// f(x + e_i) - f(x - e_i) are summed over both fields first (grad_prod_add),
// then scaled once (source_from_prod): dn/4 (e_i e_j - delta_ij |e|^2 / 3),
// the same tensor as source_add64 in fewer instructions.
__device__ __forceinline__ void grad_prod_add(const Nb7<float> &f, float (&P)[6]) {
    const float e1 = f.v[1] - f.v[2], e2 = f.v[3] - f.v[4], e3 = f.v[5] - f.v[6];
    P[0] = fmaf(e1, e1, P[0]);
    P[1] = fmaf(e2, e2, P[1]);
    P[2] = fmaf(e3, e3, P[2]);
    P[3] = fmaf(e1, e2, P[3]);
    P[4] = fmaf(e1, e3, P[4]);
    P[5] = fmaf(e2, e3, P[5]);
}
__device__ __forceinline__ void source_from_prod(float q /* dn / 4 */, const float (&P)[6], float *s) {
    const float t = (1.f / 3.f) * ((P[0] + P[1]) + P[2]);
    s[0] = q * (P[0] - t);
    s[1] = q * P[3];
    s[2] = q * P[4];
    s[3] = q * (P[1] - t);
    s[4] = q * P[5];
}

// Homogeneous-trajectory values of the FP32 path (start and midpoint of a
// step; the midpoint momentum is affine in adot0: dfb1 = p + adot0 q).
struct MeanTraj {
    double fb0[2], dfb0[2], fb1[2], pbar[2], qbar[2];
};
__device__ __forceinline__ MeanTraj mean_traj(const LatticeConsts &c, const DevScalars *sc) {
    MeanTraj m;
    const double h = c.half_dt, a0 = sc->a[0];
    for (int f = 0; f < 2; f++) { m.fb0[f] = sc->fbar[f]; m.dfb0[f] = sc->dfbar[f]; }
    for (int f = 0; f < 2; f++) {
        m.fb1[f] = m.fb0[f] + h * m.dfb0[f];
        m.pbar[f] = m.dfb0[f] - h * dv_h(c.model, c.mc, f, m.fb0[0], m.fb0[1]);
        m.qbar[f] = -h * 3. * m.dfb0[f] / a0;
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
    m.pb2 = (float)(2. * fb[0]);
    m.cb2 = (float)(2. * fb[1]);
    m.pbsq = (float)(fb[0] * fb[0]);
    m.pb3sq = (float)(3. * fb[0] * fb[0]);
    return m;
}

// FP32 energy sums (the FP32 sweeps here and in sweep32.cuh).
// Reduced values of sweep A / E0 are sums over sites of expressions such as
// (dfbar + d)^2 whose large homogeneous parts are known per launch.  Each
// thread accumulates only FP32 moments of the fluctuations (sum d, sum d^2,
// sum Pd, ...) over a group of kGroup planes and folds them into its FP64
// sums once per group with the exact expansions, e.g.
//   sum (dfbar + d)^2 = n dfbar^2 + 2 dfbar sum d + sum d^2,
// so no site needs an FP32 -> FP64 conversion (that conversion pipe, not
// HBM, bounded the per-site FP64 form).
constexpr int kGroup = 8;
struct Moments {
    float a[2];  // sum d (momentum fluctuation) per field
    float b;     // sum over fields of d^2
    float c[2];  // sum Pd per field (stage-1 momentum before the adot0 term)
    float e;     // sum over fields of Pd^2
    float f;     // sum over fields of Pd d
    float g0, g1;  // sum over fields of f lap f, stage 0 and stage 1
    float v0, v1;  // potential differences, stage 0 and stage 1
};
__device__ __forceinline__ void zero(Moments &m) {
    m.a[0] = m.a[1] = m.b = m.c[0] = m.c[1] = m.e = m.f = m.g0 = m.g1 = m.v0 = m.v1 = 0.f;
}

// Folds the moments of n sites into the FP64 sums kin0 pot0 grad0 | pot1
// grad1 PP PQ QQ (the kNV values finish_a expects) and clears them.  With
// P = pbar + Pd, Q = qbar + q3 d:  sum P^2 = n pbar^2 + 2 pbar sum Pd + sum Pd^2,
// sum PQ = n pbar qbar + pbar q3 sum d + qbar sum Pd + q3 sum Pd d,
// sum Q^2 = n qbar^2 + 2 qbar q3 sum d + q3^2 sum d^2.
template <int MODE>
__device__ __forceinline__ void fold(const MeanTraj &t, float q3f, int n, Moments &m, double (&acc)[kNV]) {
    const double dn = (double)n, q3 = (double)q3f;
    const double a0 = m.a[0], a1 = m.a[1], b = m.b;
    acc[0] += dn * (t.dfb0[0] * t.dfb0[0] + t.dfb0[1] * t.dfb0[1]) + 2. * (t.dfb0[0] * a0 + t.dfb0[1] * a1) + b;
    acc[1] += (double)m.v0;
    acc[2] -= (double)m.g0;
    if constexpr (MODE != MODE_E0) {
        const double c0 = m.c[0], c1 = m.c[1];
        acc[3] += (double)m.v1;
        acc[4] -= (double)m.g1;
        acc[5] += dn * (t.pbar[0] * t.pbar[0] + t.pbar[1] * t.pbar[1]) + 2. * (t.pbar[0] * c0 + t.pbar[1] * c1) +
                  (double)m.e;
        acc[6] += dn * (t.pbar[0] * t.qbar[0] + t.pbar[1] * t.qbar[1]) + q3 * (t.pbar[0] * a0 + t.pbar[1] * a1) +
                  (t.qbar[0] * c0 + t.qbar[1] * c1) + q3 * (double)m.f;
        acc[7] += dn * (t.qbar[0] * t.qbar[0] + t.qbar[1] * t.qbar[1]) + 2. * q3 * (t.qbar[0] * a0 + t.qbar[1] * a1) +
                  q3 * q3 * b;
    }
    zero(m);
}

// ---------------------------------------------------------------------------
// plane march: 4 arrays (f0 phi, f0 chi, fdot0 phi, fdot0 chi)
// ---------------------------------------------------------------------------
template <typename T, int TK, int TJ>
struct March {
    static constexpr int C = TK + 2, R = TJ + 2, P = C * R, NA = 4;
    static constexpr int NH = 2 * TK + 2 * TJ;  // halo points of a plane tile
    const T *src[NA];
    int N, j0, k0, tx, ty, tid;
    bool wrap;  // periodic along i (whole lattice) or slab planes addressed as they are
    // halo duty of this thread: (row, col) in the tile and global (j, k)
    int hr, hc, hj, hk;
    bool has_halo;
    T prev[NA], cur[NA], nxt[NA], nn[NA], hal[NA];

    __device__ __forceinline__ void init(const T *X, const T *D, int N_, size_t n3, int j0_, int k0_, bool wrap_) {
        src[0] = X; src[1] = X + n3; src[2] = D; src[3] = D + n3;
        N = N_;
        wrap = wrap_;
        tid = threadIdx.x;
        tx = tid % TK; ty = tid / TK;
        j0 = j0_; k0 = k0_;
        has_halo = tid < NH;
        int t = tid;
        if (t < TK) { hr = 0; hc = t + 1; }
        else if (t < 2 * TK) { hr = TJ + 1; hc = t - TK + 1; }
        else if (t < 2 * TK + TJ) { hr = t - 2 * TK + 1; hc = 0; }
        else { hr = t - 2 * TK - TJ + 1; hc = TK + 1; }
        hj = wrapi(j0 + hr - 1, N);
        hk = wrapi(k0 + hc - 1, N);
    }
    __device__ __forceinline__ int plane(int i) const { return wrap ? wrapi(i, N) : i; }
    __device__ __forceinline__ size_t own(int i) const {
        return ((size_t)plane(i) * N + (j0 + ty)) * N + (k0 + tx);
    }
    __device__ __forceinline__ size_t halo(int i) const { return ((size_t)plane(i) * N + hj) * N + hk; }
    __device__ __forceinline__ void load_own(T (&dst)[NA], int i) const {
        const size_t o = own(i);
#pragma unroll
        for (int a = 0; a < NA; a++) dst[a] = __ldg(src[a] + o);
    }
    __device__ __forceinline__ void load_halo(int i) {
        if (has_halo) {
            const size_t o = halo(i);
#pragma unroll
            for (int a = 0; a < NA; a++) hal[a] = __ldg(src[a] + o);
        }
    }
    // writes plane values (own = v, halo = hal) into shared buffer sb
    __device__ __forceinline__ void store(T *sb, const T (&v)[NA]) const {
#pragma unroll
        for (int a = 0; a < NA; a++) sb[a * P + (ty + 1) * C + (tx + 1)] = v[a];
        if (has_halo)
#pragma unroll
            for (int a = 0; a < NA; a++) sb[a * P + hr * C + hc] = hal[a];
    }
    // 7-point neighbourhood of array a at plane i (sb holds plane i)
    __device__ __forceinline__ Nb7<T> nb(const T *sb, int a) const {
        const T *p = sb + a * P + (ty + 1) * C + (tx + 1);
        Nb7<T> n;
        n.v[0] = cur[a]; n.v[1] = nxt[a]; n.v[2] = prev[a];
        n.v[3] = p[C]; n.v[4] = p[-C]; n.v[5] = p[1]; n.v[6] = p[-1];
        return n;
    }
};

template <typename T>
__device__ __forceinline__ Nb7<T> axpy7(const Nb7<T> &x, T h, const Nb7<T> &y) {
    Nb7<T> r;
#pragma unroll
    for (int q = 0; q < 7; q++) r.v[q] = x.v[q] + h * y.v[q];
    return r;
}

// sources [10][splanes][N][N+2]: the whole lattice (splanes = N, sfirst = 0)
// or a slab's own planes (plane i at i - sfirst)
template <typename T>
__device__ __forceinline__ void store_sources(T *S, int N, int splanes, int sfirst, int i, int j, int k, const T *s0,
                                              const T *s1) {
    const size_t slot = (size_t)splanes * N * (N + 2);
    const size_t o = ((size_t)(i - sfirst) * N + j) * (N + 2) + k;
#pragma unroll
    for (int q = 0; q < kSrc; q++) {
        S[q * slot + o] = s0[q];
        S[(kSrc + q) * slot + o] = s1[q];
    }
}

// Final scalars of sweep A / E0 from the block-summed values (thread 0 of
// the last block).
template <typename T, int MODE>
__device__ __forceinline__ void finish_a(const LatticeConsts &c, DevScalars *s, const double *tot, int slot) {
    const double a0 = s->a[0];
    double ek0 = tot[0] / c.gridsize / 2.;
    double ep0 = tot[1] / c.gridsize;
    const double eg0 = tot[2] / c.gridsize / 2. / a0 / a0;
    MeanTraj m{};
    if constexpr (sizeof(T) == 4) {
        m = mean_traj(c, s);
        ep0 += pot_h(c.model, c.mc, m.fb0[0], m.fb0[1]);
    }
    const double rho0 = ek0 + ep0 + eg0;
    s->edkin[0] = ek0;
    s->edpot[0] = ep0;
    s->edgrad[0] = eg0;
    s->edrho[0] = rho0;
    // adf(0), g2functions.cpp:270; without expansion (type 0, :207-232) a and
    // adot keep their initial values and only calcEnergy(0) is taken (:231)
    if (!s->adot_given && c.expansion != 0) s->adot[0] = sqrt(c.eight_pi_3 * rho0) * a0;
    if (!isfinite(rho0)) s->status |= ST_NONFINITE;
    if constexpr (MODE == MODE_E0) return;
    if (c.expansion == 0) return;
    const double ad0 = s->adot[0];
    const double a1 = a0 + c.half_dt * ad0; /* :250 */
    const double ek1 = (tot[5] + 2. * ad0 * tot[6] + ad0 * ad0 * tot[7]) / c.gridsize / 2.;
    double ep1 = tot[3] / c.gridsize;
    const double eg1 = tot[4] / c.gridsize / 2. / a1 / a1;
    if constexpr (sizeof(T) == 4) ep1 += pot_h(c.model, c.mc, m.fb1[0], m.fb1[1]);
    const double rho1 = ek1 + ep1 + eg1;
    s->a[1] = a1;
    s->edkin[1] = ek1;
    s->edpot[1] = ep1;
    s->edgrad[1] = eg1;
    s->edrho[1] = rho1;
    s->adot[1] = sqrt(c.eight_pi_3 * rho1) * a1; /* adf(1), :252 */
    if (!isfinite(rho1)) s->status |= ST_NONFINITE;
    s->gw[slot][0] = a0;
    s->gw[slot][1] = ad0;
    s->gw[slot][2] = a1;
    s->gw[slot][3] = s->adot[1];
}

// ---------------------------------------------------------------------------
// the sweep kernel
// ---------------------------------------------------------------------------
// One tile of one lattice: the column tile (j0, k0) marched over planes
// [i0, i1) by the FP64 single-lattice kernel below (the FP32 sweeps use the
// cp.async plane march of sweep32.cuh).
template <typename T>
struct TileJob {
    const T *X, *D;   // fields and momenta in, [2][N^3] each
    T *Xo, *Do;       // sweep B outputs
    T *S;             // GW sources [10][N][N][N+2] (sweep A with GWs)
    const DevScalars *sc;
    int j0, k0, i0, i1;
    int planes;       // planes per field in the arrays (slab); 0 = N, periodic
};

template <int TK, int TJ>
struct SweepSmem {
    static constexpr int P = (TK + 2) * (TJ + 2);
};

// Marches one tile; adds this thread's share of the reduced values to acc.
template <typename T, int TK, int TJ, int MODE>
__device__ __forceinline__ void sweep_tile(const LatticeConsts &c, const TileJob<T> &job, T *smem0, T *smem1,
                                           double (&acc)[kNV]) {
    static_assert(sizeof(T) == 8, "FP64 march; FP32 storage uses sweep32.cuh");
    using M = March<T, TK, TJ>;
    const int N = c.N;
    const size_t n3 = (size_t)(job.planes ? job.planes : N) * N * N;
    M m;
    m.init(job.X, job.D, N, n3, job.j0, job.k0, job.planes == 0);
    const int i0 = job.i0, i1 = job.i1;
    const DevScalars *scp = job.sc;
    const double h = c.half_dt, dt = c.dt;
    const double a0 = scp->a[0];
    auto buf = [smem0, smem1](int i) { return (i & 1) ? smem1 : smem0; };

    double ad0 = 0., a1 = 0., ad1 = 0.;
    if constexpr (MODE == MODE_B) {
        ad0 = scp->adot[0];
        a1 = scp->a[1];
        ad1 = scp->adot[1];
    }
    const double c3H0 = (3. * ad0) / a0, c3H1 = MODE == MODE_B ? (3. * ad1) / a1 : 0.;
    (void)c3H1;

    // prologue: registers for planes i0-1, i0, i0+1; shared tile of plane i0
    m.load_own(m.prev, i0 - 1);
    m.load_own(m.cur, i0);
    m.load_own(m.nxt, i0 + 1);
    m.load_halo(i0);
    m.store(buf(i0), m.cur);
    __syncthreads();

    T *Xo = job.Xo, *Do = job.Do;
    const int j = m.j0 + m.ty, k = m.k0 + m.tx;
    for (int i = i0; i < i1; i++) {
        const bool more = i + 1 < i1;
        if (more) {
            m.load_own(m.nn, i + 2);
            m.load_halo(i + 1);
        }
        const T *sb = buf(i);
        Nb7<T> f0[2], d0[2];
        for (int f = 0; f < 2; f++) {
            f0[f] = m.nb(sb, f);
            d0[f] = m.nb(sb, 2 + f);
        }
        if constexpr (MODE == MODE_B) {
            const size_t gx = ((size_t)i * N + j) * N + k;
            const Nb7<double> f1[2] = {axpy7(f0[0], h, d0[0]), axpy7(f0[1], h, d0[1])};
            for (int f = 0; f < 2; f++) {
                const double lap0 = lap64(f0[f], c.inv_dx2_div);
                const double dd0 = lap0 / a0 / a0 - dv64(c, f, f0[0].v[0], f0[1].v[0]) - c3H0 * d0[f].v[0];
                const double d1c = d0[f].v[0] + h * dd0;                  /* g2functions.cpp:242 */
                const double lap1 = lap64(f1[f], c.inv_dx2_div);
                const double dd1 = lap1 / a1 / a1 - dv64(c, f, f1[0].v[0], f1[1].v[0]) - c3H1 * d1c;
                Xo[f * n3 + gx] = f0[f].v[0] + dt * d1c;                  /* :259 */
                Do[f * n3 + gx] = d0[f].v[0] + dt * dd1;                  /* :260 */
            }
        } else {
            T s0[kSrc] = {0, 0, 0, 0, 0}, s1[kSrc] = {0, 0, 0, 0, 0};
            for (int f = 0; f < 2; f++) {
                const double lap0 = lap64(f0[f], c.inv_dx2_div);
                acc[0] += d0[f].v[0] * d0[f].v[0];
                acc[2] -= f0[f].v[0] * lap0;
                if constexpr (MODE != MODE_E0) {
                    const Nb7<double> f1 = axpy7(f0[f], h, d0[f]);
                    const double P = d0[f].v[0] + h * (lap0 / a0 / a0 - dv64(c, f, f0[0].v[0], f0[1].v[0]));
                    const double Q = -h * 3. * d0[f].v[0] / a0;
                    acc[5] += P * P;
                    acc[6] += P * Q;
                    acc[7] += Q * Q;
                    acc[4] -= f1.v[0] * lap64(f1, c.inv_dx2_div);
                    if constexpr (MODE == MODE_A_GW) {
                        source_add64(c, f0[f], s0);
                        source_add64(c, f1, s1);
                    }
                }
            }
            acc[1] += pot64(c, f0[0].v[0], f0[1].v[0]);
            if constexpr (MODE != MODE_E0)
                acc[3] += pot64(c, f0[0].v[0] + h * d0[0].v[0], f0[1].v[0] + h * d0[1].v[0]);
            if constexpr (MODE == MODE_A_GW)
                store_sources(job.S, N, job.planes ? job.planes - 2 : N, job.planes ? 1 : 0, i, j, k, s0, s1);
        }
        if (more) {
#pragma unroll
            for (int a = 0; a < M::NA; a++) {
                m.prev[a] = m.cur[a];
                m.cur[a] = m.nxt[a];
                m.nxt[a] = m.nn[a];
            }
            m.store(buf(i + 1), m.cur);
        }
        __syncthreads();
    }
}

// End of sweep B for one lattice (thread 0 of the block that finished it
// last): the homogeneous trajectory (FP32 path) and a[0] advance.
template <typename T>
__device__ __forceinline__ void finish_b(const LatticeConsts &c, DevScalars *s) {
    const double dt = c.dt, a0 = s->a[0], ad0 = s->adot[0], a1 = s->a[1], ad1 = s->adot[1];
    const double c3H1 = (3. * ad1) / a1;
    if constexpr (sizeof(T) == 4) {
        MeanTraj q = mean_traj(c, s);
        for (int f = 0; f < 2; f++) {
            const double dfb1 = q.pbar[f] + ad0 * q.qbar[f];
            const double fbn = q.fb0[f] + dt * dfb1;
            const double dfbn = q.dfb0[f] + dt * (-dv_h(c.model, c.mc, f, q.fb1[0], q.fb1[1]) - c3H1 * dfb1);
            s->fbar[f] = fbn;
            s->dfbar[f] = dfbn;
        }
    }
    if (c.expansion != 0) s->a[0] = a0 + dt * ad1; /* g2functions.cpp:268 (type 2: :299) */
    s->adot_given = 0;
    s->step += 1;
}

// Single lattice, FP64: block (x, y, z) = column tile (k, j) and plane chunk.
template <typename T, int TK, int TJ, int MODE>
__global__ void __launch_bounds__(TK *TJ) sweep_kernel(StencilArgs args) {
    __shared__ __align__(16) T smem[2][4 * SweepSmem<TK, TJ>::P];
    __shared__ double sred[((TK * TJ + 31) / 32) * kNV];
    __shared__ int sflag;
    const LatticeConsts &c = args.c;
    TileJob<T> job;
    job.X = static_cast<const T *>(args.X);
    job.D = static_cast<const T *>(args.D);
    job.Xo = static_cast<T *>(args.Xo);
    job.Do = static_cast<T *>(args.Do);
    job.S = static_cast<T *>(args.S);
    job.sc = args.sc;
    job.k0 = blockIdx.x * TK;
    job.j0 = blockIdx.y * TJ;
    job.planes = args.planes;
    const int first = args.planes ? 1 : 0, end = args.planes ? args.planes - 1 : c.N;  // own planes
    job.i0 = first + blockIdx.z * args.ci;
    job.i1 = min(job.i0 + args.ci, end);
    double acc[kNV];
#pragma unroll
    for (int q = 0; q < kNV; q++) acc[q] = 0.;
    sweep_tile<T, TK, TJ, MODE>(c, job, smem[0], smem[1], acc);

    const int tid = threadIdx.x;
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
                finish_a<T, MODE>(c, args.sc, tot, args.slot);
            *args.counter = 0u;
        }
    } else if (tid == 0) {
        finish_b<T>(c, args.sc);
        *args.counter = 0u;
    }
}

// Slab: the end of sweep A / E0 from the totals of all slabs (one thread).
template <typename T, int MODE>
__global__ void slab_finish_kernel(LatticeConsts c, DevScalars *sc, const double *tot, int slot) {
    if (blockIdx.x == 0 && threadIdx.x == 0) finish_a<T, MODE>(c, sc, tot, slot);
}

}  // namespace gabe
