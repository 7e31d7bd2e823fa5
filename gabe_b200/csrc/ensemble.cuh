// Batched ensemble: many independent lattices of uneven size, coupling,
// amplitude and seed evolved together (FP32 storage, FP64 scalars).
//
// Each step is the single-lattice step (stencil.cuh, kspace.cuh) issued once
// for the whole ensemble:
//   * sweep A and sweep B take one work item (lattice, column tile, plane
//     chunk) per 256-thread block; each item runs the FP32 plane march of
//     the single-lattice sweeps (sweep32.cuh: cp.async plane ring, two sites
//     per thread) with the tile shape chosen for that lattice size (64x8,
//     32x16 or 16x16 sites); per-item partial sums are combined by the block
//     that finishes the last item of a lattice, in item order, so every
//     lattice gets its own Friedmann update without a grid-wide barrier;
//   * the GW transforms are one cuFFT call per lattice size (batch = 10 x
//     lattices of that size, sources of a size group contiguous);
//   * the k-space update is one kernel over the half spectra of all
//     lattices, in chunks of one lattice per block.
// The initial state is drawn on the device with the reference's randInit
// distribution (g2init.cpp:68-189) from a counter-based generator (Philox
// 4x32-10, Salmon et al., SC'11), so it matches the reference in
// distribution, not bit for bit.
#pragma once

#include <math_constants.h>

#include "kspace.cuh"
#include "sweep32.cuh"

namespace gabe {

struct EnsLat {
    LatticeConsts c;
    float *X[2], *D[2];  // [2 fields][N^3] each, ping-pong
    float *S;            // [10][N][N][N+2] sources / [..][N][N][N/2+1] spectra
    Cplx<float> *G;      // [4][M] h+, hx, l+, lx
    DevScalars *sc;
    int first_kchunk;    // first block of the k-space update that takes this lattice
    int first_item, nitems;
    int N;
    unsigned long long seed;  // IC: counter-based generator key
    double amp;               // IC: amplitude multiplier
    double rescale_B;         // B of the program units
};

struct EnsItem {
    int lat, shape, j0, k0, i0, i1;
};

struct EnsArgs {
    const EnsLat *lat;
    const EnsItem *items;
    int nitems, nlat;
    int cur, slot;
    double *partials;         // [nitems][kNV]
    unsigned int *lat_count;  // [nlat]
};

// ---------------------------------------------------------------------------
// sweeps over the work list: one item (lattice, column tile, plane chunk) per
// block, the FP32 plane march of the single-lattice sweeps (sweep32.cuh)
// ---------------------------------------------------------------------------
constexpr int kEnsThreads = 256;
// Plane slots of the cp.async ring per sweep (the wide slots of sweep32.cuh,
// as the single-lattice sweeps: six for sweep A, five for sweep B, four for
// the energies-only sweep).
template <int MODE>
__host__ __device__ constexpr int ens_ring() {
    return MODE == MODE_E0 ? 4 : (MODE == MODE_B ? 5 : 6);
}

// Tile shapes of the work items, sites along k x j: 0 = 64 x 8, 1 = 32 x 16,
// 2 = 16 x 16 (128 of the 256 threads march; for N = 16 (mod 32)).
__host__ __device__ constexpr int ens_tile_k(int shape) { return shape == 0 ? 64 : (shape == 1 ? 32 : 16); }
__host__ __device__ constexpr int ens_tile_j(int shape) { return shape == 0 ? 8 : 16; }
template <int MODE>
constexpr size_t ens_ring_bytes() {
    constexpr int a = s32::Ring<32, 8, true>::SLOT, b = s32::Ring<16, 16, true>::SLOT, c = s32::Ring<8, 16, true>::SLOT;
    return sizeof(float) * ens_ring<MODE>() * (a > b ? (a > c ? a : c) : (b > c ? b : c));
}

template <int MODE>
__global__ void __launch_bounds__(kEnsThreads, s32::sweep32_threads_per_sm<MODE>() / kEnsThreads)
    ens_sweep_kernel(EnsArgs a) {
    extern __shared__ __align__(16) float ring[];
    __shared__ double sred[(kEnsThreads / 32) * kNV];
    __shared__ int sflag;
    const int tid = threadIdx.x, it = blockIdx.x;
    const EnsItem item = a.items[it];
    const EnsLat &L = a.lat[item.lat];
    const LatticeConsts c = L.c;
    s32::Tile32 t;
    t.X = L.X[a.cur];
    t.D = L.D[a.cur];
    t.Xo = L.X[a.cur ^ 1];
    t.Do = L.D[a.cur ^ 1];
    t.S = L.S;
    t.k0 = item.k0;
    t.j0 = item.j0;
    t.i0 = item.i0;
    t.i1 = item.i1;
    t.planes = 0;
    const s32::Site32 s = s32::site32_consts<MODE>(c, L.sc);
    double acc[kNV];
#pragma unroll
    for (int q = 0; q < kNV; q++) acc[q] = 0.;
    constexpr int S = ens_ring<MODE>();
    if (item.shape == 0) s32::march32<32, 8, MODE, S, kEnsThreads, -1, true>(c, s, t, ring, acc);
    else if (item.shape == 1) s32::march32<16, 16, MODE, S, kEnsThreads, -1, true>(c, s, t, ring, acc);
    else s32::march32<8, 16, MODE, S, kEnsThreads, -1, true>(c, s, t, ring, acc);
    if constexpr (MODE != MODE_B) {
        block_reduce<kNV>(acc, sred);
        if (tid == 0)
            for (int q = 0; q < kNV; q++) a.partials[(size_t)it * kNV + q] = acc[q];
    }
    // the block that completes a lattice's last item takes its scalar update
    __threadfence();
    __syncthreads();
    if (tid == 0) sflag = atomicAdd(&a.lat_count[item.lat], 1u) == (unsigned)(L.nitems - 1);
    __syncthreads();
    if (!sflag) return;
    __threadfence();
    if constexpr (MODE != MODE_B) {
        double tot[kNV];
        sum_partials<kNV>(a.partials + (size_t)L.first_item * kNV, L.nitems, tot, sred);
        if (tid == 0) finish_a<float, MODE>(c, L.sc, tot, a.slot);
    } else if (tid == 0) {
        finish_b<float>(c, L.sc);
    }
    if (tid == 0) a.lat_count[item.lat] = 0u;
}

// ---------------------------------------------------------------------------
// k-space update over all lattices: block b takes chunk b of the concatenated
// half spectra (chunks never straddle two lattices), the per-point update of
// the single-lattice kernel (kspace.cuh kspace_point)
// ---------------------------------------------------------------------------
constexpr int kEnsKChunk = 4096;  // k-points per block

__device__ __forceinline__ int ens_find_kchunk(const EnsLat *lat, int nlat, int b) {
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (lat[mid].first_kchunk <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) ens_kspace_kernel(EnsArgs a) {
    __shared__ int s_lat;
    if (threadIdx.x == 0) s_lat = ens_find_kchunk(a.lat, a.nlat, blockIdx.x);
    __syncthreads();
    const EnsLat &L = a.lat[s_lat];
    const int N = L.N;
    const size_t M = (size_t)N * N * (N / 2 + 1);
    const size_t m0 = (size_t)(blockIdx.x - L.first_kchunk) * kEnsKChunk;
    const size_t m1 = m0 + kEnsKChunk < M ? m0 + kEnsKChunk : M;
    const KsCoef<float> kc = ks_coef<float>(L.c, L.sc->gw[a.slot]);
    const Cplx<float> *Sc = reinterpret_cast<const Cplx<float> *>(L.S);
    for (size_t idx = m0 + threadIdx.x; idx < m1; idx += blockDim.x) kspace_point<float>(kc, N, M, Sc, L.G, idx);
}

// ---------------------------------------------------------------------------
// initial conditions: Philox 4x32-10 and the randInit distribution
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
    // round constants of the published Philox 4x32 generator
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
        const unsigned hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
        ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
        key.x += W0;
        key.y += W1;
    }
    return ctr;
}

// uniform in (0, 1): never 0, so -log(u) stays finite
__device__ __forceinline__ double u01(unsigned x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

// Half-spectrum modes of one field of every lattice (g2init.cpp:88-172,
// field_full_rand == 1): omega_k = sqrt(k^2 + m2), two (Rayleigh amplitude
// B sqrt(-ln u/(2 omega L^3)), uniform phase) draws per mode, f_k =
// (R1+R2)/sqrt2, fdot_k = i-rotated (R2-R1) omega/sqrt2 - H0 f_k, zero mode 0.
// Writes f_k to complex slot 0 and fdot_k to slot 1 of the lattice's buffer.
__global__ void __launch_bounds__(256) ens_ic_modes_kernel(const EnsLat *lats, int fld, const double *m2,
                                                           double H0, double L, double cut, double smooth,
                                                           int deterministic) {
    const EnsLat &E = lats[blockIdx.y];
    const int N = E.N, nz = N / 2 + 1;
    const size_t M = (size_t)N * N * nz;
    Cplx<float> *fk = reinterpret_cast<Cplx<float> *>(E.S);
    Cplx<float> *fd = fk + M;  // slot stride N*N*(N+2) floats = M complex
    const double dk2 = 4. * M_PI * M_PI / L / L, L3 = L * L * L;
    const double m2e = m2[blockIdx.y];
    const double B = E.rescale_B * E.amp;
    const uint2 key = make_uint2((unsigned)E.seed, (unsigned)(E.seed >> 32) ^ (0x85EBCA6Bu * (unsigned)(fld + 1)));
    const double s2 = sqrt(2.);
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = (int)(t % N), i = (int)(t / N);
        if (i + j + kz == 0) {
            fk[idx] = Cplx<float>{0.f, 0.f};
            fd[idx] = Cplx<float>{0.f, 0.f};
            continue;
        }
        const double i2 = i < N / 2 + 1 ? (double)i * i : (double)(N - i) * (N - i);
        const double j2 = j < N / 2 + 1 ? (double)j * j : (double)(N - j) * (N - j);
        const double n2 = i2 + j2 + (double)kz * kz;
        const double wk = sqrt(dk2 * n2 + m2e);
        // spectral window of spec_cut_off (g2init.cpp:117-165); 1 without a cut-off
        const double win = cut > 0 ? 0.5 * (1. - tanh(smooth * (sqrt(n2) - N * cut))) : 1.;
        if (deterministic) {  // field_full_rand 0: real amplitude, no draws
            const double amp = B * sqrt(1. / (2. * wk * L3)) * win;
            fk[idx] = Cplx<float>{(float)amp, 0.f};
            fd[idx] = Cplx<float>{(float)(-H0 * amp), 0.f};
            continue;
        }
        const uint4 r = philox4x32_10(make_uint4((unsigned)idx, (unsigned)(idx >> 32), 0u, 0u), key);
        const double a1 = win * B * sqrt(-log(u01(r.x)) / (2. * wk * L3)), th1 = 2. * M_PI * u01(r.y);
        const double a2 = win * B * sqrt(-log(u01(r.z)) / (2. * wk * L3)), th2 = 2. * M_PI * u01(r.w);
        const double r1re = a1 * cos(th1), r1im = a1 * sin(th1), r2re = a2 * cos(th2), r2im = a2 * sin(th2);
        const double fre = (r1re + r2re) / s2, fim = (r1im + r2im) / s2;
        fk[idx] = Cplx<float>{(float)fre, (float)fim};
        fd[idx] = Cplx<float>{(float)((r2im - r1im) * wk / s2 - H0 * fre), (float)((r1re - r2re) * wk / s2 - H0 * fim)};
    }
}

// The reference fills the kz = 0 and kz = N/2 planes of the half spectrum
// with independent draws at n and -n; its FFTW-convention c2r then uses the
// Hermitian part of those planes.  cuFFT's c2r expects Hermitian input, so
// this pass replaces each pair (n, -n) on those planes by
// ((X_n + conj X_-n)/2, its conjugate) -- the same real field.
__global__ void ens_ic_symm_kernel(const EnsLat *lats) {
    const EnsLat &E = lats[blockIdx.y];
    const int N = E.N, nz = N / 2 + 1;
    const size_t M = (size_t)N * N * nz;
    Cplx<float> *base = reinterpret_cast<Cplx<float> *>(E.S);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 2 * N * N; q += gridDim.x * blockDim.x) {
        const int kz = (q < N * N) ? 0 : N / 2, ij = q % (N * N);
        const int i = ij / N, j = ij % N;
        const int ip = (N - i) % N, jp = (N - j) % N;
        const size_t a = ((size_t)i * N + j) * nz + kz, b = ((size_t)ip * N + jp) * nz + kz;
        if (a > b) continue;
        for (int s = 0; s < 2; s++) {
            Cplx<float> *X = base + (size_t)s * M;
            const Cplx<float> u = X[a], v = X[b];
            const Cplx<float> m = {0.5f * (u.re + v.re), 0.5f * (u.im - v.im)};
            X[a] = m;
            X[b] = Cplx<float>{m.re, -m.im};
        }
    }
}

// After the in-place c2r: copy the real fields (padded rows) into the state
// as fluctuations, and accumulate sum(delta^2) per lattice (for chi's m_eff).
__global__ void __launch_bounds__(256) ens_ic_place_kernel(const EnsLat *lats, int fld, int cur, double *sumsq) {
    const EnsLat &E = lats[blockIdx.y];
    const int N = E.N;
    const size_t n3 = (size_t)N * N * N, slot = (size_t)N * N * (N + 2);
    const float *rf = E.S, *rd = E.S + slot;
    float *X = E.X[cur] + fld * n3, *D = E.D[cur] + fld * n3;
    double acc = 0.;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n3; x += (size_t)gridDim.x * blockDim.x) {
        const size_t row = x / N, k = x % N;
        const float v = rf[row * (N + 2) + k];
        X[x] = v;
        D[x] = rd[row * (N + 2) + k];
        acc += (double)v * (double)v;
    }
    __shared__ double sred[8];
    double v1[1] = {acc};
    block_reduce<1>(v1, sred);
    if (threadIdx.x == 0) atomicAdd(&sumsq[blockIdx.y], v1[0]);
}

// ---------------------------------------------------------------------------
// spectra: per-lattice native bins, then log bins
// ---------------------------------------------------------------------------
struct EnsBinArgs {
    const EnsLat *lat;
    int nlat, nb_max, nblk, quirk;
    double *part;            // [nlat][nblk][3*nb_max] power sums
    unsigned int *part_cnt;  // [nlat][nblk][nb_max]
};

__global__ void __launch_bounds__(256) ens_bin_kernel(EnsBinArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nb = a.nb_max;
    double *hs = reinterpret_cast<double *>(smem_raw);
    unsigned int *hc = reinterpret_cast<unsigned int *>(hs + 3 * nb);
    for (int q = threadIdx.x; q < 3 * nb; q += blockDim.x) hs[q] = 0.;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) hc[q] = 0u;
    __syncthreads();
    const EnsLat &E = a.lat[blockIdx.y];
    const int N = E.N, nz = N / 2 + 1;
    const size_t M = (size_t)N * N * nz;
    const Cplx<float> *F = reinterpret_cast<const Cplx<float> *>(E.S);
    const double zre[2] = {E.c.gridsize * E.sc->fbar[0], E.c.gridsize * E.sc->fbar[1]};
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < M; idx += (size_t)a.nblk * blockDim.x) {
        const int kz = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = (int)(t % N), i = (int)(t / N);
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        const int b = (int)sqrt((double)px * px + (double)py * py + (double)kz * kz);
        const bool edge = (kz == 0) || (kz == N / 2);
        const double w = edge ? 1.0 : 2.0;
        atomicAdd(&hc[b], edge ? 1u : 2u);
        for (int f = 0; f < 2; f++) {
            double re = (double)F[(size_t)f * M + idx].re, im = (double)F[(size_t)f * M + idx].im;
            if (idx == 0) re += zre[f];
            atomicAdd(&hs[f * nb + b], w * (re * re + im * im));
        }
        if (E.G) {
            const size_t src = (a.quirk && kz == 0) ? idx + (size_t)(N / 2) : idx;
            const Cplx<float> lp = E.G[2 * M + src], lx = E.G[3 * M + src];
            const double p =
                2. * (((double)lp.re * lp.re + (double)lp.im * lp.im) + ((double)lx.re * lx.re + (double)lx.im * lx.im));
            atomicAdd(&hs[2 * nb + b], w * p);
        }
    }
    __syncthreads();
    double *ps = a.part + ((size_t)blockIdx.y * a.nblk + blockIdx.x) * 3 * nb;
    unsigned int *pc = a.part_cnt + ((size_t)blockIdx.y * a.nblk + blockIdx.x) * nb;
    for (int q = threadIdx.x; q < 3 * nb; q += blockDim.x) ps[q] = hs[q];
    for (int q = threadIdx.x; q < nb; q += blockDim.x) pc[q] = hc[q];
}

// One block per lattice: native sums (fixed order over blocks), then log bins
// whose values are count-weighted means of the native bins' values, i.e.
//   P = spec_norm sum(S_b)/sum(n_b),  Delta^2 = spec_norm/(2 pi^2) sum(k_b^3 S_b)/sum(n_b),
//   Omega_gw = norm1 sum(k_b^3 S_b)/sum(n_b)   (g2spectra.cpp:94-103, 186-195),
// over native bins b >= 1 with log-spaced edges in b (b_lo = 1, b_hi = nb_max).
// out: [nlat][3][nlog] log10 of (Delta^2_phi, Delta^2_chi, Omega_gw), NaN where
// a log bin holds no native bin; cnt: [nlat][nlog]; native: [nlat][4][nb_max]
// (sums of phi, chi, GW and counts) for exact checks.
__global__ void ens_rebin_kernel(EnsBinArgs a, int nlog, double hi, double L, double *out, double *cnt, double *native) {
    const int e = blockIdx.x, nb = a.nb_max;
    const EnsLat &E = a.lat[e];
    const int N = E.N;
    const int nbe = (int)(sqrt(3.) * N / 2 + 1);  // native bins of this lattice
    double *nat = native + (size_t)e * 4 * nb;
    for (int q = threadIdx.x; q < 4 * nb; q += blockDim.x) {
        const int s = q / nb, b = q % nb;
        double v = 0.;
        for (int k = 0; k < a.nblk; k++) {
            const size_t base = ((size_t)e * a.nblk + k);
            v += s < 3 ? a.part[base * 3 * nb + (size_t)s * nb + b] : (double)a.part_cnt[base * nb + b];
        }
        nat[q] = b < nbe ? v : 0.;
    }
    __syncthreads();
    const double spec_norm = pow(L / (double)N, 6.) * pow(2. * M_PI / L, 3.);
    const double hub = sqrt(8. * M_PI / 3.) * sqrt(E.sc->edrho[0]);
    const double norm1 = 4.e-5 / pow(100., .333) / 24. / M_PI / M_PI / pow(L, 3.) / (hub * hub);
    const double lo = 1.0;
    for (int q = threadIdx.x; q < nlog; q += blockDim.x) {
        const double e0 = lo * pow(hi / lo, (double)q / nlog), e1 = lo * pow(hi / lo, (double)(q + 1) / nlog);
        double n = 0., s0 = 0., s1 = 0., s2 = 0.;
        for (int b = 1; b < nbe; b++) {
            const double bb = (double)b;
            if (bb < e0 || (q + 1 < nlog ? bb >= e1 : bb > e1)) continue;
            const double k3 = pow(bb * 2. * M_PI / L, 3.);
            n += nat[3 * nb + b];
            s0 += k3 * nat[b];
            s1 += k3 * nat[nb + b];
            s2 += k3 * nat[2 * nb + b];
        }
        double *o = out + (size_t)e * 3 * nlog;
        cnt[(size_t)e * nlog + q] = n;
        if (n > 0) {
            o[q] = log10(spec_norm * s0 / n / 2. / M_PI / M_PI);
            o[nlog + q] = log10(spec_norm * s1 / n / 2. / M_PI / M_PI);
            o[2 * nlog + q] = log10(norm1 * s2 / n);
        } else {
            o[q] = o[nlog + q] = o[2 * nlog + q] = CUDART_NAN;
        }
    }
}

}  // namespace gabe
