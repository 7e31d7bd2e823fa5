// Batched ensemble: many independent lattices of uneven size, coupling,
// amplitude and seed evolved together (FP32 storage, FP64 scalars).
//
// Each step is the single-lattice step (stencil.cuh, kspace.cuh) issued once
// for the whole ensemble:
//   * sweep A and sweep B are persistent kernels over a work list of
//     (lattice, column tile, plane chunk) items, 256 threads per block; each
//     item runs the same per-tile march as the single-lattice kernel with the
//     tile shape the autotuner chose for that lattice size (32x8 or 16x16);
//     per-item partial sums are combined by the block that finishes the last
//     item of a lattice, in item order, so every lattice gets its own
//     Friedmann update without a grid-wide barrier;
//   * the GW transforms are one cuFFT call per lattice size (batch = 10 x
//     lattices of that size, sources of a size group contiguous);
//   * the k-space update is one kernel over the concatenated half spectra.
// The initial state is drawn on the device with the reference's randInit
// distribution (g2init.cpp:68-189) from a counter-based generator (Philox
// 4x32-10, Salmon et al., SC'11), so it matches the reference in
// distribution, not bit for bit.
#pragma once

#include <math_constants.h>

#include "kspace.cuh"
#include "stencil.cuh"

namespace gabe {

struct EnsLat {
    LatticeConsts c;
    float *X[2], *D[2];  // [2 fields][N^3] each, ping-pong
    float *S;            // [10][N][N][N+2] sources / [..][N][N][N/2+1] spectra
    Cplx<float> *G;      // [4][M] h+, hx, l+, lx
    DevScalars *sc;
    size_t kofs;         // offset of this lattice's k-points in the ensemble k index
    int first_item, nitems;
    int N, pad;
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
// persistent sweep over the work list
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(256, 2) ens_sweep_kernel(EnsArgs a) {
    __shared__ __align__(16) float smem[2][4 * SweepSmem<32, 8>::P];
    __shared__ double sred[8 * kNV];
    __shared__ int sflag;
    static_assert(SweepSmem<16, 16>::P <= SweepSmem<32, 8>::P, "shared tile too small");
    const int tid = threadIdx.x;
    for (int it = blockIdx.x; it < a.nitems; it += gridDim.x) {
        const EnsItem item = a.items[it];
        const EnsLat &L = a.lat[item.lat];
        const LatticeConsts c = L.c;
        TileJob<float> job;
        job.X = L.X[a.cur];
        job.D = L.D[a.cur];
        job.Xo = L.X[a.cur ^ 1];
        job.Do = L.D[a.cur ^ 1];
        job.S = L.S;
        job.sc = L.sc;
        job.j0 = item.j0;
        job.k0 = item.k0;
        job.i0 = item.i0;
        job.i1 = item.i1;
        double acc[kNV];
#pragma unroll
        for (int q = 0; q < kNV; q++) acc[q] = 0.;
        if (item.shape == 0) sweep_tile<float, 32, 8, MODE>(c, job, smem[0], smem[1], acc);
        else sweep_tile<float, 16, 16, MODE>(c, job, smem[0], smem[1], acc);
        if constexpr (MODE != MODE_B) {
            block_reduce<kNV>(acc, sred);
            if (tid == 0)
                for (int q = 0; q < kNV; q++) a.partials[(size_t)it * kNV + q] = acc[q];
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) sflag = atomicAdd(&a.lat_count[item.lat], 1u) == (unsigned)(L.nitems - 1);
        __syncthreads();
        if (sflag) {
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
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k-space update over all lattices (same per-point arithmetic as kspace.cuh)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ens_find(const EnsLat *lat, int nlat, size_t g) {
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (lat[mid].kofs <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) ens_kspace_kernel(EnsArgs a, size_t ktotal) {
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < ktotal; g += (size_t)gridDim.x * blockDim.x) {
        const int e = ens_find(a.lat, a.nlat, g);
        const EnsLat &L = a.lat[e];
        const int N = L.N, nz = N / 2 + 1;
        const size_t M = (size_t)N * N * nz, idx = g - L.kofs;
        const double *g4 = L.sc->gw[a.slot];
        const double a0 = g4[0], ad0 = g4[1], a1 = g4[2], ad1 = g4[3];
        const LatticeConsts &c = L.c;
        const Cplx<float> *Sc = reinterpret_cast<const Cplx<float> *>(L.S);
        Cplx<float> s[10], gg[4];
#pragma unroll
        for (int q = 0; q < 10; q++) s[q] = Sc[(size_t)q * M + idx];
#pragma unroll
        for (int q = 0; q < 4; q++) gg[q] = L.G[(size_t)q * M + idx];
        const int kzi = (int)(idx % nz);
        const size_t t = idx / nz;
        const int j = (int)(t % N), i = (int)(t / N);
        const int px = i <= N / 2 ? i : i - N, py = j <= N / 2 ? j : j - N;
        const double m2 = ((double)px * px + (double)py * py) + (double)kzi * kzi;
        if (m2 == 0.0) continue;
        double ep[6], ex[6];
        pol_tensors(px, py, kzi, ep, ex);
        const float wp[5] = {(float)(0.5 * (ep[0] - ep[5])), (float)ep[1], (float)ep[2], (float)(0.5 * (ep[3] - ep[5])),
                             (float)ep[4]};
        const float wx[5] = {(float)(0.5 * (ex[0] - ex[5])), (float)ex[1], (float)ex[2], (float)(0.5 * (ex[3] - ex[5])),
                             (float)ex[4]};
        const float kk0 = (float)(m2 * (c.k2norm_c / a0 / a0)), kk1 = (float)(m2 * (c.k2norm_c / a1 / a1));
        const float c3H0 = (float)(3. * ad0 / a0), c3H1 = (float)(3. * ad1 / a1);
        const float src0 = (float)(2. * (c.eight_pi / a0 / a0) * c.normmm);
        const float src1 = (float)(2. * (c.eight_pi / a1 / a1) * c.normmm);
        const float hdt = (float)c.half_dt, dt = (float)c.dt;
        float Tp[2][2][2];
#pragma unroll
        for (int st = 0; st < 2; st++) {
            float sr[5], si[5];
#pragma unroll
            for (int q = 0; q < 5; q++) { sr[q] = s[5 * st + q].re; si[q] = s[5 * st + q].im; }
            const float f = st == 0 ? src0 : src1;
            Tp[st][0][0] = f * pol_contract(wp, sr);
            Tp[st][0][1] = f * pol_contract(wp, si);
            Tp[st][1][0] = f * pol_contract(wx, sr);
            Tp[st][1][1] = f * pol_contract(wx, si);
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
            Cplx<float> hn, ln;
#pragma unroll
            for (int ri = 0; ri < 2; ri++) {
                const float h0 = ri ? gg[p].im : gg[p].re, l0 = ri ? gg[2 + p].im : gg[2 + p].re;
                const float ld0 = -kk0 * h0 - c3H0 * l0 + Tp[0][p][ri];
                const float h1 = h0 + hdt * l0;
                const float l1 = l0 + hdt * ld0;
                const float ld1 = -kk1 * h1 - c3H1 * l1 + Tp[1][p][ri];
                (ri ? hn.im : hn.re) = h0 + dt * l1;
                (ri ? ln.im : ln.re) = l0 + dt * ld1;
            }
            L.G[(size_t)p * M + idx] = hn;
            L.G[(size_t)(2 + p) * M + idx] = ln;
        }
    }
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
                                                           double H0, double L) {
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
        const double wk = sqrt(dk2 * (i2 + j2 + (double)kz * kz) + m2e);
        const uint4 r = philox4x32_10(make_uint4((unsigned)idx, (unsigned)(idx >> 32), 0u, 0u), key);
        const double a1 = B * sqrt(-log(u01(r.x)) / (2. * wk * L3)), th1 = 2. * M_PI * u01(r.y);
        const double a2 = B * sqrt(-log(u01(r.z)) / (2. * wk * L3)), th2 = 2. * M_PI * u01(r.w);
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
