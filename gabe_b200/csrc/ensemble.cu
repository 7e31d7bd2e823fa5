// Host side of the batched ensemble (include/gabe.h, gabe_ensemble_*).
//
// Lattices are grouped by size.  Each size group owns contiguous pools
// (state ping-pong, GW sources, GW amplitudes) so that one cuFFT call per
// group transforms the sources of all its lattices, and the work list of the
// persistent sweeps holds every lattice's column tiles.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/gabe.h"
#include "ensemble.cuh"
#include "launch.h"

using namespace gabe;

namespace {
thread_local std::string g_ens_create_error;
constexpr int kEnsBinBlocks = 32;  // binning blocks per lattice
}  // namespace

struct gabe_ensemble {
    int nlat = 0, dev = 0, nlog = 0, quirk = 1, gws = 1, flags = 0, ic_det = 0;
    double spec_cut = 0., spec_smooth = 0.5;
    double L = 20., dt = 0.01, lambda = 9e-14, phi0 = 0.342, dphi0 = 0.;
    std::vector<int> N, shape, ci;
    std::vector<double> g, amp;
    std::vector<unsigned long long> seed;
    cudaStream_t stream = nullptr;
    struct Group {
        int N = 0;
        std::vector<int> lats;
        float *X[2] = {nullptr, nullptr}, *D[2] = {nullptr, nullptr}, *S = nullptr;
        Cplx<float> *G = nullptr;
        cufftHandle plan_src = 0, plan_ic = 0, plan_spec = 0;
        bool have_src = false, have_ic = false, have_spec = false;
    };
    std::vector<Group> groups;
    std::vector<EnsLat> h_lat;
    EnsLat *d_lat = nullptr;
    EnsItem *d_items = nullptr;
    int nitems = 0;
    double *d_partials = nullptr;
    unsigned int *d_lat_count = nullptr;
    DevScalars *d_sc = nullptr;
    int nkchunks = 0;
    void *fft_work = nullptr;
    double *d_m2 = nullptr, *d_sumsq = nullptr;
    double *d_part = nullptr, *d_log = nullptr, *d_logcnt = nullptr, *d_native = nullptr;
    unsigned int *d_part_cnt = nullptr;
    int nb_max = 0;
    int log_top = 0;  // upper end of the log bins, native-bin units
    int cur = 0;
    bool ready = false, e0_stale = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graph_tried = false, graph_ok = false;
    size_t dev_bytes = 0;
    std::vector<void *> allocs;
    std::string err;
};

namespace {

int eset(gabe_ensemble *e, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (e) e->err = buf;
    else g_ens_create_error = buf;
    return code;
}

#define ECK(e, x)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess) return eset(e, GABE_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)
#define ECF(e, x)                                                                                  \
    do {                                                                                           \
        cufftResult r_ = (x);                                                                      \
        if (r_ != CUFFT_SUCCESS) return eset(e, GABE_ERR_CUFFT, "%s: cufft error %d", #x, (int)r_); \
    } while (0)

int ealloc(gabe_ensemble *e, void **p, size_t bytes) {
    if (bytes == 0) bytes = 256;
    cudaError_t r = cudaMalloc(p, bytes);
    if (r != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return eset(e, GABE_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(r));
    }
    e->allocs.push_back(*p);
    e->dev_bytes += bytes;
    return GABE_OK;
}

gabe_params lattice_params(const gabe_ensemble *e, int l) {
    gabe_params p;
    gabe_default_params(&p, e->N[l]);
    p.L = e->L;
    p.dt = e->dt;
    p.model = GABE_MODEL_LPHI4;
    p.model_c[0] = 1. / (e->phi0 * e->phi0);
    p.model_c[1] = e->g[l] / (e->phi0 * e->phi0);
    p.precision = GABE_FP32;
    p.gws_on = e->gws;
    return p;
}

int make_plans(gabe_ensemble *e) {
    size_t wmax = 0;
    for (auto &G : e->groups) {
        const long long N = G.N, nz = N / 2 + 1, ng = (long long)G.lats.size();
        long long n[3] = {N, N, N};
        const long long slot_r = N * N * 2 * nz, slot_c = N * N * nz;  // one source slot in reals / complex
        size_t w = 0;
        if (e->gws) {
            long long inem[3] = {N, N, 2 * nz}, onem[3] = {N, N, nz};
            ECF(e, cufftCreate(&G.plan_src));
            G.have_src = true;
            ECF(e, cufftSetAutoAllocation(G.plan_src, 0));
            ECF(e, cufftMakePlanMany64(G.plan_src, 3, n, inem, 1, slot_r, onem, 1, slot_c, CUFFT_R2C, 2 * kSrc * ng, &w));
            wmax = std::max(wmax, w);
        }
        {   // initial conditions: c2r of slot 0 (or 1) of every lattice of the group, in place
            long long inem[3] = {N, N, nz}, onem[3] = {N, N, 2 * nz};
            ECF(e, cufftCreate(&G.plan_ic));
            G.have_ic = true;
            ECF(e, cufftSetAutoAllocation(G.plan_ic, 0));
            ECF(e, cufftMakePlanMany64(G.plan_ic, 3, n, inem, 1, 2 * kSrc * slot_c, onem, 1, 2 * kSrc * slot_r,
                                       CUFFT_C2R, ng, &w));
            wmax = std::max(wmax, w);
        }
        {   // spectra: field f of every lattice -> slot f of its source region
            long long inem[3] = {N, N, N}, onem[3] = {N, N, nz};
            ECF(e, cufftCreate(&G.plan_spec));
            G.have_spec = true;
            ECF(e, cufftSetAutoAllocation(G.plan_spec, 0));
            ECF(e, cufftMakePlanMany64(G.plan_spec, 3, n, inem, 1, 2 * N * N * N, onem, 1, 2 * kSrc * slot_c,
                                       CUFFT_R2C, ng, &w));
            wmax = std::max(wmax, w);
        }
    }
    int rc = ealloc(e, &e->fft_work, wmax);
    if (rc) return rc;
    for (auto &G : e->groups) {
        if (G.have_src) {
            ECF(e, cufftSetWorkArea(G.plan_src, e->fft_work));
            ECF(e, cufftSetStream(G.plan_src, e->stream));
        }
        ECF(e, cufftSetWorkArea(G.plan_ic, e->fft_work));
        ECF(e, cufftSetStream(G.plan_ic, e->stream));
        ECF(e, cufftSetWorkArea(G.plan_spec, e->fft_work));
        ECF(e, cufftSetStream(G.plan_spec, e->stream));
    }
    return GABE_OK;
}

EnsArgs ens_args(gabe_ensemble *e, int cur) {
    EnsArgs a{};
    a.lat = e->d_lat;
    a.items = e->d_items;
    a.nitems = e->nitems;
    a.nlat = e->nlat;
    a.cur = cur;
    a.slot = 0;
    a.partials = e->d_partials;
    a.lat_count = e->d_lat_count;
    return a;
}

template <int MODE>
cudaError_t launch_sweep(const EnsArgs &a, cudaStream_t s) {
    constexpr size_t smem = ens_ring_bytes<MODE>();
    cudaError_t r = cudaFuncSetAttribute(ens_sweep_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    ens_sweep_kernel<MODE><<<a.nitems, kEnsThreads, smem, s>>>(a);
    return cudaGetLastError();
}

int sweep(gabe_ensemble *e, int mode, int cur) {
    EnsArgs a = ens_args(e, cur);
    switch (mode) {
        case MODE_A: ECK(e, launch_sweep<MODE_A>(a, e->stream)); break;
        case MODE_A_GW: ECK(e, launch_sweep<MODE_A_GW>(a, e->stream)); break;
        case MODE_E0: ECK(e, launch_sweep<MODE_E0>(a, e->stream)); break;
        default: ECK(e, launch_sweep<MODE_B>(a, e->stream)); break;
    }
    return GABE_OK;
}

int enqueue_step(gabe_ensemble *e, int cur) {
    int rc = sweep(e, e->gws ? MODE_A_GW : MODE_A, cur);
    if (rc) return rc;
    if (e->gws) {
        for (auto &G : e->groups) ECF(e, cufftExecR2C(G.plan_src, (cufftReal *)G.S, (cufftComplex *)G.S));
        ens_kspace_kernel<<<e->nkchunks, 256, 0, e->stream>>>(ens_args(e, cur));
        ECK(e, cudaGetLastError());
    }
    return sweep(e, MODE_B, cur);
}

int refresh_e0(gabe_ensemble *e) {
    if (!e->e0_stale) return GABE_OK;
    int rc = sweep(e, MODE_E0, e->cur);
    if (rc) return rc;
    e->e0_stale = false;
    return GABE_OK;
}

size_t lattice_M(int N) { return (size_t)N * N * (N / 2 + 1); }

}  // namespace

extern "C" {

int gabe_ensemble_create(const gabe_ensemble_params *p, gabe_ensemble **out) {
    if (!out) return eset(nullptr, GABE_ERR_PARAM, "out is NULL");
    *out = nullptr;
    if (!p || p->struct_size != (int32_t)sizeof(gabe_ensemble_params))
        return eset(nullptr, GABE_ERR_PARAM, "bad gabe_ensemble_params");
    if (p->nlat < 1 || !p->N || !p->g2_over_lambda || !p->amplitude || !p->seed)
        return eset(nullptr, GABE_ERR_PARAM, "nlat and the per-lattice arrays are required");
    if (!(p->L > 0) || !(p->dt > 0) || !(p->lambda > 0) || !(p->phi0 != 0) || p->nlog < 1 || p->nlog > 4096 ||
        p->log_top_bin < 0 || p->log_top_bin > (1 << 20) || !(p->spec_cut_off >= 0) ||
        (p->spec_cut_off > 0 && !(p->spec_smooth > 0 && std::isfinite(p->spec_smooth))) ||
        (p->ic_deterministic != 0 && p->ic_deterministic != 1) || (p->ic_deterministic && !(p->spec_cut_off > 0)))
        return eset(nullptr, GABE_ERR_PARAM, "invalid shared parameters");
    for (int l = 0; l < p->nlat; l++) {
        const int n = p->N[l];
        if (n < 16 || n > 1024 || n % 16) return eset(nullptr, GABE_ERR_PARAM, "lattice %d: N=%d must be a multiple of 16 in [16,1024]", l, n);
        if (!(p->g2_over_lambda[l] >= 0) || !(p->amplitude[l] >= 0))
            return eset(nullptr, GABE_ERR_PARAM, "lattice %d: invalid coupling or amplitude", l);
        if (p->tile_shape && (p->tile_shape[l] < 0 || p->tile_shape[l] > 2 || n % ens_tile_k(p->tile_shape[l])))
            return eset(nullptr, GABE_ERR_PARAM,
                        "lattice %d: tile shape must be 0 (64x8, N%%64==0), 1 (32x16, N%%32==0) or 2 (16x16)", l);
    }
    gabe_ensemble *e = new (std::nothrow) gabe_ensemble();
    if (!e) return eset(nullptr, GABE_ERR_NOMEM, "host allocation failed");
    auto bail = [&](int code) {
        g_ens_create_error = e->err;
        gabe_ensemble_destroy(e);
        return code;
    };
    e->nlat = p->nlat;
    e->L = p->L; e->dt = p->dt; e->lambda = p->lambda; e->phi0 = p->phi0; e->dphi0 = p->dphi0;
    e->gws = p->gws_on ? 1 : 0;
    e->nlog = p->nlog;
    e->quirk = p->gw_spec_quirk;
    e->spec_cut = p->spec_cut_off;
    e->spec_smooth = p->spec_smooth;
    e->ic_det = p->ic_deterministic;
    e->flags = p->flags;
    e->N.assign(p->N, p->N + p->nlat);
    e->g.assign(p->g2_over_lambda, p->g2_over_lambda + p->nlat);
    e->amp.assign(p->amplitude, p->amplitude + p->nlat);
    e->seed.assign(p->seed, p->seed + p->nlat);
    for (int l = 0; l < p->nlat; l++) {
        e->shape.push_back(p->tile_shape ? p->tile_shape[l] : (e->N[l] % 64 == 0 ? 0 : (e->N[l] % 32 == 0 ? 1 : 2)));
        int c = p->tile_ci && p->tile_ci[l] > 0 ? p->tile_ci[l] : 32;
        e->ci.push_back(std::min(c, e->N[l]));
    }
    if (p->device >= 0 && cudaSetDevice(p->device) != cudaSuccess) {
        cudaGetLastError();
        eset(e, GABE_ERR_CUDA, "cudaSetDevice(%d) failed", p->device);
        return bail(GABE_ERR_CUDA);
    }
    if (cudaGetDevice(&e->dev) != cudaSuccess || cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        eset(e, GABE_ERR_CUDA, "no CUDA device");
        return bail(GABE_ERR_CUDA);
    }
    // size groups, in order of first appearance
    std::map<int, int> gidx;
    for (int l = 0; l < e->nlat; l++) {
        auto it = gidx.find(e->N[l]);
        if (it == gidx.end()) {
            gidx[e->N[l]] = (int)e->groups.size();
            e->groups.push_back({});
            e->groups.back().N = e->N[l];
        }
        e->groups[gidx[e->N[l]]].lats.push_back(l);
    }
    int rc;
    if ((rc = ealloc(e, (void **)&e->d_sc, sizeof(DevScalars) * e->nlat))) return bail(rc);
    e->h_lat.resize(e->nlat);
    for (auto &G : e->groups) {
        const size_t N = G.N, n3 = N * N * N, ng = G.lats.size();
        const size_t slot_r = N * N * (N + 2), M = lattice_M(G.N);
        for (int b = 0; b < 2; b++) {
            if ((rc = ealloc(e, (void **)&G.X[b], ng * 2 * n3 * sizeof(float)))) return bail(rc);
            if ((rc = ealloc(e, (void **)&G.D[b], ng * 2 * n3 * sizeof(float)))) return bail(rc);
        }
        if ((rc = ealloc(e, (void **)&G.S, ng * 2 * kSrc * slot_r * sizeof(float)))) return bail(rc);
        if (e->gws && (rc = ealloc(e, (void **)&G.G, ng * 4 * M * sizeof(Cplx<float>)))) return bail(rc);
        for (size_t q = 0; q < ng; q++) {
            const int l = G.lats[q];
            EnsLat &Lt = e->h_lat[l];
            std::memset(&Lt, 0, sizeof(Lt));
            gabe_params lp = lattice_params(e, l);
            Lt.c = make_lattice_consts(lp);
            for (int b = 0; b < 2; b++) {
                Lt.X[b] = G.X[b] + q * 2 * n3;
                Lt.D[b] = G.D[b] + q * 2 * n3;
            }
            Lt.S = G.S + q * 2 * kSrc * slot_r;
            Lt.G = e->gws ? G.G + q * 4 * M : nullptr;
            Lt.sc = e->d_sc + l;
            Lt.N = G.N;
            Lt.seed = e->seed[l];
            Lt.amp = e->amp[l];
            Lt.rescale_B = std::sqrt(e->lambda) * e->phi0;
        }
    }
    // work list (lattice-major) and the k-space chunks of every lattice
    std::vector<EnsItem> items;
    size_t nkc = 0;
    for (int l = 0; l < e->nlat; l++) {
        EnsLat &Lt = e->h_lat[l];
        const int n = e->N[l], TK = ens_tile_k(e->shape[l]), TJ = ens_tile_j(e->shape[l]), c = e->ci[l];
        Lt.first_item = (int)items.size();
        for (int i0 = 0; i0 < n; i0 += c)
            for (int j0 = 0; j0 < n; j0 += TJ)
                for (int k0 = 0; k0 < n; k0 += TK) items.push_back({l, e->shape[l], j0, k0, i0, std::min(i0 + c, n)});
        Lt.nitems = (int)items.size() - Lt.first_item;
        Lt.first_kchunk = (int)nkc;
        nkc += (lattice_M(n) + kEnsKChunk - 1) / kEnsKChunk;
    }
    if (items.size() > (size_t)INT32_MAX || nkc > (size_t)INT32_MAX) {
        eset(e, GABE_ERR_PARAM, "ensemble too large for one launch");
        return bail(GABE_ERR_PARAM);
    }
    e->nitems = (int)items.size();
    e->nkchunks = (int)nkc;
    if ((rc = ealloc(e, (void **)&e->d_lat, sizeof(EnsLat) * e->nlat))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_items, sizeof(EnsItem) * e->nitems))) return bail(rc);
    // per-item partial sums; also the scratch of the upload's mean reduction (256 blocks)
    if ((rc = ealloc(e, (void **)&e->d_partials, sizeof(double) * std::max(kNV * e->nitems, 4096)))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_lat_count, sizeof(unsigned int) * e->nlat))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_m2, sizeof(double) * e->nlat))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_sumsq, sizeof(double) * e->nlat))) return bail(rc);
    int nmax = *std::max_element(e->N.begin(), e->N.end());
    e->nb_max = gabe_spectra_numbins(nmax);
    e->log_top = p->log_top_bin > 0 ? p->log_top_bin : e->nb_max;
    if ((rc = ealloc(e, (void **)&e->d_part, sizeof(double) * e->nlat * kEnsBinBlocks * 3 * e->nb_max))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_part_cnt, sizeof(unsigned) * e->nlat * kEnsBinBlocks * e->nb_max))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_log, sizeof(double) * e->nlat * 3 * e->nlog))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_logcnt, sizeof(double) * e->nlat * e->nlog))) return bail(rc);
    if ((rc = ealloc(e, (void **)&e->d_native, sizeof(double) * e->nlat * 4 * e->nb_max))) return bail(rc);
    if (cudaMemcpy(e->d_lat, e->h_lat.data(), sizeof(EnsLat) * e->nlat, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(e->d_items, items.data(), sizeof(EnsItem) * e->nitems, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(e->d_lat_count, 0, sizeof(unsigned) * e->nlat) != cudaSuccess ||
        cudaMemset(e->d_sc, 0, sizeof(DevScalars) * e->nlat) != cudaSuccess) {
        cudaGetLastError();
        eset(e, GABE_ERR_CUDA, "ensemble set-up copies failed");
        return bail(GABE_ERR_CUDA);
    }
    for (auto &G : e->groups)
        if (G.G && cudaMemset(G.G, 0, G.lats.size() * 4 * lattice_M(G.N) * sizeof(Cplx<float>)) != cudaSuccess) {
            cudaGetLastError();
            eset(e, GABE_ERR_CUDA, "cudaMemset failed");
            return bail(GABE_ERR_CUDA);
        }
    if ((rc = make_plans(e))) return bail(rc);
    *out = e;
    return GABE_OK;
}

int gabe_ensemble_destroy(gabe_ensemble *e) {
    if (!e) return GABE_OK;
    cudaSetDevice(e->dev);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (int i = 0; i < 2; i++)
        if (e->graph[i]) cudaGraphExecDestroy(e->graph[i]);
    for (auto &G : e->groups) {
        if (G.have_src) cufftDestroy(G.plan_src);
        if (G.have_ic) cufftDestroy(G.plan_ic);
        if (G.have_spec) cufftDestroy(G.plan_spec);
    }
    for (void *p : e->allocs) cudaFree(p);
    if (e->stream) cudaStreamDestroy(e->stream);
    cudaGetLastError();
    delete e;
    return GABE_OK;
}

static int set_homogeneous_scalars(gabe_ensemble *e, double *H0) {
    // initexpansion (g2init.cpp:26-29) for the homogeneous state: a = 1,
    // adot = adf of kinetic + potential energy (the gradient energy is zero)
    const double lam_pr = 1. / (e->phi0 * e->phi0);
    const double rho = 0.5 * e->dphi0 * e->dphi0 + 0.25 * lam_pr * e->phi0 * e->phi0 * e->phi0 * e->phi0;
    *H0 = std::sqrt(8. * M_PI / 3. * rho);
    std::vector<DevScalars> s(e->nlat);
    for (int l = 0; l < e->nlat; l++) {
        std::memset(&s[l], 0, sizeof(DevScalars));
        s[l].a[0] = 1.;
        s[l].adot[0] = *H0;
        s[l].adot_given = 1;
        s[l].fbar[0] = e->phi0;
        s[l].dfbar[0] = e->dphi0;
    }
    ECK(e, cudaMemcpyAsync(e->d_sc, s.data(), sizeof(DevScalars) * e->nlat, cudaMemcpyHostToDevice, e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    return GABE_OK;
}

int gabe_ensemble_init(gabe_ensemble *e) {
    if (!e) return GABE_ERR_PARAM;
    ECK(e, cudaSetDevice(e->dev));
    double H0 = 0;
    int rc = set_homogeneous_scalars(e, &H0);
    if (rc) return rc;
    e->cur = 0;
    int nmax = *std::max_element(e->N.begin(), e->N.end());
    const unsigned gx = (unsigned)std::min<size_t>(1024, (lattice_M(nmax) + 255) / 256);
    const double lam_pr = 1. / (e->phi0 * e->phi0);
    // phi: m_eff^2 = <3 lam phi^2 + g chi^2> = 3 lam phi0^2 (chi = 0)  (effMass, g2model.cpp:89-108)
    std::vector<double> m2(e->nlat, 3. * lam_pr * e->phi0 * e->phi0);
    for (int fld = 0; fld < 2; fld++) {
        ECK(e, cudaMemcpyAsync(e->d_m2, m2.data(), sizeof(double) * e->nlat, cudaMemcpyHostToDevice, e->stream));
        ens_ic_modes_kernel<<<dim3(gx, e->nlat), 256, 0, e->stream>>>(e->d_lat, fld, e->d_m2, H0, e->L, e->spec_cut,
                                                                    e->spec_smooth, e->ic_det);
        ECK(e, cudaGetLastError());
        ens_ic_symm_kernel<<<dim3(64, e->nlat), 256, 0, e->stream>>>(e->d_lat);
        ECK(e, cudaGetLastError());
        for (auto &G : e->groups) {
            const size_t slot_r = (size_t)G.N * G.N * (G.N + 2);
            for (int s = 0; s < 2; s++)
                ECF(e, cufftExecC2R(G.plan_ic, (cufftComplex *)(G.S + s * slot_r), (cufftReal *)(G.S + s * slot_r)));
        }
        ECK(e, cudaMemsetAsync(e->d_sumsq, 0, sizeof(double) * e->nlat, e->stream));
        ens_ic_place_kernel<<<dim3(gx, e->nlat), 256, 0, e->stream>>>(e->d_lat, fld, 0, e->d_sumsq);
        ECK(e, cudaGetLastError());
        if (fld == 0) {
            // chi: m_eff^2 = g <phi^2> = g (phi0^2 + <dphi^2>) of the fluctuated phi
            std::vector<double> ss(e->nlat);
            ECK(e, cudaMemcpyAsync(ss.data(), e->d_sumsq, sizeof(double) * e->nlat, cudaMemcpyDeviceToHost, e->stream));
            ECK(e, cudaStreamSynchronize(e->stream));
            for (int l = 0; l < e->nlat; l++) {
                const double n3 = (double)e->N[l] * e->N[l] * e->N[l];
                m2[l] = (e->g[l] / (e->phi0 * e->phi0)) * (e->phi0 * e->phi0 + ss[l] / n3);
            }
        }
    }
    for (auto &G : e->groups)
        if (G.G) ECK(e, cudaMemsetAsync(G.G, 0, G.lats.size() * 4 * lattice_M(G.N) * sizeof(Cplx<float>), e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    e->ready = true;
    e->e0_stale = true;
    return GABE_OK;
}

int gabe_ensemble_upload(gabe_ensemble *e, int lat, const double *field0, const double *dfield0, double a0,
                         double adot0) {
    if (!e || lat < 0 || lat >= e->nlat || !field0 || !dfield0 || !(a0 > 0) || !std::isfinite(a0) ||
        !std::isfinite(adot0))
        return GABE_ERR_PARAM;
    // an upload replaces one lattice's state; the others must hold one already, or the ensemble would step
    // uninitialised lattices beside it
    if (!e->ready) return eset(e, GABE_ERR_STATE, "upload before gabe_ensemble_init (it draws every lattice's state)");
    ECK(e, cudaSetDevice(e->dev));
    const EnsLat &Lt = e->h_lat[lat];
    const size_t n3 = (size_t)Lt.N * Lt.N * Lt.N;
    double *stage = reinterpret_cast<double *>(Lt.S);
    DevScalars s{};
    s.a[0] = a0;
    s.adot[0] = adot0;
    s.adot_given = 1;
    ECK(e, cudaMemcpyAsync(Lt.sc, &s, sizeof(s), cudaMemcpyHostToDevice, e->stream));
    const double *src[2] = {field0, dfield0};
    float *const *dstb[2] = {Lt.X, Lt.D};
    for (int a = 0; a < 2; a++)
        for (int f = 0; f < 2; f++) {
            double *mean = reinterpret_cast<double *>(reinterpret_cast<char *>(Lt.sc) +
                                                      (a ? offsetof(DevScalars, dfbar) : offsetof(DevScalars, fbar))) + f;
            ECK(e, cudaMemcpyAsync(stage, src[a] + f * n3, n3 * 8, cudaMemcpyHostToDevice, e->stream));
            ECK(e, mean_f64(stage, n3, e->d_partials, e->d_lat_count + lat, mean, 256, e->stream));
            ECK(e, to_fluct(stage, n3, mean, dstb[a][e->cur] + f * n3, e->stream));
        }
    if (Lt.G) ECK(e, cudaMemsetAsync(Lt.G, 0, 4 * lattice_M(Lt.N) * sizeof(Cplx<float>), e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    e->ready = true;
    e->e0_stale = true;
    return GABE_OK;
}

int gabe_ensemble_step(gabe_ensemble *e, int nsteps) {
    if (!e || nsteps < 0) return GABE_ERR_PARAM;
    if (!e->ready) return eset(e, GABE_ERR_STATE, "step before init/upload");
    ECK(e, cudaSetDevice(e->dev));
    if (!e->graph_tried) {
        e->graph_tried = true;
        if (!(e->flags & GABE_FLAG_NO_GRAPH)) {
            bool ok = true;
            for (int par = 0; par < 2 && ok; par++) {
                cudaGraph_t g = nullptr;
                if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { ok = false; break; }
                int rc = enqueue_step(e, par);
                cudaError_t r = cudaStreamEndCapture(e->stream, &g);
                if (rc || r != cudaSuccess || !g || cudaGraphInstantiate(&e->graph[par], g, 0) != cudaSuccess) ok = false;
                if (g) cudaGraphDestroy(g);
            }
            cudaGetLastError();
            e->err.clear();
            e->graph_ok = ok;
        }
    }
    for (int s = 0; s < nsteps; s++) {
        if (e->graph_ok) ECK(e, cudaGraphLaunch(e->graph[e->cur], e->stream));
        else {
            int rc = enqueue_step(e, e->cur);
            if (rc) return rc;
        }
        e->cur ^= 1;
    }
    if (nsteps) e->e0_stale = true;
    return GABE_OK;
}

int gabe_ensemble_sync(gabe_ensemble *e) {
    if (!e) return GABE_ERR_PARAM;
    ECK(e, cudaSetDevice(e->dev));
    ECK(e, cudaStreamSynchronize(e->stream));
    return GABE_OK;
}

int gabe_ensemble_scalars(gabe_ensemble *e, double *out) {
    if (!e || !out) return GABE_ERR_PARAM;
    if (!e->ready) return eset(e, GABE_ERR_STATE, "scalars before init/upload");
    ECK(e, cudaSetDevice(e->dev));
    int rc = refresh_e0(e);
    if (rc) return rc;
    std::vector<DevScalars> s(e->nlat);
    ECK(e, cudaMemcpyAsync(s.data(), e->d_sc, sizeof(DevScalars) * e->nlat, cudaMemcpyDeviceToHost, e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    bool bad = false;
    for (int l = 0; l < e->nlat; l++) {
        const double *src[6] = {s[l].a, s[l].adot, s[l].edkin, s[l].edpot, s[l].edgrad, s[l].edrho};
        for (int q = 0; q < 6; q++) {
            out[12 * l + 2 * q] = src[q][0];
            out[12 * l + 2 * q + 1] = src[q][1];
        }
        bad |= (s[l].status & ST_NONFINITE) != 0;
    }
    return bad ? eset(e, GABE_ERR_NONFINITE, "non-finite energy density in the ensemble") : GABE_OK;
}

int gabe_ensemble_native_bins(const gabe_ensemble *e) { return e ? e->nb_max : 0; }

int gabe_ensemble_log_spectra(gabe_ensemble *e, double *logspec, double *counts, double *native) {
    if (!e || !logspec || !counts) return GABE_ERR_PARAM;
    if (!e->ready) return eset(e, GABE_ERR_STATE, "spectra before init/upload");
    ECK(e, cudaSetDevice(e->dev));
    int rc = refresh_e0(e);  // Omega_gw uses rho of the current state
    if (rc) return rc;
    for (auto &G : e->groups) {
        const size_t n3 = (size_t)G.N * G.N * G.N, slot_r = (size_t)G.N * G.N * (G.N + 2);
        for (int f = 0; f < 2; f++)
            ECF(e, cufftExecR2C(G.plan_spec, (cufftReal *)(G.X[e->cur] + f * n3), (cufftComplex *)(G.S + f * slot_r)));
    }
    EnsBinArgs b{};
    b.lat = e->d_lat;
    b.nlat = e->nlat;
    b.nb_max = e->nb_max;
    b.nblk = kEnsBinBlocks;
    b.quirk = e->quirk;
    b.part = e->d_part;
    b.part_cnt = e->d_part_cnt;
    const size_t smem = (size_t)e->nb_max * (3 * 8 + 4);
    ens_bin_kernel<<<dim3(kEnsBinBlocks, e->nlat), 256, smem, e->stream>>>(b);
    ECK(e, cudaGetLastError());
    ens_rebin_kernel<<<e->nlat, 128, 0, e->stream>>>(b, e->nlog, (double)e->log_top, e->L, e->d_log, e->d_logcnt, e->d_native);
    ECK(e, cudaGetLastError());
    ECK(e, cudaMemcpyAsync(logspec, e->d_log, sizeof(double) * e->nlat * 3 * e->nlog, cudaMemcpyDeviceToHost, e->stream));
    ECK(e, cudaMemcpyAsync(counts, e->d_logcnt, sizeof(double) * e->nlat * e->nlog, cudaMemcpyDeviceToHost, e->stream));
    if (native)
        ECK(e, cudaMemcpyAsync(native, e->d_native, sizeof(double) * e->nlat * 4 * e->nb_max, cudaMemcpyDeviceToHost,
                               e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    return GABE_OK;
}

int gabe_ensemble_download(gabe_ensemble *e, int lat, double *field0, double *dfield0, double *h0, double *l0) {
    if (!e || lat < 0 || lat >= e->nlat) return GABE_ERR_PARAM;
    if (!e->ready) return eset(e, GABE_ERR_STATE, "download before init/upload");
    ECK(e, cudaSetDevice(e->dev));
    const EnsLat &Lt = e->h_lat[lat];
    const size_t n3 = (size_t)Lt.N * Lt.N * Lt.N, M = lattice_M(Lt.N);
    double *stage = reinterpret_cast<double *>(Lt.S);  // 10 N^2(N+2) floats >= N^3 or 12 M doubles
    double *dst[2] = {field0, dfield0};
    float *const *srcb[2] = {Lt.X, Lt.D};
    for (int a = 0; a < 2; a++) {
        if (!dst[a]) continue;
        for (int f = 0; f < 2; f++) {
            const double *mean = reinterpret_cast<const double *>(
                                     reinterpret_cast<const char *>(Lt.sc) +
                                     (a ? offsetof(DevScalars, dfbar) : offsetof(DevScalars, fbar))) + f;
            ECK(e, from_fluct(srcb[a][e->cur] + f * n3, n3, mean, stage, e->stream));
            ECK(e, cudaMemcpyAsync(dst[a] + f * n3, stage, n3 * 8, cudaMemcpyDeviceToHost, e->stream));
        }
    }
    // The source slots hold 5 N^2 (N+2) doubles: unpack h/l in chunks of
    // modes so that the 12 reference-layout components fit.
    const size_t chunk = (size_t)5 * Lt.N * Lt.N * (Lt.N + 2) / 12;
    double *gdst[2] = {h0, l0};
    for (int w = 0; w < 2; w++) {
        if (!gdst[w] || !Lt.G) continue;
        for (size_t m0 = 0; m0 < M; m0 += chunk) {
            const size_t cnt = (M - m0) < chunk ? (M - m0) : chunk;
            ECK(e, gw_unpack_f32(Lt.G, cnt, m0, Lt.N, M, w, stage, 0, e->stream));
            for (int q = 0; q < 12; q++)
                ECK(e, cudaMemcpyAsync(gdst[w] + (size_t)q * M + m0, stage + (size_t)q * cnt, cnt * 8,
                                       cudaMemcpyDeviceToHost, e->stream));
        }
    }
    ECK(e, cudaStreamSynchronize(e->stream));
    return GABE_OK;
}

const char *gabe_ensemble_last_error(const gabe_ensemble *e) { return e ? e->err.c_str() : g_ens_create_error.c_str(); }

size_t gabe_ensemble_device_bytes(const gabe_ensemble *e) { return e ? e->dev_bytes : 0; }

void *gabe_ensemble_stream(const gabe_ensemble *e) { return e ? (void *)e->stream : nullptr; }

int gabe_ensemble_launches_per_step(const gabe_ensemble *e) { return e ? (e->gws ? 3 : 2) : 0; }

int gabe_ensemble_graph_active(const gabe_ensemble *e) {
    if (!e) return GABE_ERR_PARAM * -1;
    return e->graph_tried ? (e->graph_ok ? 1 : 0) : -1;
}

}  // extern "C"
