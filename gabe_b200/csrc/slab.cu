// One slab of a lattice split along i over several processes (GPUs):
// field evolution, the tensor modes and the spectra (gabe_slab_*,
// include/gabe.h; the GW transpose is in slabgw.cuh).
//
// Each rank holds its own planes i in [plane0, plane0 + nplanes) of the
// four state arrays between two halo planes (the last own plane of the rank
// below and the first of the rank above, periodic in i), and runs the same
// two sweeps per step as a whole lattice (stencil.cuh / sweep32.cuh with
// StencilArgs::planes set).  The Friedmann update of the reference's step()
// (g2functions.cpp:234-271) needs full-volume energies, so sweep A (and the
// energies between steps) end with their block-summed totals in device
// memory; the caller adds the totals of all ranks (an all-reduce of kNV
// FP64 values) and runs the finish, which every rank then takes with the
// same totals.  After sweep B the caller exchanges the boundary planes:
// pack -> send/recv -> unpack.  The library does no communication itself.
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <cufft.h>

#include "../../include/gabe.h"
#include "launch.h"
#include "slabsplit.h"

using namespace gabe;

namespace {
thread_local std::string g_slab_create_error;
constexpr int kSlabBinBlocks = 296;  // blocks of the spectrum binning (2 per SM)
}

struct gabe_slab {
    gabe_params p{};
    LatticeConsts lc{};
    int N = 0, plane0 = 0, nloc = 0, planes = 0, dev = 0, cur = 0;
    bool f32 = false, uploaded = false;
    size_t plane_elems = 0, w = 8;
    cudaStream_t stream = nullptr;
    void *X[2] = {nullptr, nullptr}, *D[2] = {nullptr, nullptr};
    DevScalars *sc = nullptr;
    double *partials = nullptr, *sums = nullptr, *stage = nullptr;
    unsigned int *counters = nullptr;
    void *send[2] = {nullptr, nullptr}, *recv[2] = {nullptr, nullptr};  // [lo, hi]: 4 planes each
    int shape = 0, ci = 1;
    dim3 grid;
    // GW branch: the ranks' split, sources [10][nloc][N][N+2] (the all-to-all receive buffer
    // after the 2-D transforms), the send buffer (then T[10][N][m][nz]), amplitudes
    // [4][N][m][nz] of this rank's ky columns [plane0, plane0 + nloc)
    bool gws = false, spec = false;  // spec: the spectra transpose (FP64, or FP32 with N in {64, ..., 512})
    int W = 1, rank = 0, nbins = 0;
    cufftHandle plan_spec = 0;  // FP64: 2-D D2Z of the two fields' planes
    bool have_plan_spec = false;
    double *bin_part = nullptr, *bin_sum = nullptr;
    unsigned int *bin_cnt_part = nullptr;
    float *S = nullptr;
    void *Tb = nullptr, *G = nullptr, *fft_work = nullptr;
    size_t nz = 0, cplx_loc = 0;  // complex values of one component over this rank's planes or columns
    size_t csz = 8;               // bytes of one complex value (FP32 8, FP64 16)
    cufftHandle plan_i = 0;       // FP64: the pass along i (strided Z2Z, one component per call)
    bool have_plan_i = false;
    cufftHandle plan2d = 0;  // FP64: 2-D D2Z of the source planes (FP32 uses the library's passes)
    bool have_plan = false;
    std::string err;
};

namespace {

int serr(gabe_slab *s, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    else g_slab_create_error = buf;
    return code;
}

#define SCK(s, x)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) return serr(s, GABE_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

int salloc(gabe_slab *s, void **p, size_t bytes) {
    if (cudaMalloc(p, bytes ? bytes : 256) != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return serr(s, GABE_ERR_NOMEM, "cudaMalloc(%zu bytes) failed", bytes);
    }
    return GABE_OK;
}

// Device address of array a (0 phi, 1 chi, 2 phidot, 3 chidot) at buffer plane p of state c.
char *plane_ptr(gabe_slab *s, int c, int a, int p) {
    char *base = static_cast<char *>(a < 2 ? s->X[c] : s->D[c]);
    return base + ((size_t)(a & 1) * s->planes + p) * s->plane_elems * s->w;
}

double *dev_mean(gabe_slab *s, bool momentum, int f) {
    const size_t off = momentum ? offsetof(DevScalars, dfbar) : offsetof(DevScalars, fbar);
    return reinterpret_cast<double *>(reinterpret_cast<char *>(s->sc) + off) + f;
}

StencilArgs slab_args(gabe_slab *s, int counter, double *sums_out) {
    StencilArgs a{};
    a.X = s->X[s->cur];
    a.D = s->D[s->cur];
    a.Xo = s->X[s->cur ^ 1];
    a.Do = s->D[s->cur ^ 1];
    a.S = s->S;
    a.partials = s->partials;
    a.counter = s->counters + counter;
    a.sc = s->sc;
    a.c = s->lc;
    a.ci = s->ci;
    a.slot = 0;
    a.planes = s->planes;
    a.sums_out = sums_out;
    return a;
}

// Transform helpers by precision.  The planes [ncomp][nloc][N][N+2] of S ->
// their 2-D r2c in the send buffer Tb, blocks by destination rank (FP32: the
// library's pass along k in place and its pass along j written straight to
// the blocks; FP64: a cuFFT D2Z plan in place, then the pack).  The receive
// buffer S of a transpose -> T[ncomp][N][m][nz] transformed along i (FP32:
// one column pass that gathers its lines from the blocks of S; FP64:
// unpack, then a strided cuFFT Z2Z in place).
int planes_to_send(gabe_slab *s, cufftHandle plan, int ncomp) {
    if (s->f32) {
        SCK(s, fft_plane_scatter_f32(s->N, static_cast<float *>(s->S), s->Tb, ncomp * s->nloc, s->W, s->stream));
        return GABE_OK;
    }
    if (cufftExecD2Z(plan, (cufftDoubleReal *)s->S, (cufftDoubleComplex *)s->S) != CUFFT_SUCCESS)
        return serr(s, GABE_ERR_CUFFT, "2-D r2c of the slab's planes failed");
    SCK(s, slab_gw_pack_f64(s->S, s->Tb, s->N, s->nloc, s->W, ncomp, s->stream));
    return GABE_OK;
}

int receive_pass_i(gabe_slab *s, int ncomp) {
    const long long N = s->N, m = s->nloc, nz = (long long)s->nz;
    if (s->f32) {
        SCK(s, fft_col_gather_f32(s->N, s->S, s->Tb, ncomp, s->nloc, s->W, s->stream));
        return GABE_OK;
    }
    SCK(s, slab_gw_unpack_f64(s->S, s->Tb, s->N, s->nloc, s->W, ncomp, s->stream));
    for (int q = 0; q < ncomp; q++) {
        cufftDoubleComplex *X = static_cast<cufftDoubleComplex *>(s->Tb) + (size_t)q * N * m * nz;
        if (cufftExecZ2Z(s->plan_i, X, X, CUFFT_FORWARD) != CUFFT_SUCCESS)
            return serr(s, GABE_ERR_CUFFT, "pass along i failed");
    }
    return GABE_OK;
}

}  // namespace

extern "C" {

int gabe_slab_create(const gabe_params *p, const gabe_slab_params *sp, gabe_slab **out) {
    if (!out) return serr(nullptr, GABE_ERR_PARAM, "out is NULL");
    *out = nullptr;
    if (!p || p->struct_size != (int32_t)sizeof(gabe_params)) return serr(nullptr, GABE_ERR_PARAM, "bad gabe_params");
    if (!sp || sp->struct_size != (int32_t)sizeof(gabe_slab_params))
        return serr(nullptr, GABE_ERR_PARAM, "bad gabe_slab_params");
    const int N = p->N;
    if (N < 16 || N > 1024 || N % 16 || p->nflds != 2)
        return serr(nullptr, GABE_ERR_PARAM, "N must be a multiple of 16 in [16, 1024] and nflds 2");
    if (p->gws_on && p->precision == GABE_FP32 && N != 64 && N != 128 && N != 256 && N != 512)
        return serr(nullptr, GABE_ERR_PARAM, "FP32 slabs with GWs need N in {64, 128, 256, 512}");
    if (p->gws_on && p->expansion != 1)  // tensor modes evolve with expansion_type 1 only (g2functions.cpp:272-302)
        return serr(nullptr, GABE_ERR_PARAM, "slabs with GWs need expansion_type 1");
    if (p->precision != GABE_FP64 && p->precision != GABE_FP32) return serr(nullptr, GABE_ERR_PARAM, "bad precision");
    if (p->model != GABE_MODEL_QUADRATIC && p->model != GABE_MODEL_LPHI4) return serr(nullptr, GABE_ERR_PARAM, "bad model");
    if (p->expansion < 0 || p->expansion > 2) return serr(nullptr, GABE_ERR_PARAM, "expansion must be 0, 1 or 2");
    if (!(p->L > 0) || !(p->dt > 0)) return serr(nullptr, GABE_ERR_PARAM, "L and dt must be positive");
    if (sp->nplanes < 1 || sp->plane0 < 0 || sp->plane0 + sp->nplanes > N)
        return serr(nullptr, GABE_ERR_PARAM, "planes [%d, %d) outside [0, %d)", sp->plane0, sp->plane0 + sp->nplanes, N);
    int rank = 0;
    const bool split_needed = p->gws_on || sp->nranks >= 1;
    if (split_needed) {  // the transposes need every rank's planes: the standard split of nranks
        if (sp->nranks < 1 || sp->nranks > N) return serr(nullptr, GABE_ERR_PARAM, "nranks must be in [1, N]");
        const Split spl(N, sp->nranks);
        rank = spl.owner(sp->plane0);
        if (spl.p0(rank) != sp->plane0 || spl.n(rank) != sp->nplanes)
            return serr(nullptr, GABE_ERR_PARAM, "the planes must be rank %d's share of %d ranks", rank,
                        sp->nranks);
    }
    gabe_slab *s = new (std::nothrow) gabe_slab();
    if (!s) return serr(nullptr, GABE_ERR_NOMEM, "host allocation failed");
    auto bail = [&](int code) {
        g_slab_create_error = s->err;
        gabe_slab_destroy(s);
        return code;
    };
    s->p = *p;
    s->N = N;
    s->plane0 = sp->plane0;
    s->nloc = sp->nplanes;
    s->planes = sp->nplanes + 2;
    s->f32 = p->precision == GABE_FP32;
    s->w = s->f32 ? 4 : 8;
    s->plane_elems = (size_t)N * N;
    s->lc = make_lattice_consts(*p);
    s->gws = p->gws_on != 0;
    s->spec = (!s->f32 || N == 64 || N == 128 || N == 256 || N == 512) && sp->nranks >= 1 && sp->nranks <= N;
    s->W = (p->gws_on || s->spec) ? (sp->nranks >= 1 ? sp->nranks : 1) : 1;
    s->nbins = gabe_spectra_numbins(N);
    s->rank = rank;
    s->nz = (size_t)N / 2 + 1;
    s->cplx_loc = (size_t)s->nloc * N * s->nz;
    s->csz = s->f32 ? 8 : 16;
    if (p->device >= 0 && cudaSetDevice(p->device) != cudaSuccess) {
        cudaGetLastError();
        serr(s, GABE_ERR_CUDA, "cudaSetDevice(%d) failed", p->device);
        return bail(GABE_ERR_CUDA);
    }
    if (cudaGetDevice(&s->dev) != cudaSuccess || cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        serr(s, GABE_ERR_CUDA, "no CUDA device");
        return bail(GABE_ERR_CUDA);
    }
    // the whole lattice's tile and plane chunk, with the chunks cut from this slab's planes
    GridPlan g = s->f32 ? plan_grid32(N, p->tile_shape, p->tile_ci) : plan_grid(N, p->tile_shape, p->tile_ci);
    if (g.shape < 0) {
        serr(s, GABE_ERR_PARAM, "N = %d: no stencil tile divides N", N);
        return bail(GABE_ERR_PARAM);
    }
    s->shape = g.shape;
    s->ci = g.ci < s->nloc ? g.ci : s->nloc;
    s->grid = dim3(g.grid.x, g.grid.y, (s->nloc + s->ci - 1) / s->ci);
    const size_t arr = 2 * (size_t)s->planes * s->plane_elems * s->w;  // both fields of one array kind
    const size_t nblk = (size_t)s->grid.x * s->grid.y * s->grid.z;
    int rc;
    for (int b = 0; b < 2; b++) {
        if ((rc = salloc(s, &s->X[b], arr)) || (rc = salloc(s, &s->D[b], arr))) return bail(rc);
        if ((rc = salloc(s, &s->send[b], 4 * s->plane_elems * s->w)) || (rc = salloc(s, &s->recv[b], 4 * s->plane_elems * s->w)))
            return bail(rc);
    }
    if ((rc = salloc(s, (void **)&s->sc, sizeof(DevScalars))) ||
        (rc = salloc(s, (void **)&s->partials, kNV * sizeof(double) * (nblk > 4096 ? nblk : 4096))) ||
        (rc = salloc(s, (void **)&s->sums, kNV * sizeof(double))) ||
        (rc = salloc(s, (void **)&s->counters, 4 * sizeof(unsigned int))))
        return bail(rc);
    if (s->f32 && (rc = salloc(s, (void **)&s->stage, (size_t)s->nloc * s->plane_elems * sizeof(double)))) return bail(rc);
    const cufftType r2c = s->f32 ? CUFFT_R2C : CUFFT_D2Z;
    if (s->spec && !s->gws) {  // buffers of the two fields' transpose
        if ((rc = salloc(s, (void **)&s->S, 2 * s->cplx_loc * s->csz)) || (rc = salloc(s, &s->Tb, 2 * s->cplx_loc * s->csz)))
            return bail(rc);
    }
    if ((s->spec || s->gws) && !s->f32) {  // FP64 pass along i: N values of stride m nz, m nz of them
        long long ni[1] = {N}, em[1] = {N};
        const long long m = s->nloc, nzl = (long long)s->nz;
        if (cufftCreate(&s->plan_i) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "cufftCreate failed");
            return bail(GABE_ERR_CUFFT);
        }
        s->have_plan_i = true;
        size_t wsi = 0;
        if (cufftMakePlanMany64(s->plan_i, 1, ni, em, m * nzl, 1, em, m * nzl, 1, CUFFT_Z2Z, m * nzl, &wsi) != CUFFT_SUCCESS ||
            cufftSetStream(s->plan_i, s->stream) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "plan of the pass along i failed");
            return bail(GABE_ERR_CUFFT);
        }
    }
    if (s->spec && !s->f32) {
        long long n2[2] = {N, N}, inem[2] = {N, N + 2}, onem[2] = {N, (long long)s->nz};
        size_t ws = 0;
        if (cufftCreate(&s->plan_spec) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "cufftCreate failed");
            return bail(GABE_ERR_CUFFT);
        }
        s->have_plan_spec = true;
        if (cufftMakePlanMany64(s->plan_spec, 2, n2, inem, 1, (long long)N * (N + 2), onem, 1, (long long)N * s->nz,
                                r2c, 2LL * s->nloc, &ws) != CUFFT_SUCCESS ||
            cufftSetStream(s->plan_spec, s->stream) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "2-D r2c plan of the slab's field planes failed");
            return bail(GABE_ERR_CUFFT);
        }
    }
    if (s->spec) {
        const int ns = 3, nb = s->nbins;
        if ((rc = salloc(s, (void **)&s->bin_part, (size_t)kSlabBinBlocks * ns * nb * sizeof(double))) ||
            (rc = salloc(s, (void **)&s->bin_cnt_part, (size_t)kSlabBinBlocks * nb * sizeof(unsigned int))) ||
            (rc = salloc(s, (void **)&s->bin_sum, (size_t)(ns + 1) * nb * sizeof(double))))
            return bail(rc);
    }
    if (s->gws) {
        if ((rc = salloc(s, (void **)&s->S, 10 * s->cplx_loc * s->csz)) ||
            (rc = salloc(s, &s->Tb, 10 * s->cplx_loc * s->csz)) || (rc = salloc(s, &s->G, 4 * s->cplx_loc * s->csz)))
            return bail(rc);
    }
    if (s->gws && !s->f32) {
        long long n2[2] = {N, N}, inem[2] = {N, N + 2}, onem[2] = {N, (long long)s->nz};
        size_t ws = 0;
        if (cufftCreate(&s->plan2d) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "cufftCreate failed");
            return bail(GABE_ERR_CUFFT);
        }
        s->have_plan = true;
        if (cufftSetAutoAllocation(s->plan2d, 0) != CUFFT_SUCCESS ||
            cufftMakePlanMany64(s->plan2d, 2, n2, inem, 1, (long long)N * (N + 2), onem, 1, (long long)N * s->nz,
                                r2c, 10LL * s->nloc, &ws) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "2-D r2c plan of the slab's source planes failed");
            return bail(GABE_ERR_CUFFT);
        }
        if ((rc = salloc(s, &s->fft_work, ws))) return bail(rc);
        if (cufftSetWorkArea(s->plan2d, s->fft_work) != CUFFT_SUCCESS || cufftSetStream(s->plan2d, s->stream) != CUFFT_SUCCESS) {
            serr(s, GABE_ERR_CUFFT, "cuFFT work area / stream");
            return bail(GABE_ERR_CUFFT);
        }
    }
    if (cudaMemset(s->counters, 0, 4 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMemset(s->sc, 0, sizeof(DevScalars)) != cudaSuccess) {
        cudaGetLastError();
        serr(s, GABE_ERR_CUDA, "device initialisation failed");
        return bail(GABE_ERR_CUDA);
    }
    *out = s;
    return GABE_OK;
}

int gabe_slab_destroy(gabe_slab *s) {
    if (!s) return GABE_OK;
    cudaSetDevice(s->dev);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->have_plan) cufftDestroy(s->plan2d);
    if (s->have_plan_spec) cufftDestroy(s->plan_spec);
    if (s->have_plan_i) cufftDestroy(s->plan_i);
    void *bufs[] = {s->X[0], s->X[1], s->D[0], s->D[1], s->send[0], s->send[1], s->recv[0], s->recv[1],
                    s->sc, s->partials, s->sums, s->stage, s->counters, s->S, s->Tb, s->G, s->fft_work,
                    s->bin_part, s->bin_cnt_part, s->bin_sum};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (s->stream) cudaStreamDestroy(s->stream);
    cudaGetLastError();
    delete s;
    return GABE_OK;
}

const char *gabe_slab_last_error(gabe_slab *s) { return s ? s->err.c_str() : g_slab_create_error.c_str(); }

int gabe_slab_upload(gabe_slab *s, const double *field0, const double *dfield0, const double mean[4], double a0,
                     double adot0) {
    if (!s) return GABE_ERR_PARAM;
    if (!field0 || !dfield0) return serr(s, GABE_ERR_PARAM, "field0/dfield0 must not be NULL");
    if (s->f32 && !mean) return serr(s, GABE_ERR_PARAM, "FP32 storage needs the whole lattice's means");
    if (!(a0 > 0) || !std::isfinite(a0) || !std::isfinite(adot0)) return serr(s, GABE_ERR_PARAM, "bad a0/adot0");
    SCK(s, cudaSetDevice(s->dev));
    s->uploaded = false;  // until the whole slab is in place
    DevScalars d{};
    d.a[0] = a0;
    d.adot[0] = adot0;
    if (s->p.expansion == 0) {
        d.a[1] = a0;
        d.adot[1] = adot0;
    }
    d.adot_given = 1;
    if (s->f32)
        for (int f = 0; f < 2; f++) {
            d.fbar[f] = mean[f];
            d.dfbar[f] = mean[2 + f];
        }
    SCK(s, cudaMemcpyAsync(s->sc, &d, sizeof(d), cudaMemcpyHostToDevice, s->stream));
    const size_t nf = (size_t)s->nloc * s->plane_elems;  // own values of one field
    const double *src[2] = {field0, dfield0};
    for (int a = 0; a < 4; a++) {
        const double *h = src[a >> 1] + (size_t)(a & 1) * nf;
        char *dst = plane_ptr(s, 0, a, 1);
        if (!s->f32) {
            SCK(s, cudaMemcpyAsync(dst, h, nf * 8, cudaMemcpyHostToDevice, s->stream));
        } else {
            SCK(s, cudaMemcpyAsync(s->stage, h, nf * 8, cudaMemcpyHostToDevice, s->stream));
            SCK(s, to_fluct(s->stage, nf, dev_mean(s, a >= 2, a & 1), reinterpret_cast<float *>(dst), s->stream));
        }
    }
    if (s->gws) SCK(s, cudaMemsetAsync(s->G, 0, 4 * s->cplx_loc * s->csz, s->stream));  // h, l start at zero
    SCK(s, cudaStreamSynchronize(s->stream));
    s->cur = 0;
    s->uploaded = true;
    return GABE_OK;
}

int gabe_slab_download(gabe_slab *s, double *field0, double *dfield0) {
    if (!s) return GABE_ERR_PARAM;
    if (!s->uploaded) return serr(s, GABE_ERR_STATE, "download before upload");
    SCK(s, cudaSetDevice(s->dev));
    const size_t nf = (size_t)s->nloc * s->plane_elems;
    double *dst[2] = {field0, dfield0};
    for (int a = 0; a < 4; a++) {
        double *h = dst[a >> 1];
        if (!h) continue;
        h += (size_t)(a & 1) * nf;
        const char *src = plane_ptr(s, s->cur, a, 1);
        if (!s->f32) {
            SCK(s, cudaMemcpyAsync(h, src, nf * 8, cudaMemcpyDeviceToHost, s->stream));
        } else {
            SCK(s, from_fluct(reinterpret_cast<const float *>(src), nf, dev_mean(s, a >= 2, a & 1), s->stage, s->stream));
            SCK(s, cudaMemcpyAsync(h, s->stage, nf * 8, cudaMemcpyDeviceToHost, s->stream));
        }
    }
    SCK(s, cudaStreamSynchronize(s->stream));
    return GABE_OK;
}

int gabe_slab_buffers(gabe_slab *s, double **sums, void **send_lo, void **send_hi, void **recv_lo, void **recv_hi,
                      size_t *halo_bytes) {
    if (!s) return GABE_ERR_PARAM;
    if (sums) *sums = s->sums;
    if (send_lo) *send_lo = s->send[0];
    if (send_hi) *send_hi = s->send[1];
    if (recv_lo) *recv_lo = s->recv[0];
    if (recv_hi) *recv_hi = s->recv[1];
    if (halo_bytes) *halo_bytes = 4 * s->plane_elems * s->w;
    return GABE_OK;
}

int gabe_slab_pack(gabe_slab *s) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "pack before upload") : GABE_ERR_PARAM;
    SCK(s, cudaSetDevice(s->dev));
    const size_t pb = s->plane_elems * s->w;
    for (int a = 0; a < 4; a++) {
        SCK(s, cudaMemcpyAsync(static_cast<char *>(s->send[0]) + a * pb, plane_ptr(s, s->cur, a, 1), pb,
                               cudaMemcpyDeviceToDevice, s->stream));
        SCK(s, cudaMemcpyAsync(static_cast<char *>(s->send[1]) + a * pb, plane_ptr(s, s->cur, a, s->nloc), pb,
                               cudaMemcpyDeviceToDevice, s->stream));
    }
    return GABE_OK;
}

int gabe_slab_unpack(gabe_slab *s) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "unpack before upload") : GABE_ERR_PARAM;
    SCK(s, cudaSetDevice(s->dev));
    const size_t pb = s->plane_elems * s->w;
    for (int a = 0; a < 4; a++) {
        SCK(s, cudaMemcpyAsync(plane_ptr(s, s->cur, a, 0), static_cast<char *>(s->recv[0]) + a * pb, pb,
                               cudaMemcpyDeviceToDevice, s->stream));
        SCK(s, cudaMemcpyAsync(plane_ptr(s, s->cur, a, s->nloc + 1), static_cast<char *>(s->recv[1]) + a * pb, pb,
                               cudaMemcpyDeviceToDevice, s->stream));
    }
    return GABE_OK;
}

int gabe_slab_sweep(gabe_slab *s, int which) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "sweep before upload") : GABE_ERR_PARAM;
    if (which < 0 || which > 2) return serr(s, GABE_ERR_PARAM, "which must be 0 (sweep A), 1 (sweep B) or 2 (energies)");
    SCK(s, cudaSetDevice(s->dev));
    const int mode = which == 0 ? (s->gws ? MODE_A_GW : MODE_A) : (which == 1 ? MODE_B : MODE_E0);
    StencilArgs a = slab_args(s, which, which == 1 ? nullptr : s->sums);
    SCK(s, s->f32 ? sweep32_f32(s->shape, mode, a, s->grid, s->stream) : sweep_f64(s->shape, mode, a, s->grid, s->stream));
    if (which == 1) s->cur ^= 1;
    return GABE_OK;
}

int gabe_slab_finish(gabe_slab *s, int which) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "finish before upload") : GABE_ERR_PARAM;
    if (which != 0 && which != 2) return serr(s, GABE_ERR_PARAM, "which must be 0 (after sweep A) or 2 (energies)");
    SCK(s, cudaSetDevice(s->dev));
    const int mode = which == 0 ? (s->gws ? MODE_A_GW : MODE_A) : MODE_E0;
    SCK(s, s->f32 ? slab_finish_f32(mode, s->lc, s->sc, s->sums, s->stream)
                  : slab_finish_f64(mode, s->lc, s->sc, s->sums, s->stream));
    return GABE_OK;
}

int gabe_slab_gw_buffers(gabe_slab *s, void **send, void **recv, int64_t *send_bytes, int64_t *recv_bytes) {
    if (!s) return GABE_ERR_PARAM;
    if (!s->gws) return serr(s, GABE_ERR_STATE, "slab without GWs");
    if (send) *send = s->Tb;
    if (recv) *recv = s->S;
    const Split spl(s->N, s->W);
    for (int r = 0; r < s->W; r++) {
        if (send_bytes) send_bytes[r] = (int64_t)10 * s->nloc * spl.n(r) * s->nz * s->csz;
        if (recv_bytes) recv_bytes[r] = (int64_t)10 * spl.n(r) * s->nloc * s->nz * s->csz;
    }
    return GABE_OK;
}

int gabe_slab_gw_transform(gabe_slab *s) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "transform before upload") : GABE_ERR_PARAM;
    if (!s->gws) return serr(s, GABE_ERR_STATE, "slab without GWs");
    SCK(s, cudaSetDevice(s->dev));
    return planes_to_send(s, s->plan2d, 10);
}

int gabe_slab_gw_update(gabe_slab *s) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "update before upload") : GABE_ERR_PARAM;
    if (!s->gws) return serr(s, GABE_ERR_STATE, "slab without GWs");
    SCK(s, cudaSetDevice(s->dev));
    // pass along i: for every component and column (y, kz), the N values of stride m nz
    int rc = receive_pass_i(s, 10);
    if (rc) return rc;
    SCK(s, s->f32 ? slab_kspace_f32(s->Tb, s->G, s->sc, s->lc, s->nloc, s->plane0, s->stream)
                  : slab_kspace_f64(s->Tb, s->G, s->sc, s->lc, s->nloc, s->plane0, s->stream));
    return GABE_OK;
}

int gabe_slab_gw_download(gabe_slab *s, double *h0, double *l0) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "download before upload") : GABE_ERR_PARAM;
    if (!s->gws) return serr(s, GABE_ERR_STATE, "slab without GWs");
    SCK(s, cudaSetDevice(s->dev));
    const size_t M = s->cplx_loc;  // this rank's k-points: N kx x nloc ky x (N/2+1) kz
    const size_t chunk = 10 * s->cplx_loc * s->csz / (12 * sizeof(double));  // points staged in the send buffer
    double *stage = static_cast<double *>(s->Tb);
    double *dst[2] = {h0, l0};
    for (int w = 0; w < 2; w++) {
        if (!dst[w]) continue;
        for (size_t m0 = 0; m0 < M; m0 += chunk) {
            const size_t cnt = M - m0 < chunk ? M - m0 : chunk;
            SCK(s, s->f32 ? slab_gw_amplitudes_f32(s->G, cnt, m0, s->N, s->nloc, s->plane0, w, stage, s->stream)
                          : slab_gw_amplitudes_f64(s->G, cnt, m0, s->N, s->nloc, s->plane0, w, stage, s->stream));
            SCK(s, cudaMemcpy2DAsync(dst[w] + m0, M * sizeof(double), stage, cnt * sizeof(double), cnt * sizeof(double),
                                     12, cudaMemcpyDeviceToHost, s->stream));
        }
    }
    SCK(s, cudaStreamSynchronize(s->stream));
    return GABE_OK;
}

int gabe_slab_spectra_transform(gabe_slab *s) {
    if (!s || !s->uploaded) return s ? serr(s, GABE_ERR_STATE, "spectra before upload") : GABE_ERR_PARAM;
    if (!s->spec) return serr(s, GABE_ERR_STATE, "slab spectra need nranks (and, with FP32 storage, N in {64, ..., 512})");
    SCK(s, cudaSetDevice(s->dev));
    const size_t N = s->N, w = s->w;
    // own planes of both fields (FP32: fluctuations) into padded rows, then 2-D r2c into the send blocks
    char *S = reinterpret_cast<char *>(s->S);
    for (int f = 0; f < 2; f++)
        SCK(s, cudaMemcpy2DAsync(S + (size_t)f * s->nloc * N * (N + 2) * w, (N + 2) * w, plane_ptr(s, s->cur, f, 1), N * w,
                                 N * w, (size_t)s->nloc * N, cudaMemcpyDeviceToDevice, s->stream));
    return planes_to_send(s, s->plan_spec, 2);
}

int gabe_slab_spectra_buffers(gabe_slab *s, void **send, void **recv, int64_t *send_bytes, int64_t *recv_bytes) {
    if (!s) return GABE_ERR_PARAM;
    if (!s->spec) return serr(s, GABE_ERR_STATE, "slab without spectra");
    if (send) *send = s->Tb;
    if (recv) *recv = s->S;
    const Split spl(s->N, s->W);
    for (int r = 0; r < s->W; r++) {
        if (send_bytes) send_bytes[r] = (int64_t)2 * s->nloc * spl.n(r) * s->nz * s->csz;
        if (recv_bytes) recv_bytes[r] = (int64_t)2 * spl.n(r) * s->nloc * s->nz * s->csz;
    }
    return GABE_OK;
}

int gabe_slab_spectra_raw(gabe_slab *s, double *sums, double *counts) {
    if (!s || !s->uploaded || !sums || !counts) return s ? serr(s, GABE_ERR_PARAM, "bad arguments") : GABE_ERR_PARAM;
    if (!s->spec) return serr(s, GABE_ERR_STATE, "slab without spectra");
    SCK(s, cudaSetDevice(s->dev));
    int rc = receive_pass_i(s, 2);
    if (rc) return rc;
    SCK(s, cudaStreamSynchronize(s->stream));
    DevScalars d;
    SCK(s, cudaMemcpy(&d, s->sc, sizeof(d), cudaMemcpyDeviceToHost));
    const int ns = 2 + (s->gws ? 1 : 0), nb = s->nbins;
    BinArgs b{};
    b.F = s->Tb;
    b.G = s->gws ? s->G : nullptr;
    b.part_sum = s->bin_part;
    b.part_cnt = s->bin_cnt_part;
    b.N = s->N;
    b.nbins = nb;
    b.nseries = ns;
    b.quirk = s->p.gw_spec_quirk;
    b.fix_zero = s->f32 ? 1 : 0;  // FP32 holds fluctuations: the k = 0 term gets N^3 fbar
    b.zero_re[0] = s->lc.gridsize * d.fbar[0];
    b.zero_re[1] = s->lc.gridsize * d.fbar[1];
    b.m = s->nloc;
    b.y0 = s->plane0;
    Launch lb{dim3(kSlabBinBlocks), dim3(256), (size_t)nb * (ns * 8 + 4), s->stream};
    SCK(s, s->f32 ? bins_f32(b, lb) : bins_f64(b, lb));
    SCK(s, bin_reduce(s->bin_part, s->bin_cnt_part, kSlabBinBlocks, ns, nb, s->bin_sum, s->bin_sum + ns * nb, s->stream));
    SCK(s, cudaMemcpyAsync(sums, s->bin_sum, (size_t)ns * nb * 8, cudaMemcpyDeviceToHost, s->stream));
    SCK(s, cudaMemcpyAsync(counts, s->bin_sum + ns * nb, (size_t)nb * 8, cudaMemcpyDeviceToHost, s->stream));
    SCK(s, cudaStreamSynchronize(s->stream));
    return GABE_OK;
}

int gabe_slab_stream(gabe_slab *s, void **stream) {
    if (!s || !stream) return GABE_ERR_PARAM;
    *stream = s->stream;
    return GABE_OK;
}

int gabe_slab_sync(gabe_slab *s) {
    if (!s) return GABE_ERR_PARAM;
    SCK(s, cudaSetDevice(s->dev));
    SCK(s, cudaStreamSynchronize(s->stream));
    return GABE_OK;
}

int gabe_slab_scalars(gabe_slab *s, double out12[12]) {
    if (!s || !out12) return GABE_ERR_PARAM;
    SCK(s, cudaSetDevice(s->dev));
    SCK(s, cudaStreamSynchronize(s->stream));
    DevScalars d;
    SCK(s, cudaMemcpy(&d, s->sc, sizeof(d), cudaMemcpyDeviceToHost));
    const double *src[6] = {d.a, d.adot, d.edkin, d.edpot, d.edgrad, d.edrho};
    for (int q = 0; q < 6; q++) {
        out12[2 * q] = src[q][0];
        out12[2 * q + 1] = src[q][1];
    }
    if (d.status & ST_NONFINITE) return serr(s, GABE_ERR_NONFINITE, "non-finite energy density at step %lld", d.step);
    return GABE_OK;
}

}  // extern "C"
