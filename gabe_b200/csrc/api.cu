// C ABI of the B200 lattice-evolution library (include/gabe.h).
//
// One handle = one lattice on one GPU with one stream.  Device buffers are
// allocated once in gabe_create; a step is captured once into a CUDA graph
// per ping-pong parity and replayed by gabe_step.  cuFFT plans use a work
// area this file allocates, so nothing is allocated after creation.
#include <cufft.h>

#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/gabe.h"
#include "../../include/gabe_dump.h"
#include "launch.h"

using namespace gabe;

namespace {

thread_local std::string g_create_error;

constexpr int kBinBlocks = 296;  // 2 x 148 SMs

}  // namespace

struct gabe_handle {
    gabe_params p{};
    int dev = 0;
    bool f32 = false;
    int N = 0, nz = 0;
    size_t n3 = 0, M = 0, esz = 8;
    cudaStream_t stream = nullptr;
    void *X[2] = {nullptr, nullptr}, *D[2] = {nullptr, nullptr};
    void *G = nullptr;  // GW amplitudes h+, hx, l+, lx [4][M] complex
    double *gwnorm = nullptr;  // upload check: |h|^2, |h - TT(h)|^2, |l|^2, |l - TT(l)|^2
    void *S = nullptr;  // sources / spectra scratch / staging
    void *S2 = nullptr; // second source buffer: lets the GW chain of step n overlap sweep A of step n+1
    size_t S_bytes = 0;
    cudaStream_t gw_stream = nullptr;
    int prio_low = 0;  // priority of gw_stream (the handle's stream has the highest)
    cudaEvent_t ev_a = nullptr, ev_k[2] = {nullptr, nullptr};
    int nslots = 0;
    double *partials = nullptr;
    size_t npartials = 0;
    unsigned int *counters = nullptr;
    DevScalars *sc = nullptr;
    double *bin_part = nullptr, *bin_sum = nullptr;
    double *outres = nullptr;  // meansvars results [8]
    unsigned int *bin_cnt_part = nullptr;
    int nbins = 0;
    cufftHandle plan_src = 0, plan_spec = 0;
    bool have_plan_src = false, have_plan_spec = false;
    bool evolve_gw = false; // calc_gws with expansion_type 1: the step evolves h, l (types 0 and 2 do not)
    bool own_fft = false;   // the library's three-pass 3-D r2c (fft3d.cuh)
    bool fftt = false;      // the transposed three-pass transform with the pass along i fused into the
                            // k-space update (fftt.cuh); G is then kept as [4][kz][ky][kx]
    void *fft_work = nullptr;
    size_t fft_work_bytes = 0;
    LatticeConsts lc{};
    int shape = 0;
    int ci = 0;
    dim3 grid;
    int cur = 0;
    bool uploaded = false;
    bool e0_stale = false;  // stage-0 energies/adot of the current state not yet reduced
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // one step, by starting parity
    cudaGraphExec_t graph2[2] = {nullptr, nullptr};  // two steps, by starting parity
    bool graph_tried = false, graph_ok = false;
    size_t dev_bytes = 0;
    std::string err;
};

namespace {

int set_err(gabe_handle *h, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    else g_create_error = buf;
    return code;
}

#define CK(h, x)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess) return set_err(h, GABE_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)
#define CF(h, x)                                                                                   \
    do {                                                                                           \
        cufftResult r_ = (x);                                                                      \
        if (r_ != CUFFT_SUCCESS) return set_err(h, GABE_ERR_CUFFT, "%s: cufft error %d", #x, (int)r_); \
    } while (0)

int dalloc(gabe_handle *h, void **ptr, size_t bytes) {
    if (bytes == 0) bytes = 256;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        cudaGetLastError();
        return set_err(h, GABE_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    h->dev_bytes += bytes;
    return GABE_OK;
}

void choose_tile(gabe_handle *h) {
    GridPlan g = h->f32 ? plan_grid32(h->N, h->p.tile_shape, h->p.tile_ci)
                        : plan_grid(h->N, h->p.tile_shape, h->p.tile_ci);
    h->shape = g.shape;
    h->ci = g.ci;
    h->grid = g.grid;
}

int make_plans(gabe_handle *h) {
    const long long N = h->N, nz = h->nz;
    long long n[3] = {N, N, N};
    size_t ws_src = 0, ws_spec = 0;
    const cufftType t = h->f32 ? CUFFT_R2C : CUFFT_D2Z;
    // the library's in-layout three-pass r2c: on request
    h->own_fft = h->evolve_gw && h->f32 && !h->fftt && fft3d_supported(h->N) && (h->p.flags & GABE_FLAG_OWN_FFT);
    if (h->own_fft || h->fftt) {
        // no plan: fft3d.cuh / fftt.cuh
    } else if (h->evolve_gw) {
        long long inem[3] = {N, N, 2 * nz}, onem[3] = {N, N, nz};
        CF(h, cufftCreate(&h->plan_src));
        h->have_plan_src = true;
        CF(h, cufftSetAutoAllocation(h->plan_src, 0));
        CF(h, cufftMakePlanMany64(h->plan_src, 3, n, inem, 1, N * N * 2 * nz, onem, 1, N * N * nz, t, 2 * kSrc,
                                  &ws_src));
    }
    {
        long long inem[3] = {N, N, N}, onem[3] = {N, N, nz};
        CF(h, cufftCreate(&h->plan_spec));
        h->have_plan_spec = true;
        CF(h, cufftSetAutoAllocation(h->plan_spec, 0));
        CF(h, cufftMakePlanMany64(h->plan_spec, 3, n, inem, 1, N * N * N, onem, 1, N * N * nz, t, 2, &ws_spec));
    }
    h->fft_work_bytes = ws_src > ws_spec ? ws_src : ws_spec;
    int rc = dalloc(h, &h->fft_work, h->fft_work_bytes);
    if (rc) return rc;
    if (h->have_plan_src) {
        CF(h, cufftSetWorkArea(h->plan_src, h->fft_work));
        CF(h, cufftSetStream(h->plan_src, h->stream));
    }
    CF(h, cufftSetWorkArea(h->plan_spec, h->fft_work));
    CF(h, cufftSetStream(h->plan_spec, h->stream));
    return GABE_OK;
}

int fft_r2c(gabe_handle *h, cufftHandle plan, void *in, void *out) {
    if (h->f32) CF(h, cufftExecR2C(plan, (cufftReal *)in, (cufftComplex *)out));
    else CF(h, cufftExecD2Z(plan, (cufftDoubleReal *)in, (cufftDoubleComplex *)out));
    return GABE_OK;
}

// The GW chain of step n overlaps the field sweeps of step n+1 (two source
// buffers) -- except with the library's FFT, which runs in line (measured
// faster at 512^3) and uses the second buffer as its column passes' target.
bool overlapped(const gabe_handle *h) { return h->evolve_gw && h->S2 != nullptr && !h->own_fft && !h->fftt; }
float *fft_scratch(const gabe_handle *h) { return h->own_fft ? static_cast<float *>(h->S2) : nullptr; }
void *source_buffer(const gabe_handle *h, int slot) { return slot && h->S2 ? h->S2 : h->S; }

// Transforms of the 2*kSrc source arrays in source buffer `slot`
// (fft_stresstensor's transforms, g2evolutionpert.cpp:190-195): the full 3-D
// r2c, or -- for the transposed form, whose k-space update does the pass
// along i -- its passes along k and j.
int source_fft(gabe_handle *h, int slot, cudaStream_t s) {
    void *S = source_buffer(h, slot);
    if (h->fftt) {  // rows S -> S2, pass along j S2 -> S; the pass along i runs inside the k-space update
        CK(h, fftt_rows_f32(h->N, static_cast<const float *>(S), h->S2, 2 * kSrc, &h->sc->status, s));
        CK(h, fftt_cols_f32(h->N, h->S2, S, 2 * kSrc, &h->sc->status, s));
        return GABE_OK;
    }
    if (h->own_fft) {
        CK(h, fft3d_r2c_f32(h->N, static_cast<float *>(S), fft_scratch(h), 2 * kSrc, s));
        return GABE_OK;
    }
    CF(h, cufftSetStream(h->plan_src, s));
    return fft_r2c(h, h->plan_src, S, S);
}

// TT projection and both RK2 stages of h, l (kspace.cuh, or fftt.cuh with the pass along i).
int kspace(gabe_handle *h, int slot, cudaStream_t s) {
    KspaceArgs k{};
    k.S = source_buffer(h, slot);
    k.G = h->G;
    k.sc = h->sc;
    k.c = h->lc;
    k.slot = slot;
    if (h->fftt) {
        CK(h, fftt_ikspace_f32(h->N, k.S, h->G, h->sc, h->lc, slot, &h->sc->status, s));
        return GABE_OK;
    }
    Launch lk{dim3(148 * 8), dim3(256), 0, s};
    CK(h, h->f32 ? kspace_f32(k, lk) : kspace_f64(k, lk));
    return GABE_OK;
}

StencilArgs stencil_args(gabe_handle *h, int cur, int slot = 0) {
    StencilArgs a{};
    a.X = h->X[cur];
    a.D = h->D[cur];
    a.Xo = h->X[1 - cur];
    a.Do = h->D[1 - cur];
    a.S = source_buffer(h, slot);
    a.slot = slot;
    a.partials = h->partials;
    a.sc = h->sc;
    a.c = h->lc;
    a.ci = h->ci;
    return a;
}

int sweep(gabe_handle *h, int mode, int cur, int counter, int slot = 0) {
    StencilArgs a = stencil_args(h, cur, slot);
    a.counter = h->counters + counter;
    CK(h, h->f32 ? sweep32_f32(h->shape, mode, a, h->grid, h->stream)
                 : sweep_f64(h->shape, mode, a, h->grid, h->stream));
    return GABE_OK;
}

int gw_chain(gabe_handle *h, int slot, cudaStream_t s) {
    int rc = source_fft(h, slot, s);
    if (rc) return rc;
    return kspace(h, slot, s);
}

// Enqueues nsteps steps starting from state buffer `cur`.  The field chain
// (sweep A, sweep B) runs on the handle's stream.  With two source buffers
// the GW chain of each step (FFT, k-space) forks onto gw_stream after its
// sweep A and overlaps sweep B and the next step's sweep A; a step's sweep A
// waits for the k-space pass two steps back (same source buffer), and the
// enqueue ends joined on the handle's stream.  Nothing in the field chain
// reads the GW chain (no backreaction), so only buffer reuse orders them.
// With `ev` (5 events per step, serial only) the phase boundaries sweep A |
// FFT | k-space | sweep B are recorded for gabe_profile_steps.
int enqueue_steps(gabe_handle *h, int cur, int nsteps, bool serial, cudaEvent_t *ev = nullptr) {
    const bool fork = overlapped(h) && !serial;
    for (int s = 0; s < nsteps; s++) {
        const int c = cur ^ (s & 1);
        const int slot = fork ? c : 0;
        cudaEvent_t *e = ev ? ev + 5 * s : nullptr;
        if (fork && s >= 2) CK(h, cudaStreamWaitEvent(h->stream, h->ev_k[slot], 0));
        if (e) CK(h, cudaEventRecord(e[0], h->stream));
        int rc = sweep(h, h->evolve_gw ? MODE_A_GW : MODE_A, c, 0, slot);
        if (rc) return rc;
        if (e) CK(h, cudaEventRecord(e[1], h->stream));
        if (h->evolve_gw) {
            if (fork) {
                CK(h, cudaEventRecord(h->ev_a, h->stream));
                CK(h, cudaStreamWaitEvent(h->gw_stream, h->ev_a, 0));
                rc = gw_chain(h, slot, h->gw_stream);
                if (rc) return rc;
                CK(h, cudaEventRecord(h->ev_k[slot], h->gw_stream));
            } else {
                rc = source_fft(h, slot, h->stream);
                if (rc) return rc;
                if (e) CK(h, cudaEventRecord(e[2], h->stream));
                rc = kspace(h, slot, h->stream);
                if (rc) return rc;
            }
        } else if (e) {
            CK(h, cudaEventRecord(e[2], h->stream));
        }
        if (e) CK(h, cudaEventRecord(e[3], h->stream));
        rc = sweep(h, MODE_B, c, 1, slot);
        if (rc) return rc;
        if (e) CK(h, cudaEventRecord(e[4], h->stream));
    }
    if (fork && nsteps > 0) CK(h, cudaStreamWaitEvent(h->stream, h->ev_k[cur ^ ((nsteps - 1) & 1)], 0));
    return GABE_OK;
}

int capture(gabe_handle *h, int cur, int nsteps, cudaGraphExec_t *out) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int rc = enqueue_steps(h, cur, nsteps, false);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc != GABE_OK || e != cudaSuccess || !g) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        h->err.clear();
        return 1;
    }
    // keep the captured per-kernel stream priorities (field chain high, GW chain low)
    e = cudaGraphInstantiate(out, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return 1;
    }
    return 0;
}

int build_graphs(gabe_handle *h) {
    h->graph_tried = true;
    if (h->p.flags & GABE_FLAG_NO_GRAPH) return GABE_OK;
    for (int par = 0; par < 2; par++)
        if (capture(h, par, 1, &h->graph[par]) || capture(h, par, 2, &h->graph2[par])) return GABE_OK;
    h->graph_ok = true;
    return GABE_OK;
}

int read_scalars(gabe_handle *h, DevScalars *out) {
    if (h->e0_stale) {
        int rc = sweep(h, MODE_E0, h->cur, 2);
        if (rc) return rc;
        h->e0_stale = false;
    }
    CK(h, cudaStreamSynchronize(h->stream));
    CK(h, cudaMemcpy(out, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost));
    if (out->status & ST_TIMEOUT)
        return set_err(h, GABE_ERR_TIMEOUT, "a bulk copy of the GW transform did not complete (bounded wait gave up)");
    if (out->status & ST_NONFINITE)
        return set_err(h, GABE_ERR_NONFINITE, "non-finite energy density at step %lld", out->step);
    return GABE_OK;
}

// Device address of fbar[f] / dfbar[f] inside the scalar block.
double *dev_mean(gabe_handle *h, bool momentum, int f) {
    const size_t off = momentum ? offsetof(DevScalars, dfbar) : offsetof(DevScalars, fbar);
    return reinterpret_cast<double *>(reinterpret_cast<char *>(h->sc) + off) + f;
}

// k-points per staging chunk for the 12-component FP64 GW layout
size_t gw_chunk(gabe_handle *h) {
    size_t c = h->S_bytes / (12 * sizeof(double));
    return c < h->M ? c : h->M;
}

// h0/l0 in the reference layout -> amplitudes, rejecting non-TT input.
int upload_gw(gabe_handle *h, const double *h0, const double *l0) {
    double *stage = static_cast<double *>(h->S);
    const size_t chunk = gw_chunk(h), M = h->M;
    CK(h, cudaMemsetAsync(h->gwnorm, 0, 4 * sizeof(double), h->stream));
    const double *src[2] = {h0, l0};
    for (int w = 0; w < 2; w++) {
        if (!src[w]) {
            CK(h, cudaMemsetAsync(static_cast<char *>(h->G) + (size_t)2 * w * M * 2 * h->esz, 0, 2 * M * 2 * h->esz,
                                  h->stream));
            continue;
        }
        for (size_t m0 = 0; m0 < M; m0 += chunk) {
            const size_t cnt = (M - m0) < chunk ? (M - m0) : chunk;
            for (int q = 0; q < 12; q++)
                CK(h, cudaMemcpyAsync(stage + (size_t)q * cnt, src[w] + (size_t)q * M + m0, cnt * 8,
                                      cudaMemcpyHostToDevice, h->stream));
            CK(h, h->f32 ? gw_pack_f32(stage, cnt, m0, h->N, M, h->G, w, h->gwnorm + 2 * w, h->fftt, h->stream)
                         : gw_pack_f64(stage, cnt, m0, h->N, M, h->G, w, h->gwnorm + 2 * w, h->stream));
        }
    }
    double nr[4];
    CK(h, cudaMemcpyAsync(nr, h->gwnorm, sizeof(nr), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    for (int w = 0; w < 2; w++)
        if (!(nr[2 * w + 1] <= 1e-20 * nr[2 * w]))
            return set_err(h, GABE_ERR_PARAM,
                           "%s0 is not transverse-traceless (relative non-TT norm %.3g); the evolution keeps h and l "
                           "TT, so only TT data (e.g. from a previous run) can be uploaded",
                           w ? "l" : "h", nr[2 * w] > 0 ? sqrt(nr[2 * w + 1] / nr[2 * w]) : 0.0);
    return GABE_OK;
}

int download_gw(gabe_handle *h, double *h0, double *l0) {
    double *stage = static_cast<double *>(h->S);
    const size_t chunk = gw_chunk(h), M = h->M;
    double *dst[2] = {h0, l0};
    for (int w = 0; w < 2; w++) {
        if (!dst[w]) continue;
        for (size_t m0 = 0; m0 < M; m0 += chunk) {
            const size_t cnt = (M - m0) < chunk ? (M - m0) : chunk;
            CK(h, h->f32 ? gw_unpack_f32(h->G, cnt, m0, h->N, M, w, stage, h->fftt, h->stream)
                         : gw_unpack_f64(h->G, cnt, m0, h->N, M, w, stage, h->stream));
            for (int q = 0; q < 12; q++)
                CK(h, cudaMemcpyAsync(dst[w] + (size_t)q * M + m0, stage + (size_t)q * cnt, cnt * 8,
                                      cudaMemcpyDeviceToHost, h->stream));
        }
    }
    return GABE_OK;
}

int mean_blocks(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 592 ? (b ? b : 1) : 592);
}

}  // namespace

extern "C" {

void gabe_default_params(gabe_params *p, int N) {
    std::memset(p, 0, sizeof(*p));
    p->struct_size = (int32_t)sizeof(gabe_params);
    p->N = N;
    p->nflds = 2;
    p->gws_on = 0;
    p->expansion = 1;
    p->model = GABE_MODEL_LPHI4;
    p->precision = GABE_FP64;
    p->gw_spec_quirk = 1;
    p->L = 20.;
    p->dt = 0.01;
    const double phi0 = 0.342;
    p->model_c[0] = 1. / (phi0 * phi0);
    p->model_c[1] = 100. / (phi0 * phi0);
    p->device = -1;
    p->flags = 0;
    p->tile_ci = 0;
    p->tile_shape = -1;
}

int gabe_create(const gabe_params *p, gabe_handle **out) {
    if (!out) return set_err(nullptr, GABE_ERR_PARAM, "out is NULL");
    *out = nullptr;
    if (!p) return set_err(nullptr, GABE_ERR_PARAM, "params is NULL");
    if (p->struct_size != (int32_t)sizeof(gabe_params))
        return set_err(nullptr, GABE_ERR_PARAM, "struct_size %d != %zu", p->struct_size, sizeof(gabe_params));
    char msg[160];
    if (!params_valid(*p, msg, sizeof(msg))) return set_err(nullptr, GABE_ERR_PARAM, "%s (N = %d)", msg, p->N);
    const int known = GABE_FLAG_NO_GRAPH | GABE_FLAG_NO_OVERLAP | GABE_FLAG_OWN_FFT | GABE_FLAG_CUFFT_3D |
                      GABE_FLAG_TRANSPOSED_FFT;
    if (p->flags & ~known) return set_err(nullptr, GABE_ERR_PARAM, "unknown flags 0x%x", p->flags & ~known);
    const bool f32 = p->precision == GABE_FP32;
    if ((f32 ? plan_grid32(p->N, p->tile_shape, p->tile_ci) : plan_grid(p->N, p->tile_shape, p->tile_ci)).shape < 0)
        return set_err(nullptr, GABE_ERR_PARAM, "N = %d: no stencil tile divides N (%s)", p->N,
                       f32 ? "FP32 storage needs N %% 16 == 0" : "FP64 needs N %% 4 == 0");

    gabe_handle *h = new (std::nothrow) gabe_handle();
    if (!h) return set_err(nullptr, GABE_ERR_NOMEM, "host allocation failed");
    h->p = *p;
    int rc = GABE_OK;
    auto bail = [&](int code) {
        g_create_error = h->err;
        gabe_destroy(h);
        return code;
    };
    if (p->device >= 0) {
        if (cudaSetDevice(p->device) != cudaSuccess) {
            cudaGetLastError();
            set_err(h, GABE_ERR_CUDA, "cudaSetDevice(%d) failed", p->device);
            return bail(GABE_ERR_CUDA);
        }
    }
    if (cudaGetDevice(&h->dev) != cudaSuccess) {
        cudaGetLastError();
        set_err(h, GABE_ERR_CUDA, "no CUDA device");
        return bail(GABE_ERR_CUDA);
    }
    h->f32 = p->precision == GABE_FP32;
    h->esz = h->f32 ? 4 : 8;
    h->N = p->N;
    h->nz = p->N / 2 + 1;
    h->n3 = (size_t)p->N * p->N * p->N;
    h->M = (size_t)p->N * p->N * h->nz;
    h->lc = make_lattice_consts(*p);
    choose_tile(h);
    h->nbins = gabe_spectra_numbins(p->N);

    // The field chain (sweeps) is on the critical path of every step; the GW
    // chain (transforms, k-space) of step n may run until sweep A of step n+2.
    // The field stream gets the highest priority so that its blocks take SMs
    // as the GW chain's blocks retire instead of queueing behind them.
    int prio_low = 0, prio_high = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) {
        cudaGetLastError();
        prio_low = prio_high = 0;
    }
    h->prio_low = prio_low;
    if (cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess) {
        cudaGetLastError();
        set_err(h, GABE_ERR_CUDA, "cudaStreamCreate failed");
        return bail(GABE_ERR_CUDA);
    }
    const size_t bin_smem = (size_t)h->nbins * (3 * 8 + 4);
    if (bin_smem > 48 * 1024 && configure_bins(bin_smem) != cudaSuccess) {
        cudaGetLastError();
        set_err(h, GABE_ERR_CUDA, "cudaFuncSetAttribute(%zu bytes shared) failed", bin_smem);
        return bail(GABE_ERR_CUDA);
    }
    const size_t field_bytes = 2 * h->n3 * h->esz;
    for (int b = 0; b < 2; b++) {
        if ((rc = dalloc(h, &h->X[b], field_bytes))) return bail(rc);
        if ((rc = dalloc(h, &h->D[b], field_bytes))) return bail(rc);
    }
    if (p->gws_on) {
        if ((rc = dalloc(h, &h->G, 8 * h->M * h->esz))) return bail(rc);
        if ((rc = dalloc(h, (void **)&h->gwnorm, 4 * sizeof(double)))) return bail(rc);
    }
    // sources need 10 padded slots; spectra need 2; uploads stage one FP64 field array
    h->evolve_gw = p->gws_on && p->expansion == 1;
    // the transposed form: on request, and by default for FP32 at N >= 128 (measured fastest there:
    // per step 8.1 against ~11 ms at 512^3, 1.21 against 1.41 at 256^3, 0.170 against 0.192 at 128^3
    // with cuFFT's plan and the overlapped k-space chain; a tie at 64^3)
    h->fftt = h->evolve_gw && h->f32 && fftt_supported(h->N) &&
              ((p->flags & GABE_FLAG_TRANSPOSED_FFT) ||
               (h->N >= 128 && !(p->flags & (GABE_FLAG_OWN_FFT | GABE_FLAG_CUFFT_3D))));
    h->nslots = h->evolve_gw ? 2 * kSrc : 2;
    h->S_bytes = (size_t)h->nslots * p->N * p->N * (p->N + 2) * h->esz;
    if ((rc = dalloc(h, &h->S, h->S_bytes))) return bail(rc);
    if (h->fftt) {  // the transposed transform's first pass writes out of place
        if ((rc = dalloc(h, &h->S2, h->S_bytes))) return bail(rc);
    } else if (h->evolve_gw && !(p->flags & GABE_FLAG_NO_OVERLAP)) {
        // optional: without it the GW chain simply runs in line
        if (dalloc(h, &h->S2, h->S_bytes) != GABE_OK) {
            h->S2 = nullptr;
            h->err.clear();
        }
    }
    if (cudaStreamCreateWithPriority(&h->gw_stream, cudaStreamNonBlocking, h->prio_low) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_a, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_k[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_k[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        set_err(h, GABE_ERR_CUDA, "stream/event creation failed");
        return bail(GABE_ERR_CUDA);
    }
    const size_t nblk_stencil = (size_t)h->grid.x * h->grid.y * h->grid.z;
    h->npartials = kNV * (nblk_stencil > 4096 ? nblk_stencil : 4096);
    if ((rc = dalloc(h, (void **)&h->partials, h->npartials * sizeof(double)))) return bail(rc);
    if ((rc = dalloc(h, (void **)&h->counters, 8 * sizeof(unsigned int)))) return bail(rc);
    if ((rc = dalloc(h, (void **)&h->sc, sizeof(DevScalars)))) return bail(rc);
    if ((rc = dalloc(h, (void **)&h->bin_part, (size_t)kBinBlocks * 3 * h->nbins * sizeof(double)))) return bail(rc);
    if ((rc = dalloc(h, (void **)&h->bin_cnt_part, (size_t)kBinBlocks * h->nbins * sizeof(unsigned int))))
        return bail(rc);
    if ((rc = dalloc(h, (void **)&h->bin_sum, (size_t)4 * h->nbins * sizeof(double)))) return bail(rc);
    if ((rc = dalloc(h, (void **)&h->outres, 8 * sizeof(double)))) return bail(rc);
    if (cudaMemset(h->counters, 0, 8 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMemset(h->sc, 0, sizeof(DevScalars)) != cudaSuccess) {
        cudaGetLastError();
        set_err(h, GABE_ERR_CUDA, "cudaMemset failed");
        return bail(GABE_ERR_CUDA);
    }
    if ((rc = make_plans(h))) return bail(rc);
    *out = h;
    return GABE_OK;
}

int gabe_destroy(gabe_handle *h) {
    if (!h) return GABE_OK;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gw_stream) cudaStreamSynchronize(h->gw_stream);
    for (int i = 0; i < 2; i++) {
        if (h->graph[i]) cudaGraphExecDestroy(h->graph[i]);
        if (h->graph2[i]) cudaGraphExecDestroy(h->graph2[i]);
        if (h->ev_k[i]) cudaEventDestroy(h->ev_k[i]);
    }
    if (h->ev_a) cudaEventDestroy(h->ev_a);
    if (h->have_plan_src) cufftDestroy(h->plan_src);
    if (h->have_plan_spec) cufftDestroy(h->plan_spec);
    void *bufs[] = {h->X[0], h->X[1], h->D[0], h->D[1], h->G, h->gwnorm, h->S, h->S2, h->partials, h->counters,
                    h->sc, h->bin_part, h->bin_cnt_part, h->bin_sum, h->fft_work, h->outres};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->gw_stream) cudaStreamDestroy(h->gw_stream);
    cudaGetLastError();
    delete h;
    return GABE_OK;
}

int gabe_upload_state(gabe_handle *h, const double *field0, const double *dfield0, const double *h0,
                      const double *l0, double a0, double adot0) {
    if (!h) return GABE_ERR_PARAM;
    if (!field0 || !dfield0) return set_err(h, GABE_ERR_PARAM, "field0/dfield0 must not be NULL");
    if (!(a0 > 0) || !std::isfinite(a0) || !std::isfinite(adot0))
        return set_err(h, GABE_ERR_PARAM, "a0 must be positive and finite");
    CK(h, cudaSetDevice(h->dev));
    h->err.clear();
    h->uploaded = false;  // until the whole state is in place: a refused upload leaves no half-new state to step
    DevScalars s{};
    s.a[0] = a0;
    s.adot[0] = adot0;
    if (h->p.expansion == 0) {  // both stages keep the initial expansion (g2init.cpp:18-24)
        s.a[1] = a0;
        s.adot[1] = adot0;
    }
    s.adot_given = 1;
    CK(h, cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
    const size_t nf = h->n3;
    if (!h->f32) {
        CK(h, cudaMemcpyAsync(h->X[0], field0, 2 * nf * 8, cudaMemcpyHostToDevice, h->stream));
        CK(h, cudaMemcpyAsync(h->D[0], dfield0, 2 * nf * 8, cudaMemcpyHostToDevice, h->stream));
    } else {
        // each field array: stage in S as FP64, take its mean, store float fluctuations
        double *stage = static_cast<double *>(h->S);
        const double *src[2] = {field0, dfield0};
        void *dst[2] = {h->X[0], h->D[0]};
        for (int a = 0; a < 2; a++)
            for (int f = 0; f < 2; f++) {
                double *mean = dev_mean(h, a != 0, f);
                CK(h, cudaMemcpyAsync(stage, src[a] + f * nf, nf * 8, cudaMemcpyHostToDevice, h->stream));
                CK(h, mean_f64(stage, nf, h->partials, h->counters + 3, mean, mean_blocks(nf), h->stream));
                CK(h, to_fluct(stage, nf, mean, static_cast<float *>(dst[a]) + f * nf, h->stream));
            }
    }
    if (h->p.gws_on) {
        int rc = upload_gw(h, h0, l0);
        if (rc) return rc;
    }
    h->cur = 0;
    h->e0_stale = true;
    DevScalars chk;
    int rc = read_scalars(h, &chk);
    if (rc) return rc;
    h->uploaded = true;
    return GABE_OK;
}

int gabe_step(gabe_handle *h, int nsteps) {
    if (!h) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "gabe_step before gabe_upload_state");
    if (nsteps < 0) return set_err(h, GABE_ERR_PARAM, "nsteps < 0");
    CK(h, cudaSetDevice(h->dev));
    if (!h->graph_tried) {
        int rc = build_graphs(h);
        if (rc) return rc;
    }
    if (h->graph_ok) {
        int left = nsteps;
        for (; left >= 2; left -= 2) CK(h, cudaGraphLaunch(h->graph2[h->cur], h->stream));
        if (left) {
            CK(h, cudaGraphLaunch(h->graph[h->cur], h->stream));
            h->cur ^= 1;
        }
    } else {
        int rc = enqueue_steps(h, h->cur, nsteps, false);
        if (rc) return rc;
        h->cur ^= (nsteps & 1);
    }
    if (nsteps > 0) h->e0_stale = true;
    return GABE_OK;
}

int gabe_profile_steps(gabe_handle *h, int nsteps, double ms_out[4]) {
    if (!h || !ms_out || nsteps < 1) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "profile before upload");
    CK(h, cudaSetDevice(h->dev));
    std::vector<cudaEvent_t> ev((size_t)5 * nsteps);
    for (auto &e : ev) CK(h, cudaEventCreate(&e));
    int rc = GABE_OK;
    rc = enqueue_steps(h, h->cur, nsteps, true, ev.data());
    h->cur ^= (nsteps & 1);
    h->e0_stale = true;
    double acc[4] = {0, 0, 0, 0};
    if (rc == GABE_OK && cudaStreamSynchronize(h->stream) == cudaSuccess) {
        for (int s = 0; s < nsteps; s++)
            for (int q = 0; q < 4; q++) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[5 * s + q], ev[5 * s + q + 1]);
                acc[q] += ms;
            }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    for (int q = 0; q < 4; q++) ms_out[q] = acc[q] / nsteps;
    DevScalars sc;
    return read_scalars(h, &sc);
}

// Transposed form: nreps full steps with events around each of its three launches.
static int profile_fftt_passes(gabe_handle *h, int nreps, double ms_out[3]) {
    std::vector<cudaEvent_t> ev((size_t)4 * nreps, nullptr);
    for (auto &x : ev) CK(h, cudaEventCreate(&x));
    int rc = GABE_OK;
    for (int r = 0; r < nreps && rc == GABE_OK; r++) {
        const int c = h->cur ^ (r & 1);
        cudaEvent_t *e = ev.data() + 4 * r;
        rc = sweep(h, MODE_A_GW, c, 0, 0);
        if (rc) break;
        cudaError_t ce = cudaEventRecord(e[0], h->stream);
        if (ce == cudaSuccess) ce = fftt_rows_f32(h->N, static_cast<const float *>(h->S), h->S2, 2 * kSrc, &h->sc->status,
                                                         h->stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e[1], h->stream);
        if (ce == cudaSuccess) ce = fftt_cols_f32(h->N, h->S2, h->S, 2 * kSrc, &h->sc->status, h->stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e[2], h->stream);
        if (ce == cudaSuccess)
            ce = fftt_ikspace_f32(h->N, h->S, h->G, h->sc, h->lc, 0, &h->sc->status, h->stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e[3], h->stream);
        if (ce != cudaSuccess) {
            rc = set_err(h, GABE_ERR_CUDA, "profile launch: %s", cudaGetErrorString(ce));
            break;
        }
        rc = sweep(h, MODE_B, c, 1, 0);
    }
    h->cur ^= (nreps & 1);
    h->e0_stale = true;
    double acc[3] = {0, 0, 0};
    if (rc == GABE_OK && cudaStreamSynchronize(h->stream) == cudaSuccess)
        for (int r = 0; r < nreps; r++)
            for (int q = 0; q < 3; q++) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[4 * r + q], ev[4 * r + q + 1]);
                acc[q] += ms;
            }
    for (auto &x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    for (int q = 0; q < 3; q++) ms_out[q] = acc[q] / nreps;
    DevScalars sc;
    return read_scalars(h, &sc);
}

int gabe_profile_fft_passes(gabe_handle *h, int nreps, double ms_out[3]) {
    if (!h || !ms_out || nreps < 1) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "profile before upload");
    if (h->fftt) {
        CK(h, cudaSetDevice(h->dev));
        return profile_fftt_passes(h, nreps, ms_out);
    }
    if (!h->own_fft) return set_err(h, GABE_ERR_STATE, "this handle does not use the library's 3-D FFT");
    CK(h, cudaSetDevice(h->dev));
    CK(h, cudaStreamSynchronize(h->stream));  // the last step's GW chain has finished with the sources
    std::vector<cudaEvent_t> ev((size_t)4 * nreps, nullptr);
    cudaError_t e = cudaSuccess;
    for (auto &x : ev)
        if (e == cudaSuccess) e = cudaEventCreate(&x);
    float *S = static_cast<float *>(h->S);  // transformed in place; the next sweep A rewrites it
    for (int r = 0; r < nreps && e == cudaSuccess; r++) {
        for (int p = 0; p < 3 && e == cudaSuccess; p++) {
            e = cudaEventRecord(ev[4 * r + p], h->stream);
            if (e == cudaSuccess) e = fft3d_pass_f32(h->N, S, fft_scratch(h), 2 * kSrc, p, h->stream);
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev[4 * r + 3], h->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    double acc[3] = {0, 0, 0};
    for (int r = 0; r < nreps && e == cudaSuccess; r++)
        for (int p = 0; p < 3; p++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[4 * r + p], ev[4 * r + p + 1]);
            acc[p] += ms;
        }
    for (auto &x : ev)
        if (x) cudaEventDestroy(x);
    CK(h, e);
    for (int p = 0; p < 3; p++) ms_out[p] = acc[p] / nreps;
    return GABE_OK;
}

int gabe_stream(gabe_handle *h, void **stream) {
    if (!h || !stream) return GABE_ERR_PARAM;
    *stream = (void *)h->stream;
    return GABE_OK;
}

int gabe_sync(gabe_handle *h) {
    if (!h) return GABE_ERR_PARAM;
    CK(h, cudaSetDevice(h->dev));
    DevScalars s;
    return read_scalars(h, &s);
}

int gabe_energies(gabe_handle *h, double out4[4], double *a, double *adot) {
    if (!h) return GABE_ERR_PARAM;
    CK(h, cudaSetDevice(h->dev));
    DevScalars s;
    int rc = read_scalars(h, &s);
    if (out4) {
        out4[0] = s.edkin[0];
        out4[1] = s.edpot[0];
        out4[2] = s.edgrad[0];
        out4[3] = s.edrho[0];
    }
    if (a) *a = s.a[0];
    if (adot) *adot = s.adot[0];
    return rc;
}

int gabe_scalars(gabe_handle *h, double out12[12]) {
    if (!h || !out12) return GABE_ERR_PARAM;
    CK(h, cudaSetDevice(h->dev));
    DevScalars s;
    int rc = read_scalars(h, &s);
    const double *src[6] = {s.a, s.adot, s.edkin, s.edpot, s.edgrad, s.edrho};
    for (int q = 0; q < 6; q++) {
        out12[2 * q] = src[q][0];
        out12[2 * q + 1] = src[q][1];
    }
    return rc;
}

int gabe_download_state(gabe_handle *h, double *field0, double *dfield0, double *h0, double *l0) {
    if (!h) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "download before upload");
    CK(h, cudaSetDevice(h->dev));
    const size_t nf = h->n3;
    const int c = h->cur;
    if (!h->f32) {
        if (field0) CK(h, cudaMemcpyAsync(field0, h->X[c], 2 * nf * 8, cudaMemcpyDeviceToHost, h->stream));
        if (dfield0) CK(h, cudaMemcpyAsync(dfield0, h->D[c], 2 * nf * 8, cudaMemcpyDeviceToHost, h->stream));
    } else {
        double *stage = static_cast<double *>(h->S);
        double *dst[2] = {field0, dfield0};
        const void *src[2] = {h->X[c], h->D[c]};
        for (int a = 0; a < 2; a++) {
            if (!dst[a]) continue;
            for (int f = 0; f < 2; f++) {
                const double *mean = dev_mean(h, a != 0, f);
                CK(h, from_fluct(static_cast<const float *>(src[a]) + f * nf, nf, mean, stage, h->stream));
                CK(h, cudaMemcpyAsync(dst[a] + f * nf, stage, nf * 8, cudaMemcpyDeviceToHost, h->stream));
            }
        }
    }
    if (h->p.gws_on) {
        int rc = download_gw(h, h0, l0);
        if (rc) return rc;
    }
    CK(h, cudaStreamSynchronize(h->stream));
    return GABE_OK;
}

int gabe_spectra_numbins(int N) { return ((int)(sqrt(3.) * N / 2 + 1)); }

namespace {
OutArgs out_args(gabe_handle *h) {
    OutArgs a{};
    a.X = h->X[h->cur];
    a.D = h->D[h->cur];
    a.sc = h->sc;
    a.c = h->lc;
    a.partials = h->partials;
    a.counter = h->counters + 6;
    a.res = h->outres;
    return a;
}
}  // namespace

int gabe_meansvars(gabe_handle *h, double out4[4]) {
    if (!h || !out4) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "meansvars before upload");
    CK(h, cudaSetDevice(h->dev));
    const OutArgs a = out_args(h);
    const int nblocks = 148 * 8;  // partials hold >= 2 * nblocks doubles
    for (int pass = 0; pass < 2; pass++)
        CK(h, h->f32 ? meansvars_f32(a, pass, nblocks, h->stream) : meansvars_f64(a, pass, nblocks, h->stream));
    double r[4];
    CK(h, cudaMemcpyAsync(r, h->outres, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    for (int f = 0; f < 2; f++) {
        out4[2 * f] = r[f];
        out4[2 * f + 1] = r[2 + f];
    }
    for (int f = 0; f < 2; f++) {
        const double av = r[f];
        if (av != 0. && av / av != 1.)  // g2output.cpp:106
            return set_err(h, GABE_ERR_NONFINITE, "Unstable solution developed. Field %d not numerical", f);
    }
    return GABE_OK;
}

size_t gabe_field_slice_rows(int N, int outdim, int skip) {
    if (N <= 0 || outdim < 1 || outdim > 3 || skip < 1) return 0;
    const size_t n = (size_t)((N + skip - 1) / skip);
    return outdim == 1 ? n : outdim == 2 ? n * n : n * n * n;
}

int gabe_field_slice(gabe_handle *h, int outdim, int skip, double *out, size_t out_len) {
    if (!h || !out) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "field slice before upload");
    const size_t rows = gabe_field_slice_rows(h->N, outdim, skip);
    if (rows == 0) return set_err(h, GABE_ERR_PARAM, "outdim must be 1..3 and skip >= 1");
    if (out_len < 3 * rows) return set_err(h, GABE_ERR_PARAM, "out holds %zu doubles, %zu needed", out_len, 3 * rows);
    CK(h, cudaSetDevice(h->dev));
    const int n = (h->N + skip - 1) / skip;
    const int nj = outdim > 1 ? n : 1, nk = n;
    const OutArgs a = out_args(h);
    double *stage = static_cast<double *>(h->S);  // free between steps (the step's last wait covers the GW chain)
    const size_t chunk = h->S_bytes / (3 * sizeof(double));
    for (size_t r0 = 0; r0 < rows; r0 += chunk) {
        const size_t cnt = rows - r0 < chunk ? rows - r0 : chunk;
        CK(h, h->f32 ? slice_f32(a, nj, nk, skip, r0, cnt, stage, h->stream)
                     : slice_f64(a, nj, nk, skip, r0, cnt, stage, h->stream));
        CK(h, cudaMemcpyAsync(out + 3 * r0, stage, cnt * 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    return GABE_OK;
}

int gabe_spectra_raw(gabe_handle *h, double *sums, double *counts, int nbins, int nseries) {
    if (!h) return GABE_ERR_PARAM;
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "spectra before upload");
    const int ns = 2 + (h->p.gws_on ? 1 : 0);
    if (nbins != h->nbins || nseries != ns)
        return set_err(h, GABE_ERR_PARAM, "spectra_raw wants nbins=%d nseries=%d", h->nbins, ns);
    CK(h, cudaSetDevice(h->dev));
    DevScalars s;
    int rc = read_scalars(h, &s);
    if (rc) return rc;
    rc = fft_r2c(h, h->plan_spec, h->X[h->cur], h->S);
    if (rc) return rc;
    BinArgs b{};
    b.F = h->S;
    b.G = h->G;
    b.part_sum = h->bin_part;
    b.part_cnt = h->bin_cnt_part;
    b.N = h->N;
    b.nbins = h->nbins;
    b.nseries = ns;
    b.quirk = h->p.gw_spec_quirk;
    b.fix_zero = h->f32 ? 1 : 0;
    b.gt = h->fftt ? 1 : 0;
    b.zero_re[0] = h->lc.gridsize * s.fbar[0];
    b.zero_re[1] = h->lc.gridsize * s.fbar[1];
    const size_t smem = (size_t)h->nbins * (ns * 8 + 4);
    Launch lb{dim3(kBinBlocks), dim3(256), smem, h->stream};
    CK(h, h->f32 ? bins_f32(b, lb) : bins_f64(b, lb));
    double *dsum = h->bin_sum, *dcnt = h->bin_sum + 3 * h->nbins;
    CK(h, bin_reduce(h->bin_part, h->bin_cnt_part, kBinBlocks, ns, h->nbins, dsum, dcnt, h->stream));
    CK(h, cudaMemcpyAsync(sums, dsum, (size_t)ns * h->nbins * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaMemcpyAsync(counts, dcnt, (size_t)h->nbins * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return GABE_OK;
}

int gabe_spectra(gabe_handle *h, double *out, int nbins, int ncols) {
    if (!h || !out) return GABE_ERR_PARAM;
    const int gws = h->p.gws_on;
    const int want = 5 + (gws ? 3 : 0);
    if (nbins != h->nbins || ncols != want)
        return set_err(h, GABE_ERR_PARAM, "spectra wants nbins=%d ncols=%d", h->nbins, want);
    const int ns = 2 + gws;
    std::vector<double> sums((size_t)ns * nbins), cnt(nbins);
    int rc = gabe_spectra_raw(h, sums.data(), cnt.data(), nbins, ns);
    if (rc) return rc;
    DevScalars s;
    rc = read_scalars(h, &s);
    if (rc) return rc;
    return gabe_spectra_from_sums(&h->p, s.edrho[0], sums.data(), cnt.data(), nbins, out, ncols);
}

int gabe_spectra_from_sums(const gabe_params *p, double edrho0, const double *sums, const double *cnt, int nbins,
                           double *out, int ncols) {
    if (!p || !sums || !cnt || !out) return GABE_ERR_PARAM;
    const int gws = p->gws_on;
    if (nbins != gabe_spectra_numbins(p->N) || ncols != 5 + (gws ? 3 : 0)) return GABE_ERR_PARAM;
    // normalisation of g2spectra.cpp:27,94-103,114-117,186-195
    const double L = p->L;
    const int N = p->N;
    const double spec_norm = pow(L / (double)N, 6.) * pow(2. * M_PI / L, 3.);
    const double hub = sqrt(8. * M_PI / 3.) * sqrt(edrho0);
    const double dp = 2. * M_PI / (double)L;
    const double norm1 = 4.e-5 / pow(100., .333) / 24. / M_PI / M_PI / pow(L, 3.) / (hub * hub);
    for (int b = 0; b < nbins; b++) {
        double *row = out + (size_t)b * ncols;
        row[0] = 2. * M_PI * b / L;
        for (int f = 0; f < 2; f++) {
            const double pw = sums[(size_t)f * nbins + b], np = cnt[b];
            if (np > 0) {
                row[1 + 2 * f] = pw * spec_norm / np;
                row[2 + 2 * f] = pow((double)b * 2. * M_PI / L, 3) * pw * spec_norm / np / 2. / M_PI / M_PI;
            } else {
                row[1 + 2 * f] = 0.;
                row[2 + 2 * f] = 0.;
            }
        }
        if (gws) {
            const double pw = sums[(size_t)2 * nbins + b], np = cnt[b];
            if (np > 0) {
                row[5] = pw * spec_norm / np;
                row[6] = norm1 * pow((double)b * 2 * M_PI / L, 3.) * pw / np;
            } else {
                row[5] = 0.;
                row[6] = 0.;
            }
            row[7] = dp * (double)b;
        }
    }
    return GABE_OK;
}

// ---------------------------------------------------------------------------
// Checkpoint / restart (gabe_dump.h files with the restart block)
// ---------------------------------------------------------------------------
namespace {

struct FileCloser {
    FILE *f;
    ~FileCloser() {
        if (f) fclose(f);
    }
};

// Device bytes -> file through a pinned-free host bounce buffer of `chunk` bytes.
int write_device(gabe_handle *h, FILE *f, const void *dev, size_t bytes, std::vector<char> &bounce) {
    for (size_t o = 0; o < bytes; o += bounce.size()) {
        const size_t n = bytes - o < bounce.size() ? bytes - o : bounce.size();
        CK(h, cudaMemcpy(bounce.data(), static_cast<const char *>(dev) + o, n, cudaMemcpyDeviceToHost));
        if (fwrite(bounce.data(), 1, n, f) != n) return set_err(h, GABE_ERR_PARAM, "checkpoint write failed");
    }
    return GABE_OK;
}

int read_device(gabe_handle *h, FILE *f, void *dev, size_t bytes, std::vector<char> &bounce) {
    for (size_t o = 0; o < bytes; o += bounce.size()) {
        const size_t n = bytes - o < bounce.size() ? bytes - o : bounce.size();
        if (fread(bounce.data(), 1, n, f) != n) return set_err(h, GABE_ERR_PARAM, "checkpoint file is truncated");
        CK(h, cudaMemcpy(static_cast<char *>(dev) + o, bounce.data(), n, cudaMemcpyHostToDevice));
    }
    return GABE_OK;
}

void fill_restart(const gabe_handle *h, gabe_restart_header *r) {
    std::memset(r, 0, sizeof(*r));
    std::memcpy(r->magic, GABE_RESTART_MAGIC, 8);
    r->precision = h->p.precision;
    r->gw_layout = h->fftt ? 1 : 0;
    r->expansion = h->p.expansion;
    r->tile_shape = h->shape;
    r->tile_ci = h->ci;
    r->e0_stale = h->e0_stale ? 1 : 0;
    r->scalar_bytes = (int32_t)sizeof(DevScalars);
    r->elem_bytes = (int32_t)h->esz;
    r->field_bytes = (int64_t)(2 * h->n3 * h->esz);
    r->gw_bytes = h->p.gws_on ? (int64_t)(8 * h->M * h->esz) : 0;
}

}  // namespace

int gabe_save_state(gabe_handle *h, const char *path) {
    if (!h) return GABE_ERR_PARAM;
    if (!path) return set_err(h, GABE_ERR_PARAM, "path is NULL");
    if (!h->uploaded) return set_err(h, GABE_ERR_STATE, "save before upload");
    CK(h, cudaSetDevice(h->dev));
    DevScalars sc;
    int rc = read_scalars(h, &sc);  // synchronises; reduces the stage-0 energies if they are stale
    if (rc) return rc;
    FileCloser fc{fopen(path, "wb")};
    if (!fc.f) return set_err(h, GABE_ERR_PARAM, "cannot open %s for writing", path);
    gabe_dump_header hd;
    gabe_dump_header_init(&hd, h->N, 2, h->p.gws_on, 8, h->p.model);
    hd.step = sc.step;
    hd.t = (double)sc.step * h->p.dt;
    hd.L = h->p.L;
    hd.dt = h->p.dt;
    for (int s = 0; s < 2; s++) {
        hd.a[s] = sc.a[s];
        hd.adot[s] = sc.adot[s];
        hd.edkin[s] = sc.edkin[s];
        hd.edpot[s] = sc.edpot[s];
        hd.edgrad[s] = sc.edgrad[s];
        hd.edrho[s] = sc.edrho[s];
    }
    if (fwrite(&hd, sizeof(hd), 1, fc.f) != 1) return set_err(h, GABE_ERR_PARAM, "checkpoint write failed");
    // the portable part: FP64 arrays in the reference's layout, one at a time
    {
        const size_t nf = 2 * h->n3, ng = gabe_dump_gw_count(h->N);
        std::vector<double> buf(h->p.gws_on && ng > nf ? ng : nf);
        for (int a = 0; a < (h->p.gws_on ? 4 : 2); a++) {
            double *ptr[4] = {nullptr, nullptr, nullptr, nullptr};
            ptr[a] = buf.data();
            rc = gabe_download_state(h, ptr[0], ptr[1], ptr[2], ptr[3]);
            if (rc) return rc;
            const size_t n = a < 2 ? nf : ng;
            if (fwrite(buf.data(), sizeof(double), n, fc.f) != n)
                return set_err(h, GABE_ERR_PARAM, "checkpoint write failed");
        }
    }
    // the restart block: the device state as it is
    gabe_restart_header r;
    fill_restart(h, &r);
    if (fwrite(&r, sizeof(r), 1, fc.f) != 1 || fwrite(&sc, sizeof(sc), 1, fc.f) != 1)
        return set_err(h, GABE_ERR_PARAM, "checkpoint write failed");
    std::vector<char> bounce((size_t)64 << 20);
    if ((rc = write_device(h, fc.f, h->X[h->cur], (size_t)r.field_bytes, bounce)) ||
        (rc = write_device(h, fc.f, h->D[h->cur], (size_t)r.field_bytes, bounce)))
        return rc;
    if (r.gw_bytes && (rc = write_device(h, fc.f, h->G, (size_t)r.gw_bytes, bounce))) return rc;
    FILE *f = fc.f;
    fc.f = nullptr;
    if (fclose(f) != 0) return set_err(h, GABE_ERR_PARAM, "checkpoint write failed");
    return GABE_OK;
}

int gabe_load_state(gabe_handle *h, const char *path, int *restored) {
    if (!h) return GABE_ERR_PARAM;
    if (restored) *restored = 0;
    if (!path) return set_err(h, GABE_ERR_PARAM, "path is NULL");
    CK(h, cudaSetDevice(h->dev));
    h->err.clear();
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return set_err(h, GABE_ERR_PARAM, "cannot open %s", path);
    gabe_dump_header hd;
    if (fread(&hd, sizeof(hd), 1, fc.f) != 1 || std::memcmp(hd.magic, GABE_DUMP_MAGIC, 8) != 0 ||
        hd.version != GABE_DUMP_VERSION || hd.elem_bytes != 8)
        return set_err(h, GABE_ERR_PARAM, "%s is not a gabe_dump.h state dump", path);
    if (hd.N != h->N || hd.nflds != 2)
        return set_err(h, GABE_ERR_PARAM, "dump holds an N = %d lattice with %d fields; the handle's N is %d", hd.N,
                       hd.nflds, h->N);
    if (hd.L != h->p.L || hd.dt != h->p.dt)
        return set_err(h, GABE_ERR_PARAM, "dump was written with L = %g, dt = %g; the handle has L = %g, dt = %g",
                       hd.L, hd.dt, h->p.L, h->p.dt);
    if (hd.model != h->p.model) return set_err(h, GABE_ERR_PARAM, "dump model %d != handle model %d", hd.model, h->p.model);
    const size_t nf = 2 * h->n3, ng = gabe_dump_gw_count(h->N);
    const long long payload = (long long)(2 * nf + (hd.gws ? 2 * ng : 0)) * 8;
    // the restart block, if the file has one that fits this handle
    gabe_restart_header r;
    gabe_restart_header want;
    fill_restart(h, &want);
    bool native = false;
    if (fseeko(fc.f, (off_t)(sizeof(hd) + payload), SEEK_SET) == 0 && fread(&r, sizeof(r), 1, fc.f) == 1 &&
        std::memcmp(r.magic, GABE_RESTART_MAGIC, 8) == 0) {
        native = r.precision == want.precision && r.gw_layout == want.gw_layout && r.expansion == want.expansion &&
                 r.scalar_bytes == want.scalar_bytes && r.elem_bytes == want.elem_bytes &&
                 r.field_bytes == want.field_bytes && r.gw_bytes == want.gw_bytes && hd.gws == h->p.gws_on;
    }
    if (native) {
        DevScalars sc;
        if (fread(&sc, sizeof(sc), 1, fc.f) != 1) return set_err(h, GABE_ERR_PARAM, "checkpoint file is truncated");
        sc.status = 0;
        CK(h, cudaStreamSynchronize(h->stream));
        h->uploaded = false;  // a read that fails below leaves a partly overwritten state: no steps on it
        std::vector<char> bounce((size_t)64 << 20);
        int rc;
        if ((rc = read_device(h, fc.f, h->X[0], (size_t)r.field_bytes, bounce)) ||
            (rc = read_device(h, fc.f, h->D[0], (size_t)r.field_bytes, bounce)))
            return rc;
        if (r.gw_bytes && (rc = read_device(h, fc.f, h->G, (size_t)r.gw_bytes, bounce))) return rc;
        CK(h, cudaMemcpy(h->sc, &sc, sizeof(sc), cudaMemcpyHostToDevice));
        h->cur = 0;
        h->e0_stale = r.e0_stale != 0;
        h->uploaded = true;
        if (restored) *restored = 1;
        return GABE_OK;
    }
    // the portable part: upload as an initial state (the reference harness's dumps have no restart block)
    if (fseeko(fc.f, (off_t)sizeof(hd), SEEK_SET) != 0) return set_err(h, GABE_ERR_PARAM, "seek failed in %s", path);
    std::vector<double> f(nf), d(nf), hh, ll;
    if (fread(f.data(), 8, nf, fc.f) != nf || fread(d.data(), 8, nf, fc.f) != nf)
        return set_err(h, GABE_ERR_PARAM, "%s is truncated", path);
    if (hd.gws && h->p.gws_on) {
        hh.resize(ng);
        ll.resize(ng);
        if (fread(hh.data(), 8, ng, fc.f) != ng || fread(ll.data(), 8, ng, fc.f) != ng)
            return set_err(h, GABE_ERR_PARAM, "%s is truncated", path);
    }
    return gabe_upload_state(h, f.data(), d.data(), hh.empty() ? nullptr : hh.data(), ll.empty() ? nullptr : ll.data(),
                             hd.a[0], hd.adot[0]);
}

const char *gabe_last_error(const gabe_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

size_t gabe_device_bytes(const gabe_handle *h) { return h ? h->dev_bytes : 0; }

int gabe_graph_active(const gabe_handle *h) {
    if (!h) return -GABE_ERR_PARAM;
    return h->graph_tried ? (h->graph_ok ? 1 : 0) : -1;
}

int gabe_launches_per_step(const gabe_handle *h) {
    return h ? (h->evolve_gw ? (h->own_fft ? 6 : h->fftt ? 5 : 3) : 2) : 0;
}

}  // extern "C"
