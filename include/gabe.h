/*
 * gabe.h -- C ABI of the B200 (sm_100a) lattice-evolution library.
 *
 * The reference (GABE) has no plugin or FFI layer: its driver calls C++
 * functions that read and write global arrays.  This header is the boundary
 * that replaces the bodies of those functions:
 *
 *   reference call (file:line)                  replaced by
 *   ------------------------------------------  ---------------------------------
 *   step()             g2functions.cpp:201-304  gabe_step
 *     called from      g2main.cpp:126
 *   calcEnergy(0)      g2functions.cpp:168-174  gabe_upload_state (computes the
 *     called from      g2model.cpp:141,          stage-0 energies of the uploaded
 *                      g2init.cpp:28             state), gabe_energies
 *   adf(0)             g2functions.cpp:188-191  gabe_energies (adot)
 *   specOut(first)     g2spectra.cpp:23-234     gabe_spectra
 *     called from      g2output.cpp:161
 *   evolve_perts()     g2evolutionpert.cpp:343  inside gabe_step (calc_gws)
 *   globals field, dfield, a, adot, ed[kin,pot,  gabe_upload_state /
 *                      grad,rho], h, l (g2header.h:52-63,171-174)   gabe_download_state / gabe_scalars
 *
 * Conventions: every call returns an int status (GABE_OK == 0); the library
 * never exits the process.  Host arrays use the reference layout and FP64
 * whatever the device precision: field/dfield [nflds][N][N][N] (k fastest,
 * g2main.cpp:49,99), h/l [12][N][N][N/2+1] with the 12 components ordered as
 * (re,im) of 11,12,13,22,23,33 (g2evolutionpert.cpp:216-310).  A handle is
 * used from one host thread at a time and owns one CUDA stream; gabe_step
 * only enqueues work, calls that return data synchronise.
 */
#ifndef GABE_H
#define GABE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GABE_ABI_VERSION 1

enum gabe_status {
    GABE_OK = 0,
    GABE_ERR_PARAM = 1,     /* invalid or unsupported parameter */
    GABE_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    GABE_ERR_CUFFT = 3,     /* a cuFFT call failed */
    GABE_ERR_NOMEM = 4,     /* device allocation failed */
    GABE_ERR_NONFINITE = 5, /* NaN/Inf in the energies (the reference's meansvars abort, g2output.cpp:106-117) */
    GABE_ERR_TIMEOUT = 6,   /* a bounded device wait gave up */
    GABE_ERR_STATE = 7      /* call out of order (e.g. step before upload) */
};

enum gabe_precision {
    GABE_FP64 = 0, /* reference arithmetic, operation order kept */
    GABE_FP32 = 1  /* FP32 storage of fluctuations about an FP64 homogeneous
                      trajectory; FP64 scalars and reductions */
};

enum gabe_model {
    GABE_MODEL_QUADRATIC = 0, /* V = phi^2/2 + (g^2/m^2) phi^2 chi^2/2 (g2model.cpp:66-87);
                                 model_c = {mphi, gsq} */
    GABE_MODEL_LPHI4 = 1      /* V = lam phi^4/4 + g phi^2 chi^2/2 in program units;
                                 model_c = {lam_pr, gsq_pr} */
};

/* Flag values 4, 8 and 32 belonged to transform forms that measured slower
 * on B200 and were removed; gabe_create refuses them, like any unknown bit. */
enum gabe_flags {
    GABE_FLAG_NO_GRAPH = 1,  /* launch kernels one by one instead of replaying a CUDA graph */
    GABE_FLAG_NO_OVERLAP = 2, /* one source buffer: the GW transforms and k-space update run in line
                                 instead of overlapping the next field sweeps (saves 10 N^2(N+2)
                                 words of device memory).  With the library's 3-D FFT the chain runs
                                 in line anyway and the second buffer is the target of its column
                                 passes (out of place, faster); this flag makes them in place */
    GABE_FLAG_OWN_FFT = 16,     /* FP32 with N in {64, 128, 256, 512}: transform the GW sources with the
                                   library's in-layout three-pass 3-D r2c (the layout of a library r2c)
                                   followed by the separate k-space pass, instead of the default */
    GABE_FLAG_CUFFT_3D = 64,    /* FP32 at N in {128, 256, 512}: cuFFT's 3-D plan and the separate k-space
                                   pass instead of the default transposed transform (cuFFT's plan is the
                                   default at every other size and for FP64) */
    GABE_FLAG_TRANSPOSED_FFT = 128 /* FP32 with N in {64, 128, 256, 512}: the library's transposed three-pass
                                   transform -- rows along k, then along j, each written transposed so
                                   that every pass reads whole contiguous lines (bulk copies), and the
                                   pass along i fused with the TT projection and h/l update, so the
                                   transformed sources are never written back.  The default for FP32 at
                                   N in {128, 256, 512} (the fastest form measured there on B200; a tie
                                   with cuFFT's plan at 64); needs the second source buffer whatever
                                   GABE_FLAG_NO_OVERLAP says */
};

/* Run-time form of the g2parameters.h knobs that the hot path reads.  Two
 * fields are named differently from their knobs (gws_on, expansion) because
 * GABE defines calc_gws and expansion_type as macros, and a drop-in source
 * file includes both headers. */
typedef struct {
    int32_t struct_size;    /* sizeof(gabe_params) */
    int32_t N;              /* points per side (g2parameters.h:57) */
    int32_t nflds;          /* must be 2 (g2parameters.h:43) */
    int32_t gws_on;         /* calc_gws: 0/1 (g2parameters.h:55) */
    int32_t expansion;      /* expansion_type (g2parameters.h:62): 1 Friedmann expansion with tensor modes
                               (g2functions.cpp:234-271), 0 none (a, adot fixed, :207-232), 2 type 1
                               without tensor modes (:272-302) */
    int32_t model;          /* enum gabe_model */
    int32_t precision;      /* enum gabe_precision */
    int32_t gw_spec_quirk;  /* 1: GW spectrum reads l at kz=N/2 for the kz=0 plane, as g2spectra.cpp:149-164 does */
    double L;               /* box side (g2parameters.h:58) */
    double dt;              /* time step (g2parameters.h:61) */
    double model_c[2];      /* see enum gabe_model */
    int32_t device;         /* CUDA device ordinal, -1 = current */
    int32_t flags;          /* enum gabe_flags */
    int32_t tile_ci;        /* planes per stencil block along i, 0 = autotuned/default */
    int32_t tile_shape;     /* stencil tile shape id, -1 = autotuned/default */
    int64_t reserved[4];
} gabe_params;

typedef struct gabe_handle gabe_handle;

/* Fills p with the reference's defaults for an N^3 lattice (L=20, dt=0.01,
 * lambda phi^4 model with g^2/lambda=100, phi0=0.342, FP64, GWs off). */
void gabe_default_params(gabe_params *p, int N);

/* Creates a handle and allocates every device buffer.  *out is NULL on error. */
int gabe_create(const gabe_params *p, gabe_handle **out);
int gabe_destroy(gabe_handle *h);

/* Copies stage 0 of the state to the device: field0/dfield0 [nflds][N^3],
 * h0/l0 [12][N][N][N/2+1] (NULL = zero; ignored without GWs).  a0/adot0 are
 * taken as given -- after the reference's initialisation adot[0] belongs to
 * the homogeneous state (g2init.cpp:29) -- and the stage-0 energies are
 * recomputed on the device as calcEnergy(0) would.  An upload that fails
 * (e.g. non-TT h/l, a non-finite state) leaves the handle without a state:
 * calls that need one return GABE_ERR_STATE until an upload succeeds. */
int gabe_upload_state(gabe_handle *h, const double *field0, const double *dfield0,
                      const double *h0, const double *l0, double a0, double adot0);

/* Enqueues nsteps RK2 steps (step(), g2functions.cpp:234-271). */
int gabe_step(gabe_handle *h, int nsteps);

/* Runs nsteps steps with direct launches and CUDA events between phases and
 * returns the mean milliseconds per step of {stage-1 sweep, source FFTs,
 * k-space update, stage-2 sweep} (FFT and k-space are 0 without GWs).  The
 * state advances by nsteps.  Measurement hook; no reference counterpart. */
int gabe_profile_steps(gabe_handle *h, int nsteps, double ms_out[4]);

/* For a handle whose GW sources go through the library's 3-D FFT (FP32 at
 * N = 512 by default, or GABE_FLAG_OWN_FFT): runs its three passes nreps
 * times on the source buffer (in place; the next step rewrites the
 * sources) with CUDA events between them and returns the mean milliseconds
 * of {rows along k, pass along j, pass along i}.  With
 * GABE_FLAG_TRANSPOSED_FFT: runs nreps full steps (the state advances) with
 * events around the transform's launches and returns {rows along k, pass
 * along j, pass along i fused with the k-space update}.  Other handles:
 * GABE_ERR_STATE.  Measurement hook; no reference counterpart. */
int gabe_profile_fft_passes(gabe_handle *h, int nreps, double ms_out[3]);

/* The handle's CUDA stream (a cudaStream_t), so callers can order their own
 * work or events after queued steps.  No reference counterpart. */
int gabe_stream(gabe_handle *h, void **stream);

/* Waits for queued work; returns the first error seen on the device. */
int gabe_sync(gabe_handle *h);

/* Diagnostic of the bounded device waits, no handle needed: runs the
 * library's bounded mbarrier wait (the one every bulk copy, TMA load and
 * tcgen05 MMA wait of its kernels uses) on a barrier that nothing arrives
 * at, with a limit of limit_ns of GPU time (0 < limit_ns <= 1e10).  The
 * wait gives up, raises the timeout bit (2) in a device status word and
 * the kernel returns; *status_out receives that word, *waited_ns_out the
 * GPU time waited (either may be NULL).  Returns GABE_ERR_TIMEOUT when the
 * wait gave up, as designed; the context stays usable. */
int gabe_wait_probe(int64_t limit_ns, uint32_t *status_out, int64_t *waited_ns_out);

/* Stage-0 energies {kin, pot, grad, rho} and a, adot (synchronises). */
int gabe_energies(gabe_handle *h, double out4[4], double *a, double *adot);

/* All per-stage scalars as the reference keeps them: a[2], adot[2],
 * edkin[2], edpot[2], edgrad[2], edrho[2] (12 doubles, synchronises). */
int gabe_scalars(gabe_handle *h, double out12[12]);

/* Copies stage 0 back to the host; any pointer may be NULL. */
int gabe_download_state(gabe_handle *h, double *field0, double *dfield0, double *h0, double *l0);

/* Checkpoint of the current state to `path` (synchronises).  The file is a
 * gabe_dump.h state dump -- the FP64 arrays in the reference's layout and
 * the scalars, readable by anything that reads that format (the oracle,
 * the reference harness's --ic) -- followed by a restart block holding the
 * device state as the library keeps it.  The reference has no restartable
 * output (its slices are sampled %e text, g2output.cpp:25-68); this
 * replaces a restart from a reference initial-condition dump. */
int gabe_save_state(gabe_handle *h, const char *path);

/* Loads a gabe_dump.h file written for this handle's N, L, dt and model.
 * If it carries a restart block of the same precision, amplitude layout and
 * expansion type (a gabe_save_state file of an equal handle), that block
 * becomes the state and the run continues bit for bit (with the same tile
 * plan; *restored = 1).  Otherwise its FP64 arrays are uploaded as
 * gabe_upload_state does (*restored = 0): e.g. the dumps of the reference
 * harness.  restored may be NULL.  A load that fails after it began to
 * overwrite the device state leaves the handle without a state, as a failed
 * gabe_upload_state does. */
int gabe_load_state(gabe_handle *h, const char *path, int *restored);

/* Number of native |k| bins, (int)(sqrt(3) N/2 + 1) (g2spectra.cpp:31). */
int gabe_spectra_numbins(int N);

/* specOut of the current state: out is nbins x ncols, row-major, columns
 * k, P_phi, D2_phi, P_chi, D2_chi [, P_gw, Omega_gw, p] exactly as written to
 * slices_spectra_<n>.dat (g2spectra.cpp:208-230).  ncols must be 5, or 8 with
 * GWs; nbins must equal gabe_spectra_numbins(N). */
int gabe_spectra(gabe_handle *h, double *out, int nbins, int ncols);

/* Per-bin sums and counts behind gabe_spectra (weighted power sums before
 * normalisation): sums is nseries x nbins, series-major, with nseries =
 * nflds + calc_gws (phi, chi[, GW]); counts has nbins entries.  Callers can
 * rebin these exactly (e.g. into log-spaced |k| bins). */
int gabe_spectra_raw(gabe_handle *h, double *sums, double *counts, int nbins, int nseries);

/* The table of gabe_spectra from binned sums [nseries][nbins] and counts
 * [nbins] (as gabe_spectra_raw returns them, or their sums over the slabs of
 * a split lattice) and the stage-0 energy density edrho0: the reference's
 * normalisation (g2spectra.cpp:27,94-103,114-117,186-195) for p's N, L and
 * gws_on.  No device work. */
int gabe_spectra_from_sums(const gabe_params *p, double edrho0, const double *sums, const double *counts, int nbins,
                           double *out, int ncols);

/* meansvars() (g2output.cpp:70-121) of the current state without the file
 * write: out4 = {mean, variance} of each field, variance as the reference
 * forms it, sum(f^2 - mean^2)/N^3.  All four values are written; the return
 * is GABE_ERR_NONFINITE where the reference would print "Unstable solution
 * developed" and exit (a field mean with mean != 0 and mean/mean != 1).
 * Synchronises. */
int gabe_meansvars(gabe_handle *h, double out4[4]);

/* Rows that outputfield() (g2output.cpp:25-68) writes for field_outdim
 * outdim (1..3) and field_sliceskip skip: ceil(N/skip)^outdim. */
size_t gabe_field_slice_rows(int N, int outdim, int skip);

/* The rows of outputfield(): for i (stepping by skip if outdim > 2, else
 * i = 0), j (if outdim > 1, else 0) and k, in that loop order, the nflds
 * field values and calcrho(0, i, j, k) (g2functions.cpp:176-186, with the
 * fourth-order gradients of :70-98), computed on the device.  out holds
 * out_len >= 3 * gabe_field_slice_rows(N, outdim, skip) doubles, row-major.
 * Synchronises. */
int gabe_field_slice(gabe_handle *h, int outdim, int skip, double *out, size_t out_len);

/* Stage-0 energies {kin, pot, grad, rho} (calcEnergy(0)) of a state the
 * caller already holds in device memory, without allocating anything: for
 * callers that cannot allocate device memory at that point (a framework
 * whose pool allocator owns all free device memory, or code that must not
 * let cudaMalloc synchronise the device).  field0/dfield0 are device arrays
 * [nflds][N^3] of FP64, out4 a device array of 4 doubles, stream a
 * cudaStream_t (NULL = default stream); the call only enqueues work.  Uses
 * p's N, L, model and tile fields; FP64 reference arithmetic, equal to
 * gabe_energies for the same state.  Scratch is a fixed device array of
 * 32768 blocks' partial sums (about 2 MiB), held by each device that loads
 * the library until exit; a lattice needing more blocks returns
 * GABE_ERR_PARAM.  The first call on a device looks up that array's device
 * address (make it before any stream capture) and keeps it for the life of
 * the process, so the entry point must not be called after a
 * cudaDeviceReset in the same process; calls that overlap on the GPU share
 * the array and race.  Parameters are checked as gabe_create checks them
 * (GABE_ERR_PARAM, also for N % 4 != 0).  The call has no status word: a
 * state holding NaN or Inf gives NaN or Inf in out4, so check out4.  No
 * counterpart in the reference. */
int gabe_energy_noalloc(const gabe_params *p, const double *field0, const double *dfield0, double a0,
                        double *out4, void *stream);

/* Message for the last error on this handle ("" if none).  NULL handle ->
 * message of the last failed gabe_create in this thread. */
const char *gabe_last_error(const gabe_handle *h);

/* Device bytes held by the handle. */
size_t gabe_device_bytes(const gabe_handle *h);

/* Kernel launches one step enqueues (for launch accounting). */
int gabe_launches_per_step(const gabe_handle *h);

/* 1 when gabe_step replays the captured CUDA graphs of the step, 0 when it
 * launches the kernels one by one (GABE_FLAG_NO_GRAPH, or the capture
 * failed), -1 before the first gabe_step (the graphs are captured then),
 * -GABE_ERR_PARAM for a NULL handle.  No reference counterpart. */
int gabe_graph_active(const gabe_handle *h);

/* ------------------------------------------------------------------------
 * Batched ensemble: many independent lattices of uneven size, coupling,
 * fluctuation amplitude and seed, evolved together in FP32 storage with FP64
 * scalars and reductions, one persistent launch per sweep and one cuFFT call
 * per lattice size each step (replayed as a CUDA graph).  No counterpart in
 * the reference, which runs one lattice per process; each lattice follows
 * the same step() and specOut() as a gabe_handle.
 * ------------------------------------------------------------------------ */
typedef struct {
    int32_t struct_size;            /* sizeof(gabe_ensemble_params) */
    int32_t nlat;                   /* number of lattices */
    const int32_t *N;               /* [nlat] points per side; multiple of 16 */
    const double *g2_over_lambda;   /* [nlat] coupling of V = lambda phi^4/4 + g^2 phi^2 chi^2/2 */
    const double *amplitude;        /* [nlat] multiplier of the randInit amplitudes (g2init.cpp:136-143) */
    const uint64_t *seed;           /* [nlat] generator seeds */
    const int32_t *tile_shape;      /* [nlat] sites along k x j per work item: 0 = 64x8 (N%64==0),
                                       1 = 32x16 (N%32==0), 2 = 16x16; NULL = by N */
    const int32_t *tile_ci;         /* [nlat] planes per block; NULL = default */
    double L, dt;                   /* shared box side and time step */
    double lambda, phi0, dphi0;     /* shared physical model constants (program units B = sqrt(lambda) phi0) */
    int32_t gws_on;                 /* calc_gws */
    int32_t device;                 /* CUDA device, -1 = current */
    int32_t nlog;                   /* log-spaced |k| bins of gabe_ensemble_log_spectra */
    int32_t gw_spec_quirk;          /* as in gabe_params */
    int32_t flags;                  /* GABE_FLAG_NO_GRAPH */
    int32_t log_top_bin;            /* upper end of the log bins in native-bin units (0 = the native
                                       bins of the largest lattice); fix it to compare ensembles */
    /* initial-spectrum knobs of the reference's randInit (g2init.cpp:117-165), for every lattice:
       spec_cut_off > 0 multiplies each mode's amplitude by
       (1 - tanh(spec_smooth (|n| - N spec_cut_off))) / 2 (spec_cut_off, spec_smooth); 0 = none.
       ic_deterministic = 1 replaces the random draws by the real amplitude sqrt(1/(2 omega L^3))
       and fdot_k = -H0 f_k (field_full_rand 0; needs spec_cut_off > 0, as in the reference). */
    double spec_cut_off, spec_smooth;
    int32_t ic_deterministic;
    int32_t reserved;
} gabe_ensemble_params;

typedef struct gabe_ensemble gabe_ensemble;

int gabe_ensemble_create(const gabe_ensemble_params *p, gabe_ensemble **out);
int gabe_ensemble_destroy(gabe_ensemble *e);

/* Draws every lattice's initial state on the device: homogeneous values
 * phi0, dphi0 plus Gaussian random fluctuations with the reference's
 * randInit distribution (g2init.cpp:68-189; phi first, then chi with
 * m_eff^2 from the fluctuated phi), a = 1, adot from the homogeneous energy,
 * h = l = 0. */
int gabe_ensemble_init(gabe_ensemble *e);

/* Replaces lattice `lat`'s state (FP64 host arrays in the reference
 * layout; h = l = 0).  The ensemble must hold a state already
 * (gabe_ensemble_init): GABE_ERR_STATE before it. */
int gabe_ensemble_upload(gabe_ensemble *e, int lat, const double *field0, const double *dfield0, double a0,
                         double adot0);

int gabe_ensemble_step(gabe_ensemble *e, int nsteps);
int gabe_ensemble_sync(gabe_ensemble *e);

/* Per-lattice scalars, [nlat][12] in the order of gabe_scalars. */
int gabe_ensemble_scalars(gabe_ensemble *e, double *out);

/* Native |k| bins of the largest lattice: (int)(sqrt(3) Nmax/2 + 1). */
int gabe_ensemble_native_bins(const gabe_ensemble *e);

/* Log spectra of every lattice: logspec [nlat][3][nlog] = log10 of
 * (Delta^2_phi, Delta^2_chi, Omega_gw) in nlog log-spaced bins of the native
 * bin index b in [1, native_bins], each the count-weighted mean of the
 * native bins' values (g2spectra.cpp:94-103,186-195), NaN where a log bin
 * holds no native bin; counts [nlat][nlog]; native (may be NULL)
 * [nlat][4][native_bins]: the native power sums of phi, chi, GW and the
 * counts. */
int gabe_ensemble_log_spectra(gabe_ensemble *e, double *logspec, double *counts, double *native);

/* Copies lattice `lat`'s state to the host (reference layout, FP64). */
int gabe_ensemble_download(gabe_ensemble *e, int lat, double *field0, double *dfield0, double *h0, double *l0);

const char *gabe_ensemble_last_error(const gabe_ensemble *e);
size_t gabe_ensemble_device_bytes(const gabe_ensemble *e);

/* The cudaStream_t (as void *) every ensemble call enqueues on, for timing
 * with events; and the library's own kernel launches per step (cuFFT's are
 * not counted). */
void *gabe_ensemble_stream(const gabe_ensemble *e);
int gabe_ensemble_launches_per_step(const gabe_ensemble *e);

/* As gabe_graph_active, for the ensemble's step. */
int gabe_ensemble_graph_active(const gabe_ensemble *e);

/* ------------------------------------------------------------------------
 * One slab of a lattice split along i over several processes (one GPU each).
 *
 * The reference evolves one lattice in one process (step(),
 * g2functions.cpp:234-271, OpenMP over i).  A lattice larger than one GPU
 * is split into slabs of whole planes i in [plane0, plane0 + nplanes); each
 * rank creates one slab and, per step, makes the calls below, with the
 * communication between them its own (e.g. NCCL through torch.distributed):
 *
 *   gabe_slab_sweep(s, 0)     sweep A: stage-1 sums of this slab -> sums
 *   all-reduce(sums, kNV = 8 FP64 values, sum) over the ranks
 *   gabe_slab_finish(s, 0)    adot0, a[1], adot[1] from the global sums
 *   gabe_slab_sweep(s, 1)     sweep B: new state, a[0]
 *   gabe_slab_pack(s)         own boundary planes -> send_lo / send_hi
 *   exchange: send_lo -> rank below's recv_hi, send_hi -> rank above's recv_lo
 *                             (periodic in i)
 *   gabe_slab_unpack(s)       recv_lo / recv_hi -> halo planes
 *
 * After gabe_slab_upload, exchange the halos (pack, exchange, unpack) and
 * take the energies with gabe_slab_sweep(s, 2), all-reduce, and
 * gabe_slab_finish(s, 2), as calcEnergy(0) after the reference's
 * initialisation.  All calls enqueue on the slab's stream
 * (gabe_slab_stream); order the exchange after it.
 *
 * With gws_on (FP64, or FP32 with N in {64, 128, 256, 512}; the planes must be the
 * standard share of `nranks` ranks: n(r) = N/nranks + (r < N%nranks),
 * contiguous), between gabe_slab_finish(s, 0) and gabe_slab_sweep(s, 1):
 *   gabe_slab_gw_transform(s)  2-D transforms of the own source planes ->
 *                              send buffer, one block per rank
 *   all-to-all: the block for rank r (send_bytes[r]) to rank r, arriving
 *              in rank r's receive buffer at the sender's place (recv_bytes)
 *   gabe_slab_gw_update(s)     the passes along i and the TT projection +
 *                              h/l update of this rank's k-points: kx all,
 *                              ky in [plane0, plane0 + nplanes), kz all.
 * Spectra (FP64, or FP32 with N in {64, ..., 512}): gabe_slab_spectra_transform(s)
 * packs the 2-D transforms of the two fields; all-to-all the buffers of
 * gabe_slab_spectra_buffers as above; gabe_slab_spectra_raw(s, ...) bins
 * this rank's k-points (fields and, with GWs, l); add sums and counts over
 * the ranks and pass them, with edrho[0] of gabe_slab_scalars, to
 * gabe_spectra_from_sums.  No counterpart in the reference. */
typedef struct gabe_slab gabe_slab;
typedef struct {
    int32_t struct_size; /* sizeof(gabe_slab_params) */
    int32_t plane0;      /* first own plane (global index i) */
    int32_t nplanes;     /* own planes, >= 1 */
    int32_t nranks;      /* ranks of the split: needed with gws_on and for the spectra; when set,
                            [plane0, plane0 + nplanes) must be a rank's share; 0 = fields only */
} gabe_slab_params;

int gabe_slab_create(const gabe_params *p, const gabe_slab_params *sp, gabe_slab **out);
int gabe_slab_destroy(gabe_slab *s);
const char *gabe_slab_last_error(gabe_slab *s); /* NULL: the last failed create on this thread */

/* Own planes of stage 0, [2][nplanes][N][N] FP64 (the reference's layout
 * restricted to the slab).  mean = {<phi>, <chi>, <phidot>, <chidot>} of the
 * whole lattice (FP32 storage; ignored for FP64). */
int gabe_slab_upload(gabe_slab *s, const double *field0, const double *dfield0, const double mean[4], double a0,
                     double adot0);
int gabe_slab_download(gabe_slab *s, double *field0, double *dfield0);

/* Device buffers: the kNV stage sums, and the packed boundary planes (four
 * arrays phi, chi, phidot, chidot of N^2 values in the storage precision:
 * halo_bytes each). */
int gabe_slab_buffers(gabe_slab *s, double **sums, void **send_lo, void **send_hi, void **recv_lo, void **recv_hi,
                      size_t *halo_bytes);
int gabe_slab_sweep(gabe_slab *s, int which);  /* 0 sweep A, 1 sweep B, 2 energies of the current state */
int gabe_slab_finish(gabe_slab *s, int which); /* 0 after sweep A, 2 after the energies */
int gabe_slab_pack(gabe_slab *s);
int gabe_slab_unpack(gabe_slab *s);
int gabe_slab_stream(gabe_slab *s, void **stream);
int gabe_slab_sync(gabe_slab *s);
/* a, adot, edkin, edpot, edgrad, edrho, two stages each (synchronises) */
int gabe_slab_scalars(gabe_slab *s, double out12[12]);
/* GW branch: device send / receive buffers of the all-to-all and the bytes
 * per rank (arrays of nranks). */
int gabe_slab_gw_buffers(gabe_slab *s, void **send, void **recv, int64_t *send_bytes, int64_t *recv_bytes);
int gabe_slab_gw_transform(gabe_slab *s);
int gabe_slab_gw_update(gabe_slab *s);
/* h, l of this rank's k-points in the reference's component order:
 * [12][N][nplanes][N/2+1] each (ky = plane0 + y); NULL skips one. */
int gabe_slab_gw_download(gabe_slab *s, double *h0, double *l0);
int gabe_slab_spectra_transform(gabe_slab *s);
int gabe_slab_spectra_buffers(gabe_slab *s, void **send, void **recv, int64_t *send_bytes, int64_t *recv_bytes);
/* this rank's binned sums [2 + gws_on][nbins] and counts [nbins] (host arrays; synchronises) */
int gabe_slab_spectra_raw(gabe_slab *s, double *sums, double *counts);

#ifdef __cplusplus
}
#endif

#endif
