/*
 * gabe_dropin.cpp -- GABE's step(), specOut(), specClear() and
 * outputslice() on top of the B200 library (include/gabe.h).
 *
 * Compiled inside a GABE source tree (it includes that tree's g2header.h and
 * g2parameters.h) together with the unmodified g2main.cpp, g2init.cpp, model
 * file and g2evolutionpert.cpp, and with g2functions.cpp, g2spectra.cpp and
 * g2output.cpp built with -Dstep=gabe_reference_cpu_step,
 * -DspecOut=gabe_reference_specOut -DspecClear=gabe_reference_specClear and
 * -Doutputslice=gabe_reference_outputslice so that these definitions take
 * the driver's calls (g2main.cpp:122,126,129,335).
 *
 * State ownership follows the reference: the host arrays stay the
 * program's; the device copy is made once, after the reference's own
 * initialisation (g2main.cpp:111-118), and the per-stage scalars are copied
 * back after every step (96 bytes).  The output slices need no state
 * download: the field-slice rows with calcrho (outputfield), the means and
 * variances (meansvars) and the spectra (specOut) are computed on the
 * device and only the printed numbers cross to the host.
 *
 * Knobs (compile-time, like the rest of GABE):
 *   GABE_B200_MODEL      0: the shipped model (g2model.cpp; constants mphi,
 *                        gsq from g2parameters.h), 1: lambda phi^4 in program
 *                        units with constants lam_pr, gsq_pr
 *   GABE_B200_PRECISION  0: FP64 (default), 1: FP32 fluctuation storage
 *   fftw_flag (the tree's g2parameters.h) 1: long double host arrays; the
 *                        state crosses the boundary as doubles, the device
 *                        computes in FP64, and the files are printed with
 *                        %Le as the reference prints them
 *
 * Checkpoint and restart (run-time, environment; the reference has neither):
 *   GABE_B200_CHECKPOINT_EVERY=n and GABE_B200_CHECKPOINT=<file> write a
 *   checkpoint (gabe_save_state) every n steps; a %d in <file> takes the
 *   step count.
 *   GABE_B200_RESTART=<file> starts from such a file -- or any gabe_dump.h
 *   dump of this lattice -- instead of the state the reference's
 *   initialisation made, and sets t to starttime + step * dt of the dump,
 *   so the run continues the saved one (bit for bit from a checkpoint of
 *   the same build and precision).
 */
#include <cstdlib>
#include <string>
#include <vector>

#include "gabe.h"
#include "gabe_dump.h"
#include "g2header.h"

#ifndef GABE_B200_MODEL
#define GABE_B200_MODEL 0
#endif
#ifndef GABE_B200_PRECISION
#define GABE_B200_PRECISION 0
#endif

namespace {

gabe_handle *g_gpu = nullptr;
long g_steps = 0;

void gabe_die(const char *what, int rc)
{
    fprintf(stderr, "gabe_b200: %s failed (status %d): %s\n", what, rc, gabe_last_error(g_gpu));
    exit(1);
}

void pull_scalars()
{
    double s[12];
    int rc = gabe_scalars(g_gpu, s);
    if (rc != GABE_OK) gabe_die("gabe_scalars", rc);
    for (int q = 0; q < 2; q++) {
        a[q] = s[q]; adot[q] = s[2 + q]; edkin[q] = s[4 + q];
        edpot[q] = s[6 + q]; edgrad[q] = s[8 + q]; edrho[q] = s[10 + q];
    }
}

void ensure_device_state()
{
    if (g_gpu) return;
    gabe_params p;
    gabe_default_params(&p, N);
    p.nflds = nflds;
    p.gws_on = calc_gws;
    p.expansion = expansion_type;
    p.L = L;
    p.dt = dt;
    p.precision = GABE_B200_PRECISION;
#if GABE_B200_MODEL == 0
    p.model = GABE_MODEL_QUADRATIC;
    p.model_c[0] = mphi;
    p.model_c[1] = gsq;
#else
    p.model = GABE_MODEL_LPHI4;
    p.model_c[0] = lam_pr;
    p.model_c[1] = gsq_pr;
#endif
    int rc = gabe_create(&p, &g_gpu);
    if (rc != GABE_OK) {
        fprintf(stderr, "gabe_b200: gabe_create failed (status %d): %s\n", rc, gabe_last_error(nullptr));
        exit(1);
    }
    const char *restart = getenv("GABE_B200_RESTART");
    if (restart && *restart) {
        int restored = 0;
        rc = gabe_load_state(g_gpu, restart, &restored);
        if (rc != GABE_OK) gabe_die("gabe_load_state", rc);
        gabe_dump_header hd;
        FILE *f = fopen(restart, "rb");
        if (!f || fread(&hd, sizeof(hd), 1, f) != 1) {
            fprintf(stderr, "gabe_b200: cannot read the header of %s\n", restart);
            exit(1);
        }
        fclose(f);
        t = starttime + (gNum)hd.step * dt;
        g_steps = (long)hd.step;
        pull_scalars();
        printf("gabe_b200: %s %s at step %lld, t = %e\n", restored ? "restarted from" : "initial state from", restart,
               (long long)hd.step, (double)t);
        return;
    }
#if fftw_flag == 1
    // long double host arrays: the library computes in FP64, so the state
    // crosses the boundary as doubles
    const size_t nf = (size_t)nflds * N * N * N;
    std::vector<double> f0(nf), d0(nf), hv, lv;
    const gNum *fs = &field[0][0][0][0][0], *ds = &dfield[0][0][0][0][0];
    for (size_t q = 0; q < nf; q++) {
        f0[q] = (double)fs[q];
        d0[q] = (double)ds[q];
    }
#if calc_gws == 1
    const size_t ng = (size_t)12 * N * N * (N / 2 + 1);
    hv.resize(ng);
    lv.resize(ng);
    const gNum *hs = &h[0][0][0][0][0], *ls = &l[0][0][0][0][0];
    for (size_t q = 0; q < ng; q++) {
        hv[q] = (double)hs[q];
        lv[q] = (double)ls[q];
    }
#endif
    rc = gabe_upload_state(g_gpu, f0.data(), d0.data(), hv.empty() ? nullptr : hv.data(),
                           lv.empty() ? nullptr : lv.data(), (double)a[0], (double)adot[0]);
#else
    const double *h0 = nullptr, *l0 = nullptr;
#if calc_gws == 1
    h0 = &h[0][0][0][0][0];
    l0 = &l[0][0][0][0][0];
#endif
    rc = gabe_upload_state(g_gpu, &field[0][0][0][0][0], &dfield[0][0][0][0][0], h0, l0, a[0], adot[0]);
#endif
    if (rc != GABE_OK) gabe_die("gabe_upload_state", rc);
}

#if field_outdim != 0
// outputfield(first) (g2output.cpp:25-68): the same rows and format, computed
// on the device (gabe_field_slice).
void device_outputfield(int first)
{
    ensure_device_state();
    const size_t rows = gabe_field_slice_rows(N, field_outdim, field_sliceskip);
    double *buf = (double *)malloc(sizeof(double) * 3 * rows);
    if (!buf) {
        fprintf(stderr, "gabe_b200: host allocation failed\n");
        exit(1);
    }
    int rc = gabe_field_slice(g_gpu, field_outdim, field_sliceskip, buf, 3 * rows);
    if (rc != GABE_OK) gabe_die("gabe_field_slice", rc);
    char name[64];
    snprintf(name, sizeof(name), "./slices/slices_fields_%d.dat", first);
    FILE *f = fopen(name, "w");
    if (!f) {
        fprintf(stderr, "gabe_b200: cannot open %s\n", name);
        exit(1);
    }
    for (size_t r = 0; r < rows; r++) {
        for (int c = 0; c < 3; c++) {
#if fftw_flag == 1
            fprintf(f, "%Le ", (long double)buf[3 * r + c]);
#else
            fprintf(f, "%e ", buf[3 * r + c]);
#endif
        }
        fprintf(f, "\n");
    }
    fclose(f);
    free(buf);
}
#endif

#if var_output != 0
// meansvars() (g2output.cpp:70-121): the same line of meansvariances.dat and
// the same stop on a non-numerical field mean, from gabe_meansvars.
void device_meansvars()
{
    ensure_device_state();
    double mv[4];
    int rc = gabe_meansvars(g_gpu, mv);
    if (rc != GABE_OK && rc != GABE_ERR_NONFINITE) gabe_die("gabe_meansvars", rc);
    FILE *out = fopen("./slices/meansvariances.dat", "a");
#if fftw_flag == 1
    fprintf(out, "%Lf", t);
#else
    fprintf(out, "%f", t);
#endif
    for (int fld = 0; fld < nflds; fld++) {
        const double av = mv[2 * fld], var = mv[2 * fld + 1];
#if fftw_flag == 1
        fprintf(out, " %Le %Le", (long double)av, (long double)var);
#else
        fprintf(out, " %e %e", av, var);
#endif
        if (av != 0. && av / av != 1.) {
#if fftw_flag == 1
            printf("Unstable solution developed. Field %d not numerical at t=%Le\n", fld, t);
#else
            printf("Unstable solution developed. Field %d not numerical at t=%e\n", fld, t);
#endif
            output_parameters();
            fflush(out);
            exit(1);
        }
    }
    fprintf(out, "\n");
    fclose(out);
}
#endif

}  // namespace

void step()
{
    ensure_device_state();
    int rc = gabe_step(g_gpu, 1);
    if (rc != GABE_OK) gabe_die("gabe_step", rc);
    g_steps++;
    pull_scalars();
    static const char *every_s = getenv("GABE_B200_CHECKPOINT_EVERY"), *path = getenv("GABE_B200_CHECKPOINT");
    static const long every = every_s ? atol(every_s) : 0;
    if (every > 0 && path && *path && g_steps % every == 0) {
        std::string name(path);
        const size_t at = name.find("%d");
        if (at != std::string::npos) name.replace(at, 2, std::to_string(g_steps));
        rc = gabe_save_state(g_gpu, name.c_str());
        if (rc != GABE_OK) gabe_die("gabe_save_state", rc);
    }
}

// outputslice() (g2output.cpp:129-186): the same cadence, the same files in
// the same order, with the field slice and means/variances from the device.
void outputslice()
{
    static FILE *slicetime;
    static int first = 0;
    static int lastslice, lastspec;
    static int slicewaitm;
    ensure_device_state();  // a restart sets t before the first row is written
    if (first == 0) {
        slicewaitm = slicewait == 0 ? slicewaitf() : slicewait;
        lastslice = slicewaitm;
        lastspec = specnumber;
    }
    lastslice++;
    if (lastslice < slicewaitm) return;
#if field_outdim != 0
    device_outputfield(first);
#endif
#if spec_output == 1
    lastspec++;
    if (lastspec >= specnumber) {
        specOut(first / specnumber);
        lastspec = 0;
    }
#endif
#if var_output != 0
    device_meansvars();
#endif
    slicetime = fopen("./slices/slices_time.dat", "a");
#if fftw_flag == 1
    fprintf(slicetime, "%Le %Le %Le %Le %Le %Le %Le %Le\n", t, a[0], adot[0], adot[0] / a[0], edkin[0], edpot[0],
            edgrad[0], edrho[0]);
#else
    fprintf(slicetime, "%e %e %e %e %e %e %e %e\n", t, a[0], adot[0], adot[0] / a[0], edkin[0], edpot[0], edgrad[0],
            edrho[0]);
#endif
    fclose(slicetime);
    first++;
    lastslice = 0;
}

#if spec_output == 1
void specOut(int first)
{
    ensure_device_state();
    const int nb = gabe_spectra_numbins(N);
    const int nc = calc_gws == 1 ? 8 : 5;
    double *tab = (double *)malloc(sizeof(double) * nb * nc);
    int rc = gabe_spectra(g_gpu, tab, nb, nc);
    if (rc != GABE_OK) gabe_die("gabe_spectra", rc);
    char name[64];
    snprintf(name, sizeof(name), "./slices/slices_spectra_%d.dat", first);
    FILE *f = fopen(name, "w");
    if (!f) {
        fprintf(stderr, "gabe_b200: cannot open %s\n", name);
        exit(1);
    }
    for (int b = 0; b < nb; b++) {
#if fftw_flag == 1
        fprintf(f, "%Le", (long double)tab[b * nc]);
        for (int c = 1; c < nc; c++) fprintf(f, " %Le", (long double)tab[b * nc + c]);
#else
        fprintf(f, "%e", tab[b * nc]);
        for (int c = 1; c < nc; c++) fprintf(f, " %e", tab[b * nc + c]);
#endif
        fprintf(f, "\n");
    }
    fclose(f);
    free(tab);
}

void specClear()
{
    gabe_destroy(g_gpu);
    g_gpu = nullptr;
}
#endif
