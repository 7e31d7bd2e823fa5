/*
 * gabe_dropin.cpp -- GABE's step(), specOut() and specClear() on top of the
 * B200 library (include/gabe.h).
 *
 * Compiled inside a GABE source tree (it includes that tree's g2header.h and
 * g2parameters.h) together with the unmodified g2main.cpp, g2output.cpp,
 * g2init.cpp, model file and g2evolutionpert.cpp, and with g2functions.cpp
 * and g2spectra.cpp built with -Dstep=gabe_reference_cpu_step and
 * -DspecOut=gabe_reference_specOut -DspecClear=gabe_reference_specClear so
 * that these definitions take the driver's calls (g2main.cpp:126,
 * g2output.cpp:161, g2main.cpp:335).
 *
 * State ownership follows the reference: the host arrays stay the
 * program's; the device copy is made once, after the reference's own
 * initialisation (g2main.cpp:111-118), and the host mirrors are refreshed
 * as the output code needs them -- the per-stage scalars after every step,
 * field[0]/dfield[0] on the steps where outputslice() writes
 * (g2output.cpp:136-149).  Spectra are computed on the device.
 *
 * Knobs (compile-time, like the rest of GABE):
 *   GABE_B200_MODEL      0: the shipped model (g2model.cpp; constants mphi,
 *                        gsq from g2parameters.h), 1: lambda phi^4 in program
 *                        units with constants lam_pr, gsq_pr
 *   GABE_B200_PRECISION  0: FP64 (default), 1: FP32 fluctuation storage
 */
#include "gabe.h"
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
    const double *h0 = nullptr, *l0 = nullptr;
#if calc_gws == 1
    h0 = &h[0][0][0][0][0];
    l0 = &l[0][0][0][0][0];
#endif
    rc = gabe_upload_state(g_gpu, &field[0][0][0][0][0], &dfield[0][0][0][0][0], h0, l0, a[0], adot[0]);
    if (rc != GABE_OK) gabe_die("gabe_upload_state", rc);
}

// outputslice() writes after the n-th step when n is a multiple of its
// wait (g2output.cpp:136-149); the first call at t = starttime always writes.
bool output_due(long n)
{
    const int w = slicewait == 0 ? (int)(endtime / dt / slicenumber) : slicewait;
    return w <= 1 || n % w == 0;
}

}  // namespace

void step()
{
    ensure_device_state();
    int rc = gabe_step(g_gpu, 1);
    if (rc != GABE_OK) gabe_die("gabe_step", rc);
    g_steps++;
    pull_scalars();
    if (output_due(g_steps)) {
        rc = gabe_download_state(g_gpu, &field[0][0][0][0][0], &dfield[0][0][0][0][0], nullptr, nullptr);
        if (rc != GABE_OK) gabe_die("gabe_download_state", rc);
    }
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
        fprintf(f, "%e", tab[b * nc]);
        for (int c = 1; c < nc; c++) fprintf(f, " %e", tab[b * nc + c]);
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
