/*
 * gabe_dump.h -- binary state dump / checkpoint format.
 *
 * The reference has no restartable output: its field slices are %e text of
 * a sampled plane (g2output.cpp:25-68).  This format carries the full FP64
 * state that the reference's step() reads and writes -- field[0] and
 * dfield[0] (g2header.h:54-55), h[0] and l[0] (g2header.h:171-172), and the
 * per-stage scalars a, adot, edkin, edpot, edgrad, edrho (g2header.h:58-63)
 * -- so that the reference build, the oracle and the CUDA library can all
 * start from the same initial state and be compared at any step.
 *
 * Layout (little endian): a 256-byte header, then
 *   field[0]  nflds*N^3 doubles, index [fld][i][j][k], k fastest
 *   dfield[0] same
 *   if gws:  h[0] 12*N*N*(N/2+1) doubles, index [comp][i][j][kz]
 *            l[0] same
 * The 12 GW components are (re,im) pairs of 11,12,13,22,23,33 in the order
 * the reference stores them (g2evolutionpert.cpp:216-310, 406-431).
 */
#ifndef GABE_DUMP_H
#define GABE_DUMP_H

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GABE_DUMP_MAGIC "GABEDMP1"
#define GABE_DUMP_VERSION 1

typedef struct {
    char magic[8];
    int32_t version;
    int32_t N;
    int32_t nflds;
    int32_t gws;
    int32_t elem_bytes;
    int32_t model;
    int64_t step;
    double t, L, dt;
    double a[2], adot[2], edkin[2], edpot[2], edgrad[2], edrho[2];
    char reserved[96];
} gabe_dump_header;

typedef char gabe_dump_header_is_256_bytes[(sizeof(gabe_dump_header) == 256) ? 1 : -1];

static inline void gabe_dump_header_init(gabe_dump_header *h, int N, int nflds, int gws,
                                         int elem_bytes, int model)
{
    memset(h, 0, sizeof(*h));
    memcpy(h->magic, GABE_DUMP_MAGIC, 8);
    h->version = GABE_DUMP_VERSION;
    h->N = N;
    h->nflds = nflds;
    h->gws = gws;
    h->elem_bytes = elem_bytes;
    h->model = model;
}

static inline size_t gabe_dump_field_count(int N, int nflds)
{
    return (size_t)nflds * (size_t)N * (size_t)N * (size_t)N;
}

static inline size_t gabe_dump_gw_count(int N)
{
    return (size_t)12 * (size_t)N * (size_t)N * (size_t)(N / 2 + 1);
}

/* arrays: {field0, dfield0, h0, l0}; h0/l0 ignored unless hd->gws. */
static inline int gabe_dump_write(const char *path, const gabe_dump_header *hd,
                                  const double *const arrays[4])
{
    FILE *f = fopen(path, "wb");
    if (!f) return 1;
    int bad = fwrite(hd, sizeof(*hd), 1, f) != 1;
    size_t nf = gabe_dump_field_count(hd->N, hd->nflds);
    size_t ng = gabe_dump_gw_count(hd->N);
    for (int a = 0; a < 4 && !bad; a++) {
        size_t n = a < 2 ? nf : ng;
        if (a >= 2 && !hd->gws) break;
        bad = fwrite(arrays[a], sizeof(double), n, f) != n;
    }
    if (fclose(f) != 0) bad = 1;
    return bad;
}

/* Reads a dump whose N/nflds/gws must equal the caller's.  Returns 0 on
 * success.  If the file has GW arrays but the caller passes NULL for them,
 * they are skipped. */
static inline int gabe_dump_read(const char *path, gabe_dump_header *hd, double *const arrays[4],
                                 int N, int nflds, int gws)
{
    FILE *f = fopen(path, "rb");
    if (!f) return 1;
    int bad = fread(hd, sizeof(*hd), 1, f) != 1;
    if (!bad) bad = memcmp(hd->magic, GABE_DUMP_MAGIC, 8) != 0 || hd->version != GABE_DUMP_VERSION ||
                    hd->N != N || hd->nflds != nflds || hd->elem_bytes != 8 || (gws && !hd->gws);
    size_t nf = gabe_dump_field_count(N, nflds);
    size_t ng = gabe_dump_gw_count(N);
    for (int a = 0; a < 4 && !bad; a++) {
        size_t n = a < 2 ? nf : ng;
        if (a >= 2 && !hd->gws) break;
        if (arrays[a]) bad = fread(arrays[a], sizeof(double), n, f) != n;
        else bad = fseek(f, (long)(n * sizeof(double)), SEEK_CUR) != 0;
    }
    fclose(f);
    return bad;
}

/* Restart block.  A checkpoint written by the library (gabe_save_state)
 * is a dump as above -- any reader of the format takes its FP64 arrays --
 * followed by this header, the library's device scalar block
 * (scalar_bytes bytes), and the device arrays as the library holds them:
 * field and momenta of stage 0 (field_bytes each: FP64 values, or for
 * FP32 storage the FP32 fluctuations about the homogeneous trajectory kept
 * in the scalar block) and, with GWs, the four TT amplitudes h+, hx, l+,
 * lx (gw_bytes; complex, [4][i][j][kz] for gw_layout 0 or [4][kz][j][i]
 * for gw_layout 1).  Loading the block into a handle of the same precision,
 * amplitude layout and tile plan continues the run bit for bit. */
#define GABE_RESTART_MAGIC "GABERST1"

typedef struct {
    char magic[8];
    int32_t precision;      /* enum gabe_precision of the writer */
    int32_t gw_layout;      /* 0 [4][i][j][kz], 1 [4][kz][j][i] */
    int32_t expansion;
    int32_t tile_shape, tile_ci;
    int32_t e0_stale;       /* the stage-0 energies of the scalar block were not yet reduced */
    int32_t scalar_bytes;
    int32_t elem_bytes;     /* 8 FP64, 4 FP32 storage */
    int64_t field_bytes, gw_bytes;
    char reserved[72];
} gabe_restart_header;

typedef char gabe_restart_header_is_128_bytes[(sizeof(gabe_restart_header) == 128) ? 1 : -1];

#ifdef __cplusplus
}
#endif

#endif
