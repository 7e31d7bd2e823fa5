// Host-side launch entry points of the precision-specific kernel units.
// kernels_f64.cu is compiled without FMA contraction so that the FP64 path
// rounds every operation as the reference's x86-64 build does;
// kernels_f32.cu is compiled with contraction on.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "../../include/gabe.h"
#include "kspace.cuh"
#include "output.cuh"
#include "spectra.cuh"
#include "stencil.cuh"

namespace gabe {

struct Launch {
    dim3 grid, block;
    size_t smem;
    cudaStream_t stream;
};

// Stencil tile shapes (TK x TJ), index = tile shape id of gabe_params.
constexpr int kNumShapes = 6;
constexpr int kShapes[kNumShapes][2] = {{32, 8}, {16, 16}, {32, 4}, {16, 8}, {8, 8}, {4, 4}};

// Constants with the operation sequence the reference's compiler folds
// (g2parameters.h:93, g2functions.cpp:41, g2evolutionpert.cpp:53,198,486-487,
// g2model.cpp:64,68).
inline LatticeConsts make_lattice_consts(const gabe_params &p) {
    LatticeConsts c{};
    c.N = p.N;
    c.model = p.model;
    c.expansion = p.expansion;
    const double L = p.L, dt = p.dt;
    const double dx = L / ((double)p.N);
    c.dx = dx;
    c.dt = dt;
    c.half_dt = .5 * dt;
    c.inv_dx2_div = dx * dx;
    c.dn = (double)(1 / (dx * dx));
    c.c13 = (1. / 3.) * c.dn;
    c.c23 = (2. / 3.) * c.dn;
    if (p.model == GABE_MODEL_QUADRATIC) {
        const double mphi = p.model_c[0], gsq = p.model_c[1];
        c.mc[0] = gsq / mphi / mphi;
        c.mc[1] = 0.5 * gsq / mphi / mphi;
    } else {
        const double lam = p.model_c[0], g = p.model_c[1];
        c.mc[0] = lam;
        c.mc[1] = g;
        c.mc[2] = 0.25 * lam;
        c.mc[3] = 0.5 * g;
        c.mc[4] = 3. * lam;
    }
    c.gridsize = (double)((long long)p.N * p.N * p.N);
    c.eight_pi_3 = 8. * M_PI / 3.;
    c.k2norm_c = 4. * M_PI * M_PI / L / L;
    c.eight_pi = 8. * M_PI;
    c.normmm = pow(dx, 3);
    return c;
}

// Stencil grid: tile shape (the requested one if it divides N, else the first
// in kShapes that does) and planes per block, shrunk until the grid has at
// least 8 blocks per SM of a 148-SM B200.  shape = -1 (and an empty grid)
// when no tile shape divides N.
struct GridPlan {
    int shape, ci;
    dim3 grid;
};
inline GridPlan plan_grid(int N, int want_shape, int want_ci) {
    auto fits = [N](int s) {
        const int tk = kShapes[s][0], tj = kShapes[s][1];
        return tk <= N && tj <= N && N % tk == 0 && N % tj == 0;
    };
    int shape = (want_shape >= 0 && want_shape < kNumShapes && fits(want_shape)) ? want_shape : -1;
    for (int q = 0; shape < 0 && q < kNumShapes; q++)
        if (fits(q)) shape = q;
    if (shape < 0) return GridPlan{-1, 0, dim3(0, 0, 0)};  // no tile divides N (N % 4 != 0)
    const int TK = kShapes[shape][0], TJ = kShapes[shape][1];
    const int bxy = (N / TK) * (N / TJ);
    int ci = want_ci > 0 ? want_ci : N;
    if (want_ci <= 0)
        while (ci > 4 && (long long)bxy * ((N + ci - 1) / ci) < 8 * 148) ci /= 2;
    if (ci > N) ci = N;
    return GridPlan{shape, ci, dim3(N / TK, N / TJ, (N + ci - 1) / ci)};
}

// FP32 sweeps (sweep32.cuh): tile shapes (TK x TJ), two sites per thread along k.
constexpr int kNumShapes32 = 7;
constexpr int kShapes32[kNumShapes32][2] = {{64, 8}, {64, 4}, {128, 4}, {32, 8}, {64, 16}, {32, 4}, {16, 8}};

inline GridPlan plan_grid32(int N, int want_shape, int want_ci) {
    auto fits = [N](int s) {
        const int tk = kShapes32[s][0], tj = kShapes32[s][1];
        return tk <= N && tj <= N && N % tk == 0 && N % tj == 0;
    };
    int shape = (want_shape >= 0 && want_shape < kNumShapes32 && fits(want_shape)) ? want_shape : -1;
    // 128 x 4 columns at 512^3: sweep A 1.69 ms against 1.81 for 64 x 8 (sweep B 0.84 against 0.83)
    if (shape < 0 && N == 512 && fits(2)) shape = 2;
    for (int q = 0; shape < 0 && q < kNumShapes32; q++)
        if (fits(q)) shape = q;
    if (shape < 0) return GridPlan{-1, 0, dim3(0, 0, 0)};  // no tile divides N (N % 16 != 0)
    const int TK = kShapes32[shape][0], TJ = kShapes32[shape][1];
    const int bxy = (N / TK) * (N / TJ);
    // planes per block: N / 8 from N = 128 on (the fastest measured at 128^3, 256^3 and 512^3: 64 planes at
    // 512^3 ran sweep A 1.69-1.81 ms against 1.97 with 128); below, enough blocks for four per SM
    int ci = want_ci > 0 ? want_ci : (N >= 128 ? N / 8 : N);
    if (want_ci <= 0 && N < 128)
        while (ci > 4 && (long long)bxy * ((N + ci - 1) / ci) < 4 * 148) ci /= 2;
    if (ci > N) ci = N;
    return GridPlan{shape, ci, dim3(N / TK, N / TJ, (N + ci - 1) / ci)};
}

// Checks of gabe_params shared by gabe_create and gabe_energy_noalloc; false
// with a message in msg when p is invalid.  The stencil tiling is checked
// separately (plan_grid / plan_grid32 return shape -1).
inline bool params_valid(const gabe_params &p, char *msg, size_t n) {
    auto fail = [&](const char *m) {
        if (msg && n) {
            size_t i = 0;
            for (; m[i] && i + 1 < n; i++) msg[i] = m[i];
            msg[i] = 0;
        }
        return false;
    };
    if (p.struct_size != (int32_t)sizeof(gabe_params)) return fail("struct_size differs from sizeof(gabe_params)");
    if (p.N < 4 || p.N > 1290 || (p.N & 1)) return fail("N must be even and in [4, 1290]");
    if (p.nflds != 2) return fail("nflds must be 2");
    if (p.expansion < 0 || p.expansion > 2) return fail("expansion_type must be 0, 1 or 2");
    if (p.gws_on != 0 && p.gws_on != 1) return fail("calc_gws must be 0 or 1");
    if (p.model != GABE_MODEL_QUADRATIC && p.model != GABE_MODEL_LPHI4) return fail("unknown model");
    if (p.precision != GABE_FP64 && p.precision != GABE_FP32) return fail("unknown precision");
    if (!(p.L > 0) || !(p.dt > 0) || !std::isfinite(p.L) || !std::isfinite(p.dt))
        return fail("L and dt must be positive and finite");
    if (!std::isfinite(p.model_c[0]) || !std::isfinite(p.model_c[1]) ||
        (p.model == GABE_MODEL_QUADRATIC && p.model_c[0] == 0.0))
        return fail("invalid model constants (non-finite, or mphi = 0 for the quadratic model)");
    return true;
}

cudaError_t sweep_f64(int shape, int mode, const StencilArgs &a, dim3 grid, cudaStream_t s);
cudaError_t sweep32_f32(int shape, int mode, const StencilArgs &a, dim3 grid, cudaStream_t s);
// Slab: finish_a of sweep A (mode MODE_A) or of the energies (MODE_E0) from the totals of all slabs.
cudaError_t slab_finish_f32(int mode, const LatticeConsts &c, DevScalars *sc, const double *tot, cudaStream_t s);
cudaError_t slab_finish_f64(int mode, const LatticeConsts &c, DevScalars *sc, const double *tot, cudaStream_t s);
// Slab GW branch, FP32 (slabgw.cuh): pack the 2-D transforms for the all-to-all, unpack what
// arrived into [10][N][m][nz], the k-space update of the rank's k-points, amplitudes -> 12 components.
cudaError_t slab_kspace_f32(const void *T, void *G, const DevScalars *sc, const LatticeConsts &c, int m, int y0,
                            cudaStream_t s);
cudaError_t slab_gw_amplitudes_f32(const void *G, size_t cnt, size_t m0, int N, int m, int y0, int which, double *dst,
                                   cudaStream_t s);
cudaError_t slab_gw_pack_f64(const void *S, void *send, int N, int nloc, int W, int ncomp, cudaStream_t s);
cudaError_t slab_gw_unpack_f64(const void *recv, void *T, int N, int m, int W, int ncomp, cudaStream_t s);
cudaError_t slab_kspace_f64(const void *T, void *G, const DevScalars *sc, const LatticeConsts &c, int m, int y0,
                            cudaStream_t s);
cudaError_t slab_gw_amplitudes_f64(const void *G, size_t cnt, size_t m0, int N, int m, int y0, int which, double *dst,
                                   cudaStream_t s);
cudaError_t kspace_f64(const KspaceArgs &a, const Launch &l);
cudaError_t kspace_f32(const KspaceArgs &a, const Launch &l);
cudaError_t bins_f64(const BinArgs &a, const Launch &l);
cudaError_t bins_f32(const BinArgs &a, const Launch &l);
cudaError_t configure_bins(size_t max_smem);
cudaError_t gw_pack_f64(const double *src, size_t cnt, size_t m0, int N, size_t M, void *G, int which, double *norms,
                        cudaStream_t s);
// gt = 1: G in the transposed order [..][kz][j][i] of the transposed transform (fftt.cuh)
cudaError_t gw_pack_f32(const double *src, size_t cnt, size_t m0, int N, size_t M, void *G, int which, double *norms,
                        int gt, cudaStream_t s);
cudaError_t gw_unpack_f64(const void *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst, cudaStream_t s);
cudaError_t gw_unpack_f32(const void *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst, int gt,
                          cudaStream_t s);

// meansvars() and outputfield() rows on the device (output.cuh)
cudaError_t meansvars_f64(const OutArgs &a, int pass, int nblocks, cudaStream_t s);
cudaError_t meansvars_f32(const OutArgs &a, int pass, int nblocks, cudaStream_t s);
cudaError_t slice_f64(const OutArgs &a, int nj, int nk, int skip, size_t r0, size_t cnt, double *out, cudaStream_t s);
cudaError_t slice_f32(const OutArgs &a, int nj, int nk, int skip, size_t r0, size_t cnt, double *out, cudaStream_t s);

cudaError_t mean_f64(const double *x, size_t n, double *partials, unsigned int *counter, double *out, int nblocks,
                     cudaStream_t s);
cudaError_t to_fluct(const double *x, size_t n, const double *mean, float *out, cudaStream_t s);
cudaError_t from_fluct(const float *x, size_t n, const double *mean, double *out, cudaStream_t s);

// FP32 3-D r2c of ncomp arrays [N][N][N+2] in three passes (fft3d.cuh), result in S;
// T (S's size, or null for in place) is the target of the pass along j, read by the pass along i.
bool fft3d_supported(int N);
cudaError_t fft3d_r2c_f32(int N, float *S, float *T, int ncomp, cudaStream_t s);
// One of its passes: 0 rows along k, 1 along j, 2 along i.
cudaError_t fft3d_pass_f32(int N, float *S, float *T, int ncomp, int pass, cudaStream_t s);
// One column pass (fft3d.cuh col_fft_kernel): for b1 < n1, b2 < n2, c < ncol the N complex
// values at X + b1 s1 + b2 s2 + n sn + c.
cudaError_t fft_col_pass_f32(int N, void *X, long long s1, long long s2, long long sn, int n1, int n2, int ncol,
                             cudaStream_t s);
// The pass along i of a slab transpose's receive buffer (blocks by source rank of
// [ncomp][n(r)][m][N/2+1]) into T[ncomp][N][m][N/2+1], out of place (fft3d.cuh).
cudaError_t fft_col_gather_f32(int N, const void *recv, void *T, int ncomp, int m, int ranks, cudaStream_t s);
// 2-D r2c over (j, k) of nplanes planes [N][N+2] of S (rows transformed in place), the
// pass along j written to the transpose's send buffer (blocks by destination rank of
// [nplanes][n(r)][N/2+1]), for N in {64, 128, 256, 512} (fft3d.cuh).
cudaError_t fft_plane_scatter_f32(int N, float *S, void *send, int nplanes, int ranks, cudaStream_t s);

// FP32 transposed three-pass transform (fftt.cuh): rows along k S -> T1, the pass
// along j T1 -> T2, and the pass along i fused with the TT projection and h/l
// update of the amplitudes G (kept in the transposed order [4][kz][ky][kx]).
bool fftt_supported(int N);
cudaError_t fftt_rows_f32(int N, const float *S, void *T1, int ncomp, unsigned int *status, cudaStream_t s);
cudaError_t fftt_cols_f32(int N, const void *T1, void *T2, int ncomp, unsigned int *status, cudaStream_t s);
cudaError_t fftt_ikspace_f32(int N, const void *T2, void *G, const DevScalars *sc, const LatticeConsts &c, int slot,
                             unsigned int *status, cudaStream_t s);

cudaError_t bin_reduce(const double *part_sum, const unsigned int *part_cnt, int nblocks, int nseries, int nbins,
                       double *sum, double *cnt, cudaStream_t s);

}  // namespace gabe
