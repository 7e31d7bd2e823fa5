// Device-side output quantities: the field means and variances of
// meansvars() (g2output.cpp:70-121) and the field-slice rows of
// outputfield() (g2output.cpp:25-68) with calcrho() (g2functions.cpp:176-186)
// and its fourth-order gradients dfdi/dfdj/dfdk (:70-98), so that an output
// step needs no download of the state.
//
// FP64 storage keeps the reference's operation order (the FP64
// instantiations are compiled without FMA contraction).  FP32 storage holds
// fluctuations d about the homogeneous values fbar: a field value is
// fbar + d, its gradient that of d (the constant cancels), and its variance
// sum (f^2 - av^2) = sum (d - dbar)(2 fbar + d + dbar) without cancellation.
#pragma once

#include "common.cuh"

namespace gabe {

struct OutArgs {
    const void *X, *D;  // fields and momenta of the current stage 0, [2][N^3]
    const DevScalars *sc;
    LatticeConsts c;
    double *partials;  // >= gridDim.x * 2 doubles
    unsigned int *counter;
    double *res;  // [8]: av[2], var[2], FP32: mean fluctuation[2]
};

template <typename T>
__device__ __forceinline__ double field_value(const OutArgs &a, int fld, size_t x) {
    const T *X = static_cast<const T *>(a.X);
    if constexpr (sizeof(T) == 8) return X[(size_t)fld * a.c.N * a.c.N * a.c.N + x];
    else return a.sc->fbar[fld] + (double)X[(size_t)fld * a.c.N * a.c.N * a.c.N + x];
}

// pass 0: av = sum f / N^3; pass 1: var = sum (f f - av av) / N^3, per field
template <typename T>
__global__ void __launch_bounds__(256) meansvars_kernel(OutArgs a, int pass) {
    __shared__ double sred[8 * 2];
    __shared__ int sflag;
    const size_t n3 = (size_t)a.c.N * a.c.N * a.c.N;
    const T *X = static_cast<const T *>(a.X);
    double acc[2] = {0., 0.};
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const T *x = X + f * n3;
        double av = 0., fb = 0., db = 0.;
        if (pass == 1) {
            av = a.res[f];
            if constexpr (sizeof(T) == 4) {
                fb = a.sc->fbar[f];
                db = a.res[4 + f];
            }
        }
        double s = 0.;
        for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n3; q += (size_t)gridDim.x * blockDim.x) {
            const double v = (double)x[q];
            if (pass == 0) s += v;
            else if constexpr (sizeof(T) == 8) s += v * v - av * av;  // g2output.cpp:98
            else s += (v - db) * (2. * fb + v + db);
        }
        acc[f] = s;
    }
    block_reduce<2>(acc, sred);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = acc[0];
        a.partials[2 * blockIdx.x + 1] = acc[1];
    }
    if (!last_block_done(a.counter, &sflag)) return;
    double tot[2];
    sum_partials<2>(a.partials, gridDim.x, tot, sred);
    if (threadIdx.x == 0) {
        const double gs = a.c.gridsize;
        for (int f = 0; f < 2; f++) {
            if (pass == 0) {
                if constexpr (sizeof(T) == 8) {
                    a.res[f] = tot[f] / gs;  // g2output.cpp:92
                } else {
                    a.res[4 + f] = tot[f] / gs;
                    a.res[f] = a.sc->fbar[f] + tot[f] / gs;
                }
            } else {
                a.res[2 + f] = tot[f] / gs;  // g2output.cpp:99
            }
        }
        *a.counter = 0u;
    }
}

// dfdi (g2functions.cpp:70-78) of one array along a stride, reference order
__device__ __forceinline__ double d4(double m2, double m1, double p1, double p2, double dx) {
    return ((1. / 12.) * m2 + ((-2.) / 3.) * m1 + (2. / 3.) * p1 + ((-1.) / 12.) * p2) / dx;
}

// Rows of outputfield(): for ii < ni, jj < nj, kk < nk the point
// (ii skip, jj skip, kk skip): nflds field values, then calcrho(0, i, j, k).
template <typename T>
__global__ void __launch_bounds__(256) slice_kernel(OutArgs a, int nj, int nk, int skip, size_t r0, size_t cnt,
                                                    double *out) {
    const int N = a.c.N;
    const size_t n3 = (size_t)N * N * N;
    const T *X = static_cast<const T *>(a.X), *D = static_cast<const T *>(a.D);
    const double dx = a.c.dx, a0 = a.sc->a[0];
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
        const size_t r = r0 + q;
        const int k = (int)(r % nk) * skip;
        const int j = (int)((r / nk) % nj) * skip;
        const int i = (int)(r / ((size_t)nk * nj)) * skip;
        auto at = [&](int fld, int ii, int jj, int kk) {
            return (double)X[fld * n3 + ((size_t)((ii + N) % N) * N + (jj + N) % N) * N + (kk + N) % N];
        };
        const size_t x = ((size_t)i * N + j) * N + k;
        double fv[2], dv[2];
        for (int f = 0; f < 2; f++) {
            fv[f] = field_value<T>(a, f, x);
            if constexpr (sizeof(T) == 8) dv[f] = D[f * n3 + x];
            else dv[f] = a.sc->dfbar[f] + (double)D[f * n3 + x];
        }
        double rho = pot64(a.c, fv[0], fv[1]);  // potential(0, i, j, k)
        for (int f = 0; f < 2; f++) {
            const double gi = d4(at(f, i - 2, j, k), at(f, i - 1, j, k), at(f, i + 1, j, k), at(f, i + 2, j, k), dx);
            const double gj = d4(at(f, i, j - 2, k), at(f, i, j - 1, k), at(f, i, j + 1, k), at(f, i, j + 2, k), dx);
            const double gk = d4(at(f, i, j, k - 2), at(f, i, j, k - 1), at(f, i, j, k + 1), at(f, i, j, k + 2), dx);
            const double g2 = gi * gi + gj * gj + gk * gk;  // gradF2 (:118-122)
            rho += (.5 * dv[f] * dv[f] + .5 * g2 / a0 / a0);
        }
        double *row = out + q * 3;
        row[0] = fv[0];
        row[1] = fv[1];
        row[2] = rho;
    }
}

}  // namespace gabe
