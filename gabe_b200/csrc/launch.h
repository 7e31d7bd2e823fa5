// Host-side launch entry points of the precision-specific kernel units.
// kernels_f64.cu is compiled without FMA contraction so that the FP64 path
// rounds every operation as the reference's x86-64 build does;
// kernels_f32.cu is compiled with contraction on.
#pragma once

#include <cuda_runtime.h>

#include "kspace.cuh"
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

cudaError_t sweep_f64(int shape, int mode, const StencilArgs &a, dim3 grid, cudaStream_t s);
cudaError_t sweep_f32(int shape, int mode, const StencilArgs &a, dim3 grid, cudaStream_t s);
cudaError_t kspace_f64(const KspaceArgs &a, const Launch &l);
cudaError_t kspace_f32(const KspaceArgs &a, const Launch &l);
cudaError_t bins_f64(const BinArgs &a, const Launch &l);
cudaError_t bins_f32(const BinArgs &a, const Launch &l);
cudaError_t configure_bins(size_t max_smem);
cudaError_t gw_pack_f64(const double *src, size_t cnt, size_t m0, int N, size_t M, void *G, int which, double *norms,
                        cudaStream_t s);
cudaError_t gw_pack_f32(const double *src, size_t cnt, size_t m0, int N, size_t M, void *G, int which, double *norms,
                        cudaStream_t s);
cudaError_t gw_unpack_f64(const void *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst, cudaStream_t s);
cudaError_t gw_unpack_f32(const void *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst, cudaStream_t s);

cudaError_t mean_f64(const double *x, size_t n, double *partials, unsigned int *counter, double *out, int nblocks,
                     cudaStream_t s);
cudaError_t to_fluct(const double *x, size_t n, const double *mean, float *out, cudaStream_t s);
cudaError_t from_fluct(const float *x, size_t n, const double *mean, double *out, cudaStream_t s);

cudaError_t bin_reduce(const double *part_sum, const unsigned int *part_cnt, int nblocks, int nseries, int nbins,
                       double *sum, double *cnt, cudaStream_t s);

}  // namespace gabe
