// Host<->device conversions of the FP32 path: the host interface is FP64 in
// the reference layout; the device keeps FP32 fluctuations about FP64 means.
#pragma once

#include "common.cuh"

namespace gabe {

// Deterministic mean of n doubles into *out (block partials + last block).
__global__ void __launch_bounds__(256) mean_kernel(const double *x, size_t n, double *partials, unsigned int *counter,
                                                   double *out) {
    __shared__ double sred[8];
    __shared__ int sflag;
    double s = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) s += x[q];
    double v[1] = {s};
    block_reduce<1>(v, sred);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
    if (!last_block_done(counter, &sflag)) return;
    double tot[1];
    sum_partials<1>(partials, gridDim.x, tot, sred);
    if (threadIdx.x == 0) {
        *out = tot[0] / (double)n;
        *counter = 0u;
    }
}

__global__ void to_fluct_kernel(const double *x, size_t n, const double *mean, float *out) {
    const double m = mean ? *mean : 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        out[q] = (float)(x[q] - m);
}

__global__ void from_fluct_kernel(const float *x, size_t n, const double *mean, double *out) {
    const double m = mean ? *mean : 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        out[q] = m + (double)x[q];
}

}  // namespace gabe
