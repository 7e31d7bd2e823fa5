// FP32-storage kernels; built with FMA contraction.
#include "convert.cuh"
#include "launch.h"

namespace gabe {

cudaError_t configure_f32(size_t max_smem) {
    cudaError_t e = cudaSuccess;
    int v = (int)max_smem;
    if ((e = cudaFuncSetAttribute(stage1_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    if ((e = cudaFuncSetAttribute(stage1_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    if ((e = cudaFuncSetAttribute(stage2_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    if ((e = cudaFuncSetAttribute(bin_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    return e;
}

cudaError_t stage1_f32(const StencilArgs &a, const Launch &l) {
    if (a.gws) stage1_kernel<float, true><<<l.grid, l.block, l.smem, l.stream>>>(a);
    else stage1_kernel<float, false><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t stage2_f32(const StencilArgs &a, const Launch &l) {
    stage2_kernel<float><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t kspace_f32(const KspaceArgs &a, const Launch &l) {
    kspace_kernel<float><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t energy0_f32(const EnergyArgs &a, const Launch &l) {
    energy0_kernel<float><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t bins_f32(const BinArgs &a, const Launch &l) {
    bin_kernel<float><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t mean_f64(const double *x, size_t n, double *partials, unsigned int *counter, double *out, int nblocks,
                     cudaStream_t s) {
    mean_kernel<<<nblocks, 256, 0, s>>>(x, n, partials, counter, out);
    return cudaGetLastError();
}

cudaError_t to_fluct(const double *x, size_t n, const double *mean, float *out, cudaStream_t s) {
    to_fluct_kernel<<<4 * 148, 256, 0, s>>>(x, n, mean, out);
    return cudaGetLastError();
}

cudaError_t from_fluct(const float *x, size_t n, const double *mean, double *out, cudaStream_t s) {
    from_fluct_kernel<<<4 * 148, 256, 0, s>>>(x, n, mean, out);
    return cudaGetLastError();
}

}  // namespace gabe
