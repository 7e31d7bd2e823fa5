// FP64 kernels; built with -fmad=false (reference rounding, no FMA contraction).
#include "launch.h"

namespace gabe {

cudaError_t configure_f64(size_t max_smem) {
    cudaError_t e = cudaSuccess;
    int v = (int)max_smem;
    if ((e = cudaFuncSetAttribute(stage1_kernel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    if ((e = cudaFuncSetAttribute(stage1_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    if ((e = cudaFuncSetAttribute(stage2_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    if ((e = cudaFuncSetAttribute(bin_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, v))) return e;
    return e;
}

cudaError_t stage1_f64(const StencilArgs &a, const Launch &l) {
    if (a.gws) stage1_kernel<double, true><<<l.grid, l.block, l.smem, l.stream>>>(a);
    else stage1_kernel<double, false><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t stage2_f64(const StencilArgs &a, const Launch &l) {
    stage2_kernel<double><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t kspace_f64(const KspaceArgs &a, const Launch &l) {
    kspace_kernel<double><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t energy0_f64(const EnergyArgs &a, const Launch &l) {
    energy0_kernel<double><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t bins_f64(const BinArgs &a, const Launch &l) {
    bin_kernel<double><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t bin_reduce(const double *part_sum, const unsigned int *part_cnt, int nblocks, int nseries, int nbins,
                       double *sum, double *cnt, cudaStream_t s) {
    const int n = nseries * nbins;
    bin_reduce_kernel<<<(n + 127) / 128, 128, 0, s>>>(part_sum, part_cnt, nblocks, nseries, nbins, sum, cnt);
    return cudaGetLastError();
}

}  // namespace gabe
