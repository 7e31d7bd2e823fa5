// FP64 kernels; built with -fmad=false (reference rounding, no FMA contraction).
#include "launch.h"
#include "slabgw.cuh"

namespace gabe {

template <int TK, int TJ>
static cudaError_t sweep_shape(int mode, const StencilArgs &a, dim3 grid, cudaStream_t s) {
    const dim3 block(TK * TJ);
    switch (mode) {
        case MODE_A: sweep_kernel<double, TK, TJ, MODE_A><<<grid, block, 0, s>>>(a); break;
        case MODE_A_GW: sweep_kernel<double, TK, TJ, MODE_A_GW><<<grid, block, 0, s>>>(a); break;
        case MODE_E0: sweep_kernel<double, TK, TJ, MODE_E0><<<grid, block, 0, s>>>(a); break;
        default: sweep_kernel<double, TK, TJ, MODE_B><<<grid, block, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

cudaError_t sweep_f64(int shape, int mode, const StencilArgs &a, dim3 grid, cudaStream_t s) {
    switch (shape) {
        case 0: return sweep_shape<32, 8>(mode, a, grid, s);
        case 1: return sweep_shape<16, 16>(mode, a, grid, s);
        case 2: return sweep_shape<32, 4>(mode, a, grid, s);
        case 3: return sweep_shape<16, 8>(mode, a, grid, s);
        case 4: return sweep_shape<8, 8>(mode, a, grid, s);
        case 5: return sweep_shape<4, 4>(mode, a, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t slab_finish_f64(int mode, const LatticeConsts &c, DevScalars *sc, const double *tot, cudaStream_t s) {
    switch (mode) {
        case MODE_A: slab_finish_kernel<double, MODE_A><<<1, 32, 0, s>>>(c, sc, tot, 0); break;
        case MODE_A_GW: slab_finish_kernel<double, MODE_A_GW><<<1, 32, 0, s>>>(c, sc, tot, 0); break;
        case MODE_E0: slab_finish_kernel<double, MODE_E0><<<1, 32, 0, s>>>(c, sc, tot, 0); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t slab_gw_pack_f64(const void *S, void *send, int N, int nloc, int W, int ncomp, cudaStream_t s) {
    return slab_gw_pack<double>(S, send, N, nloc, W, ncomp, s);
}
cudaError_t slab_gw_unpack_f64(const void *recv, void *T, int N, int m, int W, int ncomp, cudaStream_t s) {
    return slab_gw_unpack<double>(recv, T, N, m, W, ncomp, s);
}
cudaError_t slab_kspace_f64(const void *T, void *G, const DevScalars *sc, const LatticeConsts &c, int m, int y0,
                            cudaStream_t s) {
    return slab_kspace<double>(T, G, sc, c, m, y0, s);
}
cudaError_t slab_gw_amplitudes_f64(const void *G, size_t cnt, size_t m0, int N, int m, int y0, int which, double *dst,
                                   cudaStream_t s) {
    return slab_gw_amplitudes<double>(G, cnt, m0, N, m, y0, which, dst, s);
}

cudaError_t kspace_f64(const KspaceArgs &a, const Launch &l) {
    kspace_kernel<double><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t gw_pack_f64(const double *src, size_t cnt, size_t m0, int N, size_t M, void *G, int which, double *norms,
                      cudaStream_t s) {
    gw_pack_kernel<double><<<4 * 148, 256, 0, s>>>(src, cnt, m0, N, M, static_cast<Cplx<double> *>(G), which, norms, 0);
    return cudaGetLastError();
}

cudaError_t gw_unpack_f64(const void *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst, cudaStream_t s) {
    gw_unpack_kernel<double><<<4 * 148, 256, 0, s>>>(static_cast<const Cplx<double> *>(G), cnt, m0, N, M, which, dst, 0);
    return cudaGetLastError();
}

cudaError_t bins_f64(const BinArgs &a, const Launch &l) {
    bin_kernel<double><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t configure_bins(size_t max_smem) {
    cudaError_t e = cudaFuncSetAttribute(bin_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(bin_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
}

cudaError_t bin_reduce(const double *part_sum, const unsigned int *part_cnt, int nblocks, int nseries, int nbins,
                       double *sum, double *cnt, cudaStream_t s) {
    const int n = nseries * nbins;
    bin_reduce_kernel<<<(n + 127) / 128, 128, 0, s>>>(part_sum, part_cnt, nblocks, nseries, nbins, sum, cnt);
    return cudaGetLastError();
}

cudaError_t meansvars_f64(const OutArgs &a, int pass, int nblocks, cudaStream_t s) {
    meansvars_kernel<double><<<nblocks, 256, 0, s>>>(a, pass);
    return cudaGetLastError();
}

cudaError_t slice_f64(const OutArgs &a, int nj, int nk, int skip, size_t r0, size_t cnt, double *out, cudaStream_t s) {
    const int blocks = (int)((cnt + 255) / 256 < 4 * 148 ? (cnt + 255) / 256 : 4 * 148);
    slice_kernel<double><<<blocks > 0 ? blocks : 1, 256, 0, s>>>(a, nj, nk, skip, r0, cnt, out);
    return cudaGetLastError();
}

}  // namespace gabe
