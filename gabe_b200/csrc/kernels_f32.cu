// FP32-storage kernels; built with FMA contraction.
#include <algorithm>

#include "convert.cuh"
#include "launch.h"
#include "sweep32.cuh"
#include "slabgw.cuh"

namespace gabe {

// Plane slots of a sweep's ring (three planes being read, the rest in
// flight), all in the wide layout (sweep32.cuh, Ring).  Measured at 512^3:
// sweep A 1.81 ms with six slots (2.10 with four, 2.18 with ten); sweep B
// 0.835 with five (0.87 with six narrow ones, 1.02 with four); the
// energies-only sweep 0.2-0.4 with four against ~0.75 with six narrow ones.
// Fewer slots leave more of the SM's shared memory to L1.
template <int MODE>
constexpr int ring_slots() {
    return MODE == MODE_E0 ? 4 : (MODE == MODE_B ? 5 : 6);
}

template <int TK2, int TJ, int MODE, int MODEL>
static cudaError_t launch32m(const StencilArgs &a, dim3 grid, cudaStream_t s) {
    constexpr int S = ring_slots<MODE>();
    auto k = s32::sweep32_kernel<TK2, TJ, MODE, S, MODEL, true>;
    const size_t smem = (size_t)S * s32::Ring<TK2, TJ, true>::SLOT * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, TK2 * TJ, smem, s>>>(a);
    return cudaGetLastError();
}

// One instantiation per potential, so that no site branches on the model.
template <int TK2, int TJ, int MODE>
static cudaError_t launch32(const StencilArgs &a, dim3 grid, cudaStream_t s) {
    return a.c.model == MODEL_QUADRATIC ? launch32m<TK2, TJ, MODE, MODEL_QUADRATIC>(a, grid, s)
                                        : launch32m<TK2, TJ, MODE, MODEL_LPHI4>(a, grid, s);
}

template <int TK2, int TJ>
static cudaError_t sweep32_shape(int mode, const StencilArgs &a, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_A: return launch32<TK2, TJ, MODE_A>(a, grid, s);
        case MODE_A_GW: return launch32<TK2, TJ, MODE_A_GW>(a, grid, s);
        case MODE_E0: return launch32<TK2, TJ, MODE_E0>(a, grid, s);
        default: return launch32<TK2, TJ, MODE_B>(a, grid, s);
    }
}

// shape ids follow kShapes32 (launch.h); TK2 = TK / 2 threads along k
cudaError_t sweep32_f32(int shape, int mode, const StencilArgs &a, dim3 grid, cudaStream_t s) {
    switch (shape) {
        case 0: return sweep32_shape<32, 8>(mode, a, grid, s);
        case 1: return sweep32_shape<32, 4>(mode, a, grid, s);
        case 2: return sweep32_shape<64, 4>(mode, a, grid, s);
        case 3: return sweep32_shape<16, 8>(mode, a, grid, s);
        case 4: return sweep32_shape<32, 16>(mode, a, grid, s);
        case 5: return sweep32_shape<16, 4>(mode, a, grid, s);
        case 6: return sweep32_shape<8, 8>(mode, a, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t slab_finish_f32(int mode, const LatticeConsts &c, DevScalars *sc, const double *tot, cudaStream_t s) {
    switch (mode) {
        case MODE_A: slab_finish_kernel<float, MODE_A><<<1, 32, 0, s>>>(c, sc, tot, 0); break;
        case MODE_A_GW: slab_finish_kernel<float, MODE_A_GW><<<1, 32, 0, s>>>(c, sc, tot, 0); break;
        case MODE_E0: slab_finish_kernel<float, MODE_E0><<<1, 32, 0, s>>>(c, sc, tot, 0); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t slab_kspace_f32(const void *T, void *G, const DevScalars *sc, const LatticeConsts &c, int m, int y0,
                            cudaStream_t s) {
    return slab_kspace<float>(T, G, sc, c, m, y0, s);
}
cudaError_t slab_gw_amplitudes_f32(const void *G, size_t cnt, size_t m0, int N, int m, int y0, int which, double *dst,
                                   cudaStream_t s) {
    return slab_gw_amplitudes<float>(G, cnt, m0, N, m, y0, which, dst, s);
}

cudaError_t kspace_f32(const KspaceArgs &a, const Launch &l) {
    kspace_kernel<float><<<l.grid, l.block, l.smem, l.stream>>>(a);
    return cudaGetLastError();
}

cudaError_t gw_pack_f32(const double *src, size_t cnt, size_t m0, int N, size_t M, void *G, int which, double *norms, int gt,
                      cudaStream_t s) {
    gw_pack_kernel<float><<<4 * 148, 256, 0, s>>>(src, cnt, m0, N, M, static_cast<Cplx<float> *>(G), which, norms, gt);
    return cudaGetLastError();
}

cudaError_t gw_unpack_f32(const void *G, size_t cnt, size_t m0, int N, size_t M, int which, double *dst, int gt,
                          cudaStream_t s) {
    gw_unpack_kernel<float><<<4 * 148, 256, 0, s>>>(static_cast<const Cplx<float> *>(G), cnt, m0, N, M, which, dst, gt);
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

cudaError_t meansvars_f32(const OutArgs &a, int pass, int nblocks, cudaStream_t s) {
    meansvars_kernel<float><<<nblocks, 256, 0, s>>>(a, pass);
    return cudaGetLastError();
}

cudaError_t slice_f32(const OutArgs &a, int nj, int nk, int skip, size_t r0, size_t cnt, double *out, cudaStream_t s) {
    const int blocks = (int)((cnt + 255) / 256 < 4 * 148 ? (cnt + 255) / 256 : 4 * 148);
    slice_kernel<float><<<blocks > 0 ? blocks : 1, 256, 0, s>>>(a, nj, nk, skip, r0, cnt, out);
    return cudaGetLastError();
}

}  // namespace gabe
