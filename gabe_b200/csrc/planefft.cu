// Host side of the FP32 plane transforms (planefft.cuh): cluster launch
// configuration and the persistent grid size.
#include "launch.h"
#include "planefft.cuh"

namespace gabe {

namespace {

template <int N>
cudaLaunchConfig_t plane_config(int grid, cudaStream_t s, cudaLaunchAttribute *attr) {
    using Gm = pfft::PlaneGeom<N>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(Gm::T);
    cfg.dynamicSmemBytes = Gm::SMEM_BYTES;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = Gm::CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <int N>
cudaError_t plane_setup_n(int *grid) {
    using Gm = pfft::PlaneGeom<N>;
    auto k = pfft::plane_r2c_kernel<N>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Gm::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (Gm::CS > 8) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = plane_config<N>(Gm::CS, nullptr, attr);
    int ncl = 0;
    e = cudaOccupancyMaxActiveClusters(&ncl, k, &cfg);
    if (e != cudaSuccess) return e;
    if (ncl < 1) return cudaErrorInvalidConfiguration;
    *grid = ncl * Gm::CS;
    return cudaSuccess;
}

template <int N>
cudaError_t plane_launch_n(float *S, int nplanes, int grid, cudaStream_t s) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = plane_config<N>(grid, s, attr);
    return cudaLaunchKernelEx(&cfg, pfft::plane_r2c_kernel<N>, S, nplanes);
}

}  // namespace

bool plane_r2c_supported(int N) { return N == 64 || N == 128 || N == 256 || N == 512; }

cudaError_t plane_r2c_setup(int N, int *grid) {
    switch (N) {
        case 64: return plane_setup_n<64>(grid);
        case 128: return plane_setup_n<128>(grid);
        case 256: return plane_setup_n<256>(grid);
        case 512: return plane_setup_n<512>(grid);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t plane_r2c_f32(int N, float *S, int nplanes, int grid, cudaStream_t s) {
    switch (N) {
        case 64: return plane_launch_n<64>(S, nplanes, grid, s);
        case 128: return plane_launch_n<128>(S, nplanes, grid, s);
        case 256: return plane_launch_n<256>(S, nplanes, grid, s);
        case 512: return plane_launch_n<512>(S, nplanes, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gabe
