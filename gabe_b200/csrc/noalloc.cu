// gabe_energy_noalloc: calcEnergy(0) of a state in caller-owned device
// memory, without allocating anything.
//
// Some callers cannot allocate device memory when they need the energies:
// a host framework that has handed all free device memory to its own pool
// allocator (a cudaMalloc there fails or evicts its cache), code that must
// not stall the device (cudaMalloc/cudaFree can synchronise it), or a
// driver that has already reserved every buffer for its run.  gabe_create
// allocates its scratch up front, which those callers cannot do, so this
// entry point takes the state by device pointer and keeps its reduction
// scratch -- per-block partial sums, the last-block counter and the scalar
// block -- in one file-scope __device__ array of fixed size.
//
// The kernel is the stage-0 energy sweep the library itself runs
// (sweep_kernel, mode E0, FP64 reference arithmetic), on the same grid
// plan, so the results equal gabe_energies for the same state bit for bit.
//
// Contract:
//   * field0/dfield0: device arrays [2][N^3] (FP64, k fastest), out4: device
//     array of 4 doubles {kin, pot, grad, rho}; stream: cudaStream_t or NULL.
//   * The scratch holds kNoAllocMaxBlocks blocks of partial sums (2 MiB plus
//     a few hundred bytes).  A lattice whose grid needs more blocks is
//     refused with GABE_ERR_PARAM before any work is queued.
//   * Every device that loads the library holds the array until the process
//     exits.  Its host-side name is only a stand-in; the device address is
//     looked up with cudaGetSymbolAddress the first time the entry point runs
//     on each device (with that device current), so that first call should
//     come before any stream capture on the device.
//   * All calls on a device share the array: calls that overlap on the GPU
//     (on different streams, or from several threads) race on it.  Each call
//     resets what must start at zero (counter, status) before its sweep.
//   * The looked-up address is kept for the life of the process.  After a
//     cudaDeviceReset the device's context, and the array's address with it,
//     are new, so the entry point must not be called again in that process.
//   * A non-finite result (a state holding NaN or Inf) is returned as NaN or
//     Inf in out4; the call has no status word, so check out4.
#include <mutex>

#include "launch.h"

namespace gabe {
namespace {

constexpr int kNoAllocMaxBlocks = 32768;
constexpr size_t kScalarDoubles = (sizeof(DevScalars) + sizeof(double) - 1) / sizeof(double);
// partials, then the scalar block, then the counter (one double slot)
constexpr size_t kScratchDoubles = (size_t)kNoAllocMaxBlocks * kNV + kScalarDoubles + 1;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
double *g_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (set-up on
// first use per device).
cudaError_t scratch_address(int dev, double **out) {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

__global__ void noalloc_begin(DevScalars *sc, unsigned int *counter, double a0) {
    DevScalars s{};
    s.a[0] = a0;
    s.adot_given = 1;  // adot is not asked for; keep the sweep from forming it
    *sc = s;
    *counter = 0u;
}

__global__ void noalloc_end(const DevScalars *sc, double *out4) {
    out4[0] = sc->edkin[0];
    out4[1] = sc->edpot[0];
    out4[2] = sc->edgrad[0];
    out4[3] = sc->edrho[0];
}

template <int TK, int TJ>
cudaError_t launch_e0(const StencilArgs &a, dim3 grid, cudaStream_t s) {
    sweep_kernel<double, TK, TJ, MODE_E0><<<grid, dim3(TK * TJ), 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace
}  // namespace gabe

using namespace gabe;

extern "C" int gabe_energy_noalloc(const gabe_params *p, const double *field0, const double *dfield0, double a0,
                                   double *out4, void *stream) {
    if (!p || !field0 || !dfield0 || !out4) return GABE_ERR_PARAM;
    // the same parameter checks as gabe_create, and the FP64 stencil tiling
    if (!params_valid(*p, nullptr, 0) || !(a0 > 0) || !std::isfinite(a0)) return GABE_ERR_PARAM;
    const GridPlan g = plan_grid(p->N, p->tile_shape, p->tile_ci);
    if (g.shape < 0) return GABE_ERR_PARAM;  // no tile divides N (N % 4 != 0)
    const long long nblocks = (long long)g.grid.x * g.grid.y * g.grid.z;
    if (nblocks > kNoAllocMaxBlocks) return GABE_ERR_PARAM;  // scratch too small for this grid
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return GABE_ERR_CUDA;
    }
    double *base = nullptr;
    if (scratch_address(dev, &base) != cudaSuccess) {
        cudaGetLastError();
        return GABE_ERR_CUDA;
    }
    DevScalars *sc = reinterpret_cast<DevScalars *>(base + (size_t)kNoAllocMaxBlocks * kNV);
    unsigned int *counter = reinterpret_cast<unsigned int *>(base + (size_t)kNoAllocMaxBlocks * kNV + kScalarDoubles);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    StencilArgs a{};
    a.X = field0;
    a.D = dfield0;
    a.partials = base;
    a.counter = counter;
    a.sc = sc;
    a.c = make_lattice_consts(*p);
    a.ci = g.ci;
    noalloc_begin<<<1, 1, 0, s>>>(sc, counter, a0);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        switch (g.shape) {
            case 0: e = launch_e0<32, 8>(a, g.grid, s); break;
            case 1: e = launch_e0<16, 16>(a, g.grid, s); break;
            case 2: e = launch_e0<32, 4>(a, g.grid, s); break;
            case 3: e = launch_e0<16, 8>(a, g.grid, s); break;
            case 4: e = launch_e0<8, 8>(a, g.grid, s); break;
            case 5: e = launch_e0<4, 4>(a, g.grid, s); break;
            default: e = cudaErrorInvalidValue; break;
        }
    }
    if (e == cudaSuccess) {
        noalloc_end<<<1, 1, 0, s>>>(sc, out4);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? GABE_OK : GABE_ERR_CUDA;
}
