// Shared device-side definitions for the GABE sm_100a kernels.
//
// State layout in HBM (per handle):
//   fields   X[buf][fld][i][j][k]     (k fastest; two ping-pong buffers)
//   momenta  D[buf][fld][i][j][k]
//   GW       h[12][i][j][kz], l[12][i][j][kz]   planar, kz < N/2+1
//   sources  S[12][i][j][N+2]  real, padded rows so cuFFT can run R2C in
//            place; afterwards the same bytes hold the 12 half-spectra
//            S^[12][i][j][kz] (complex).  Slots 0..5 carry the stage-0
//            source 11,12,13,22,23,33, slots 6..11 the stage-1 source.
//   scalars  DevScalars (a, adot, energies per stage, homogeneous
//            trajectory of the FP32 path, status word)
//   partials per-block FP64 sums of the energy reductions
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gabe {

// Status bits raised on the device and read by the host at sync points.
enum : uint32_t {
    ST_NONFINITE = 1u,
    ST_TIMEOUT = 2u,  // a bounded wait on a bulk copy gave up (tma.cuh)
};

// Per-stage scalars, laid out like the reference's globals
// a[2], adot[2], edkin[2], edpot[2], edgrad[2], edrho[2] (g2header.h:58-63).
struct DevScalars {
    double a[2], adot[2], edkin[2], edpot[2], edgrad[2], edrho[2];
    // FP32 path: homogeneous trajectory (fields and momenta) at stage 0.
    double fbar[2], dfbar[2];
    long long step;
    unsigned int status;
    unsigned int adot_given;  // adot[0] came from the caller (after an upload), not from adf(0)
    // a[0], adot[0], a[1], adot[1] of the step whose GW sources sit in source
    // buffer s, for the k-space update (which may run while the fields are
    // already one step further on)
    double gw[2][4];
};

enum Model : int { MODEL_QUADRATIC = 0, MODEL_LPHI4 = 1 };

// Constants of one lattice, computed on the host with the same sequence of
// IEEE operations the reference's compiler folds (so FP64 results agree
// bit for bit where the reference's operation order is kept).
struct LatticeConsts {
    int N;
    int model;
    int expansion;          // expansion_type: 0 none, 1 Friedmann, 2 Friedmann without tensor modes
    double dt, half_dt;     // dt, .5*dt
    double dx;              // L/((double)N) (g2parameters.h:93)
    double inv_dx2_div;     // dx*dx (the reference divides by it)
    double dn, c13, c23;    // 1/(dx*dx), (1./3.)*dn, (2./3.)*dn  (g2evolutionpert.cpp:53-116)
    double mc[5];           // model constants (see model_consts on the host)
    double gridsize;        // N^3
    double eight_pi_3;      // 8.*M_PI/3.
    double k2norm_c;        // 4.*M_PI*M_PI/L/L
    double eight_pi;        // 8.*M_PI
    double normmm;          // pow(dx,3)
};

__host__ __device__ inline int wrapi(int x, int N) { return x < 0 ? x + N : (x >= N ? x - N : x); }

// ---------------------------------------------------------------------------
// FP64 model, reference operation order (g2model.cpp:66-87 for the shipped
// model; oracle/ref_cfg/g2model_lphi4.cpp order for lambda phi^4).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pot64(const LatticeConsts &c, double P, double C) {
    if (c.model == MODEL_QUADRATIC) return (0.5 * P * P + c.mc[1] * P * P * C * C);
    return c.mc[2] * P * P * P * P + c.mc[3] * P * P * C * C;
}
__device__ __forceinline__ double dv64(const LatticeConsts &c, int fld, double P, double C) {
    if (c.model == MODEL_QUADRATIC) {
        if (fld == 0) return (P + c.mc[0] * C * C * P);
        return (c.mc[0] * P * P * C);
    }
    if (fld == 0) return c.mc[0] * P * P * P + c.mc[1] * C * C * P;
    return c.mc[1] * P * P * C;
}

// ---------------------------------------------------------------------------
// FP32 fluctuation model: differences V(fbar+d) - V(fbar) and
// V'(fbar+d) - V'(fbar) expanded so that no term cancels (pb, cb = homogeneous
// phi, chi; a, b = their fluctuations).
// ---------------------------------------------------------------------------
struct MeanF {
    float pb, cb;      // homogeneous values as float
    float q0, q1;      // model constants as float
    float q2, q3;
    float pb2, cb2;    // 2 pb, 2 cb
    float pbsq, pb3sq; // pb^2, 3 pb^2
};

__device__ __forceinline__ float dv_diff32(const MeanF &m, int model, int fld, float a, float b) {
    const float pb = m.pb;
    const float C = m.cb + b;
    if (model == MODEL_QUADRATIC) {
        // V' = phi + C1 chi^2 phi ; V'_chi = C1 phi^2 chi
        if (fld == 0) return a + m.q0 * (pb * b * (m.cb2 + b) + a * C * C);
        return m.q0 * (a * (m.pb2 + a) * C + m.pbsq * b);
    }
    // V' = lam phi^3 + g chi^2 phi ; V'_chi = g phi^2 chi
    if (fld == 0) return m.q0 * a * (m.pb3sq + a * (3.f * pb + a)) + m.q1 * (pb * b * (m.cb2 + b) + a * C * C);
    return m.q1 * (a * (m.pb2 + a) * C + m.pbsq * b);
}

__device__ __forceinline__ float v_diff32(const MeanF &m, int model, float a, float b) {
    const float pb = m.pb, cb = m.cb;
    const float P = pb + a, C = cb + b;
    const float cross = (pb * b + cb * a + a * b) * (P * C + pb * cb);
    if (model == MODEL_QUADRATIC) return a * (pb + 0.5f * a) + m.q1 * cross;
    return m.q2 * a * (4.f * pb * pb * pb + a * (6.f * pb * pb + a * (4.f * pb + a))) + m.q3 * cross;
}

// Homogeneous potential and force in FP64 (for the FP32 path's mean).
__host__ __device__ inline double pot_h(int model, const double *mc, double P, double C) {
    if (model == MODEL_QUADRATIC) return 0.5 * P * P + mc[1] * P * P * C * C;
    return mc[2] * P * P * P * P + mc[3] * P * P * C * C;
}
__host__ __device__ inline double dv_h(int model, const double *mc, int fld, double P, double C) {
    if (model == MODEL_QUADRATIC) return fld == 0 ? P + mc[0] * C * C * P : mc[0] * P * P * C;
    return fld == 0 ? mc[0] * P * P * P + mc[1] * C * C * P : mc[1] * P * P * C;
}

// ---------------------------------------------------------------------------
// block reduction of NV doubles; result valid in thread 0
// ---------------------------------------------------------------------------
// Sum over the lanes of this warp that exist (blocks need not be a multiple
// of 32 threads); the total lands in lane 0.
__device__ __forceinline__ double warp_sum(double x, int nlanes) {
    const unsigned mask = nlanes >= 32 ? 0xffffffffu : ((1u << nlanes) - 1u);
    const int lane = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double y = __shfl_down_sync(mask, x, o);
        if ((lane & 31) + o < nlanes) x += y;
    }
    return x;
}

template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double *sred) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nwarp = (nthr + 31) >> 5;
    const int my_lanes = (warp == nwarp - 1) ? nthr - 32 * warp : 32;
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q], my_lanes);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sred[warp * NV + q] = v[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nwarp ? sred[lane * NV + q] : 0.0;
            v[q] = warp_sum(x, my_lanes);
        }
    }
    __syncthreads();
}

// Deterministic sum of nblk partial vectors (stride NV) by one block, with
// compensated accumulation per thread; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void sum_partials(const double *partials, int nblk, double (&out)[NV], double *sred) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    double s[NV], comp[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) { s[q] = 0.0; comp[q] = 0.0; }
    for (int b = tid; b < nblk; b += nthr) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double y = __ldcg(partials + (size_t)b * NV + q) - comp[q];
            double t = s[q] + y;
            comp[q] = (t - s[q]) - y;
            s[q] = t;
        }
    }
    block_reduce<NV>(s, sred);
#pragma unroll
    for (int q = 0; q < NV; q++) out[q] = s[q];
}

// Returns true in every thread of the block that finished last.
__device__ __forceinline__ bool last_block_done(unsigned int *counter, int *sflag) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const unsigned int total = gridDim.x * gridDim.y * gridDim.z;
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        unsigned int prev = atomicAdd(counter, 1u);
        *sflag = (prev == total - 1) ? 1 : 0;
    }
    __syncthreads();
    bool last = *sflag != 0;
    if (last) __threadfence();
    return last;
}

}  // namespace gabe
