// calcEnergy(0) of an uploaded state (g2functions.cpp:124-174).  Runs once
// per upload, so it reads its 7-point neighbourhoods straight from global
// memory; the per-step energies come from the fused stage sweeps.
#pragma once

#include "common.cuh"

namespace gabe {

struct EnergyArgs {
    const void *X, *D;
    double *partials;
    unsigned int *counter;
    DevScalars *sc;
    LatticeConsts c;
};

template <typename T>
__global__ void __launch_bounds__(256) energy0_kernel(EnergyArgs a) {
    __shared__ double sred[8 * 3];
    __shared__ int sflag;
    const LatticeConsts &c = a.c;
    const int N = c.N;
    const size_t n3 = (size_t)N * N * N;
    const T *X = static_cast<const T *>(a.X), *D = static_cast<const T *>(a.D);
    double kin = 0., pot = 0., grad = 0.;
    const double fb0 = a.sc->fbar[0], fb1 = a.sc->fbar[1];
    MeanF m;
    if constexpr (sizeof(T) == 4) {
        const double fb[2] = {fb0, fb1};
        m.pb = (float)fb[0]; m.cb = (float)fb[1];
        m.q0 = (float)c.mc[0]; m.q1 = (float)c.mc[1]; m.q2 = (float)c.mc[2]; m.q3 = (float)c.mc[3];
    }
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n3; x += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(x % N);
        const size_t t = x / N;
        const int j = (int)(t % N), i = (int)(t / N);
        const size_t ip = ((size_t)wrapi(i + 1, N) * N + j) * N + k, im = ((size_t)wrapi(i - 1, N) * N + j) * N + k;
        const size_t jp = ((size_t)i * N + wrapi(j + 1, N)) * N + k, jm = ((size_t)i * N + wrapi(j - 1, N)) * N + k;
        const size_t kp = ((size_t)i * N + j) * N + wrapi(k + 1, N), km = ((size_t)i * N + j) * N + wrapi(k - 1, N);
        T fc[2];
        for (int f = 0; f < 2; f++) {
            const T *g = X + f * n3;
            const T d = D[f * n3 + x];
            fc[f] = g[x];
            if constexpr (sizeof(T) == 8) {
                const double lap = (g[ip] + g[im] + g[jp] + g[jm] + g[kp] + g[km] - 6. * g[x]) / c.inv_dx2_div;
                kin += d * d;
                grad -= g[x] * lap;
            } else {
                const float lap = ((g[ip] + g[im]) + (g[jp] + g[jm]) + (g[kp] + g[km]) - 6.f * g[x]) *
                                  (float)(1.0 / c.inv_dx2_div);
                const double dt = a.sc->dfbar[f] + (double)d;
                kin += dt * dt;
                grad -= (double)(g[x] * lap);
            }
        }
        if constexpr (sizeof(T) == 8) pot += pot64(c, fc[0], fc[1]);
        else pot += (double)v_diff32(m, c.model, fc[0], fc[1]);
    }
    double v[3] = {kin, pot, grad};
    block_reduce<3>(v, sred);
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) a.partials[(size_t)blockIdx.x * 3 + q] = v[q];
    if (!last_block_done(a.counter, &sflag)) return;
    double tot[3];
    sum_partials<3>(a.partials, gridDim.x, tot, sred);
    if (threadIdx.x == 0) {
        DevScalars *s = a.sc;
        const double a0 = s->a[0];
        double ek = tot[0] / c.gridsize / 2.;
        double ep = tot[1] / c.gridsize;
        const double eg = tot[2] / c.gridsize / 2. / a0 / a0;
        if constexpr (sizeof(T) == 4) ep += pot_h(c.model, c.mc, fb0, fb1);
        s->edkin[0] = ek;
        s->edpot[0] = ep;
        s->edgrad[0] = eg;
        s->edrho[0] = ek + ep + eg;
        if (!isfinite(s->edrho[0])) s->status |= ST_NONFINITE;
        *a.counter = 0u;
    }
}

}  // namespace gabe
