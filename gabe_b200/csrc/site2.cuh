// FP32 site arithmetic of the field sweeps on two sites at once.
//
// Each thread of the FP32 sweeps owns two adjacent sites along k.  Their
// updates are the same expressions on different data, so they are written
// here once on pairs (F2: one float2 holding site 0 and site 1) with
// sm_100's packed FP32 instructions (__fadd2_rn, __fmul2_rn, __ffma2_rn):
// one instruction per operation for both sites, each lane rounded exactly as
// the scalar operation would be.  The expressions are those of stencil.cuh
// and common.cuh (lap32, source_add32, dv_diff32, v_diff32), with every
// multiply-add written as a fused multiply-add.
#pragma once

#include "stencil.cuh"

namespace gabe {
namespace s2 {

struct F2 {
    float2 v;
};

__device__ __forceinline__ F2 sp(float x) { return {make_float2(x, x)}; }
__device__ __forceinline__ F2 mk(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ F2 mk(float2 a) { return {a}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
// a - b as a + (-1) b: one rounding, the same as the subtraction
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 neg(F2 a) { return {make_float2(-a.v.x, -a.v.y)}; }
__device__ __forceinline__ float lanes(F2 a) { return a.v.x + a.v.y; }

// 7-point neighbourhoods of both sites, reference order: centre, i+1, i-1,
// j+1, j-1, k+1, k-1.
struct Nb {
    F2 v[7];
};

// lap32 of both sites.
__device__ __forceinline__ F2 lap(const Nb &f, F2 inv_dx2) {
    return fma(sp(-6.f), f.v[0], ((f.v[1] + f.v[2]) + (f.v[3] + f.v[4])) + (f.v[5] + f.v[6])) * inv_dx2;
}

// x + h y per neighbour.
__device__ __forceinline__ Nb axpy(const Nb &x, F2 h, const Nb &y) {
    Nb r;
#pragma unroll
    for (int q = 0; q < 7; q++) r.v[q] = fma(h, y.v[q], x.v[q]);
    return r;
}

// source_add32: GW source components 11,12,13,22,23 of one field added into s.
__device__ __forceinline__ void source_add(F2 dn, const Nb &f, F2 (&s)[kSrc]) {
    const F2 h = sp(0.5f);
    const F2 d1 = h * (f.v[1] - f.v[2]), d2 = h * (f.v[3] - f.v[4]), d3 = h * (f.v[5] - f.v[6]);
    const F2 tn = sp(-1.f / 3.f) * fma(d3, d3, fma(d2, d2, d1 * d1));  // -|grad|^2 / 3
    s[0] = fma(dn, fma(d1, d1, tn), s[0]);
    s[1] = fma(dn * d1, d2, s[1]);
    s[2] = fma(dn * d1, d3, s[2]);
    s[3] = fma(dn, fma(d2, d2, tn), s[3]);
    s[4] = fma(dn * d2, d3, s[4]);
}

// dv_diff32: V'(fbar + delta) - V'(fbar) of field fld, a = delta phi, b = delta chi.
__device__ __forceinline__ F2 dv_diff(const MeanF &m, int model, int fld, F2 a, F2 b) {
    const F2 pb = sp(m.pb), C = sp(m.cb) + b;
    if (model == MODEL_QUADRATIC) {
        if (fld == 0) return fma(sp(m.q0), fma(pb * b, sp(m.cb2) + b, a * C * C), a);
        return sp(m.q0) * fma(a * (sp(m.pb2) + a), C, sp(m.pbsq) * b);
    }
    if (fld == 0)
        return fma(sp(m.q0) * a, fma(a, fma(sp(3.f), pb, a), sp(m.pb3sq)),
                   sp(m.q1) * fma(pb * b, sp(m.cb2) + b, a * C * C));
    return sp(m.q1) * fma(a * (sp(m.pb2) + a), C, sp(m.pbsq) * b);
}

// v_diff32: V(fbar + delta) - V(fbar).
__device__ __forceinline__ F2 v_diff(const MeanF &m, int model, F2 a, F2 b) {
    const F2 pb = sp(m.pb), cb = sp(m.cb);
    const F2 P = pb + a, C = cb + b;
    const F2 cross = fma(pb, b, fma(cb, a, a * b)) * fma(P, C, pb * cb);
    if (model == MODEL_QUADRATIC) return fma(a, fma(sp(0.5f), a, pb), sp(m.q1) * cross);
    const float pbs = m.pb;
    const F2 poly = fma(a, fma(a, fma(sp(4.f), pb, a), sp(6.f * pbs * pbs)), sp(4.f * pbs * pbs * pbs));
    return fma(sp(m.q2) * a, poly, sp(m.q3) * cross);
}

// The FP32 moments of Moments (stencil.cuh), per lane.
struct Mom {
    F2 a[2], b, c[2], e, f, g0, g1, v0, v1;
};
__device__ __forceinline__ void zero(Mom &m) {
    m.a[0] = m.a[1] = m.b = m.c[0] = m.c[1] = m.e = m.f = m.g0 = m.g1 = m.v0 = m.v1 = sp(0.f);
}
// the two lanes' moments added into the per-thread Moments that fold() takes
__device__ __forceinline__ void collapse(const Mom &m, Moments &out) {
    out.a[0] = lanes(m.a[0]);
    out.a[1] = lanes(m.a[1]);
    out.b = lanes(m.b);
    out.c[0] = lanes(m.c[0]);
    out.c[1] = lanes(m.c[1]);
    out.e = lanes(m.e);
    out.f = lanes(m.f);
    out.g0 = lanes(m.g0);
    out.g1 = lanes(m.g1);
    out.v0 = lanes(m.v0);
    out.v1 = lanes(m.v1);
}

// Per-launch constants as pairs.
struct K2 {
    F2 ia02, ia12, c3H0, c3H1, h, dt, inv_dx2, dn;
};
template <typename S>
__device__ __forceinline__ K2 k2_of(const S &s) {
    return K2{sp(s.ia02f), sp(s.ia12f), sp(s.c3H0f), sp(s.c3H1f), sp(s.hf), sp(s.dtf), sp(s.inv_dx2f), sp(s.dnf)};
}

// Sweep A / E0 on both sites (site_a32).
template <int MODE, typename S>
__device__ __forceinline__ void site_a(const LatticeConsts &c, const S &s, const K2 &k, const Nb &fp, const Nb &fc,
                                       const Nb &dp, const Nb &dc, Mom &m, F2 (&s0)[kSrc], F2 (&s1)[kSrc]) {
    const Nb *f0[2] = {&fp, &fc}, *d0[2] = {&dp, &dc};
    F2 f1c[2];
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const Nb &ff = *f0[f], &dd = *d0[f];
        const F2 lap0 = lap(ff, k.inv_dx2);
        const F2 d = dd.v[0];
        m.a[f] = m.a[f] + d;
        m.b = fma(d, d, m.b);
        m.g0 = fma(ff.v[0], lap0, m.g0);
        if constexpr (MODE != MODE_E0) {
            const Nb f1 = axpy(ff, k.h, dd);
            f1c[f] = f1.v[0];
            const F2 Pd = fma(k.h, fma(lap0, k.ia02, neg(dv_diff(s.m0, c.model, f, fp.v[0], fc.v[0]))), d);
            m.c[f] = m.c[f] + Pd;
            m.e = fma(Pd, Pd, m.e);
            m.f = fma(Pd, d, m.f);
            m.g1 = fma(f1.v[0], lap(f1, k.inv_dx2), m.g1);
            if constexpr (MODE == MODE_A_GW) {
                source_add(k.dn, ff, s0);
                source_add(k.dn, f1, s1);
            }
        }
    }
    m.v0 = m.v0 + v_diff(s.m0, c.model, fp.v[0], fc.v[0]);
    if constexpr (MODE != MODE_E0) m.v1 = m.v1 + v_diff(s.m1, c.model, f1c[0], f1c[1]);
}

// Sweep B on both sites (site_b32): new fields xo and momenta dout.
template <typename S>
__device__ __forceinline__ void site_b(const LatticeConsts &c, const S &s, const K2 &k, const Nb &fp, const Nb &fc,
                                       const Nb &dp, const Nb &dc, F2 (&xo)[2], F2 (&dout)[2]) {
    const Nb *f0[2] = {&fp, &fc}, *d0[2] = {&dp, &dc};
    const Nb f1[2] = {axpy(fp, k.h, dp), axpy(fc, k.h, dc)};
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const Nb &ff = *f0[f], &dd = *d0[f];
        const F2 lap0 = lap(ff, k.inv_dx2);
        const F2 dd0 = fma(neg(k.c3H0), dd.v[0], fma(lap0, k.ia02, neg(dv_diff(s.m0, c.model, f, fp.v[0], fc.v[0]))));
        const F2 d1c = fma(k.h, dd0, dd.v[0]);
        const F2 lap1 = lap(f1[f], k.inv_dx2);
        const F2 dd1 = fma(neg(k.c3H1), d1c, fma(lap1, k.ia12, neg(dv_diff(s.m1, c.model, f, f1[0].v[0], f1[1].v[0]))));
        xo[f] = fma(k.dt, d1c, ff.v[0]);
        dout[f] = fma(k.dt, dd1, dd.v[0]);
    }
}

}  // namespace s2
}  // namespace gabe
