// In-register FFT building blocks of the library's transforms (fft3d.cuh,
// fftt.cuh): complex helpers, radix-2 DFTs of up to 32 points held in
// registers, and the four-step split N = L1 L2 used to transform a line of N
// points in shared memory (L2-point FFTs over n2 at stride L1, twiddles
// W_N^(n1 k2), L1-point FFTs over n1, output k = k2 + L2 k1).  Forward sign
// e^{-i}, unnormalised: FFTW's convention, which the reference's transforms
// use (g2evolutionpert.cpp:183-195, g2spectra.cpp:47-61).
#pragma once

#include "common.cuh"

namespace gabe {
namespace pfft {

// cos(pi m / 16) for m = 0..8 (the real parts of the 32nd roots of unity).
constexpr double kCos16[9] = {1.0,
                              0.98078528040323044913,
                              0.92387953251128675613,
                              0.83146961230254523708,
                              0.70710678118654752440,
                              0.55557023301960222474,
                              0.38268343236508977173,
                              0.19509032201612826785,
                              0.0};
__host__ __device__ constexpr double cos32(int m) {
    m &= 31;
    if (m > 16) m = 32 - m;
    return m <= 8 ? kCos16[m] : -kCos16[16 - m];
}
__host__ __device__ constexpr double sin32(int m) { return cos32(8 - m); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// v * W_32^M, W_32 = exp(-2 pi i / 32), with M known at compile time.
template <int M>
__device__ __forceinline__ float2 mulw(float2 v) {
    constexpr int m = M & 31;
    if constexpr (m == 0) {
        return v;
    } else if constexpr (m == 8) {
        return make_float2(v.y, -v.x);
    } else if constexpr (m == 16) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (m == 24) {
        return make_float2(-v.y, v.x);
    } else {
        constexpr float c = (float)cos32(m), s = (float)sin32(m);
        return make_float2(v.x * c + v.y * s, v.y * c - v.x * s);
    }
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
__host__ __device__ constexpr int bitrev(int x, int bits) {
    int r = 0;
    for (int b = 0; b < bits; b++) r = (r << 1) | ((x >> b) & 1);
    return r;
}

template <int R, int I>
__device__ __forceinline__ void bitrev_swap(float2 (&x)[R]) {
    if constexpr (I < R) {
        constexpr int J = bitrev(I, ilog2(R));
        if constexpr (J > I) {
            const float2 t = x[I];
            x[I] = x[J];
            x[J] = t;
        }
        bitrev_swap<R, I + 1>(x);
    }
}

template <int R, int LEN, int J>
__device__ __forceinline__ void butterflies(float2 (&x)[R]) {
    if constexpr (J < LEN / 2) {
#pragma unroll
        for (int i = 0; i < R; i += LEN) {
            const float2 u = x[i + J], v = mulw<J * (32 / LEN)>(x[i + J + LEN / 2]);
            x[i + J] = cadd(u, v);
            x[i + J + LEN / 2] = csub(u, v);
        }
        butterflies<R, LEN, J + 1>(x);
    }
}

template <int R, int LEN>
__device__ __forceinline__ void stages(float2 (&x)[R]) {
    if constexpr (LEN <= R) {
        butterflies<R, LEN, 0>(x);
        stages<R, 2 * LEN>(x);
    }
}

// In-register forward DFT of R <= 32 points, natural order in and out
// (radix-2 decimation in time).
template <int R>
__device__ __forceinline__ void fft_reg(float2 (&x)[R]) {
    static_assert(R >= 2 && R <= 32 && (R & (R - 1)) == 0, "R must be a power of two in [2, 32]");
    bitrev_swap<R, 0>(x);
    stages<R, 2>(x);
}

// Four-step split N = L1 L2 per line length.
template <int N>
struct FourStep;
template <>
struct FourStep<512> {
    static constexpr int L1 = 32, L2 = 16;
};
template <>
struct FourStep<256> {
    static constexpr int L1 = 16, L2 = 16;
};
template <>
struct FourStep<128> {
    static constexpr int L1 = 16, L2 = 8;
};
template <>
struct FourStep<64> {
    static constexpr int L1 = 8, L2 = 8;
};

}  // namespace pfft
}  // namespace gabe
