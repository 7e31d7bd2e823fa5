// The split of N planes (or ky columns) over W ranks used by the slab
// decomposition (slab.cu, slabgw.cuh; gabe_b200.slab.split_planes): rank r
// owns [p0(r), p0(r) + n(r)) with n(r) = N/W + (r < N%W), contiguous.
#pragma once

namespace gabe {

struct Split {
    int base, extra;  // N / W, N % W
    __host__ __device__ Split(int N, int W) : base(N / W), extra(N % W) {}
    __host__ __device__ int n(int r) const { return base + (r < extra ? 1 : 0); }
    __host__ __device__ int p0(int r) const { return r * base + (r < extra ? r : extra); }
    __host__ __device__ int owner(int x) const {
        const int big = extra * (base + 1);
        return x < big ? x / (base + 1) : extra + (x - big) / base;
    }
};

}  // namespace gabe
