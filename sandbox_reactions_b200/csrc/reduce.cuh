// reduce.cuh — deterministic grid-wide FP64 sums in a single launch.
//
// Every CTA reduces its threads' values (warp shuffles, then the warps in order) and stores one partial per value;
// the CTA that arrives last (a ticket counter) sums every CTA's partials in CTA order and writes the totals, then
// re-arms the counter for the next launch on the stream. The order of every addition depends only on indices, so the
// result is bit-identical from run to run (no float atomics).
#pragma once

#include <cuda_runtime.h>

template <int K>
__device__ __forceinline__ bool grid_sum_last(const double (&v)[K], double* part, unsigned* counter, double* out) {
    __shared__ double red[K][32];
    __shared__ bool last;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthreads = blockDim.x * blockDim.y;
    const int lane = tid & 31, warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
    const unsigned nb = gridDim.x * gridDim.y;
    const unsigned b = blockIdx.y * gridDim.x + blockIdx.x;
#pragma unroll
    for (int q = 0; q < K; q++) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[q][warp] = x;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) {
            double t = 0.0;
            for (int w = 0; w < nwarps; w++) t += red[q][w];
            part[(size_t)q * nb + b] = t;
        }
        __threadfence();
        const unsigned ticket = atomicAdd(counter, 1u);
        last = ticket == nb - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < K; q++) {
        double x = 0.0;
        for (unsigned i = tid; i < nb; i += nthreads) x += __ldcg(part + (size_t)q * nb + i);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[q][warp] = x;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) {
            double t = 0.0;
            for (int w = 0; w < nwarps; w++) t += red[q][w];
            out[q] = t;
        }
        *counter = 0u;
    }
    return true;
}

// One value.
// Returns true in the last CTA (after the totals are written).
__device__ __forceinline__ bool grid_sum_last1(double v, double* part, unsigned* counter, double* out) {
    const double a[1] = {v};
    return grid_sum_last<1>(a, part, counter, out);
}
