// Kernels of the cell-length derivative (stress) of ln Q, computed from the stored
// contour of the last iteration by the adjoint identity
//   dQ/dL_a = (1/M) sum_t < q+[t+1], D_t (dT/dL_a) D_t q[t] >,
// where q (forward) and q+ (backward) are the two contour stores and D_t is the
// Boltzmann factor of segment t.  Every term is independent, so slices are processed
// in large batches through the per-axis kernels.
#pragma once
#include <cuda_runtime.h>

#include "field_kernels.cuh"

namespace crysscft {

// X[i][r] = D[r] * q[(t0 + i) M + r] for i < nt.  T: the stored contour's type (FP32 when
// the last iteration ran the precision form); the derivative triplets run in FP64.
template <typename T>
__global__ void stress_scale_kernel(double* __restrict__ X, const T* __restrict__ q,
                                    const T* __restrict__ D, long long t0, long long nt, long long M) {
    const long long total = nt * M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / M, r = e - i * M;
        X[e] = (double)D[r] * (double)q[(t0 + i) * M + r];
    }
}

// partials[block] = sum_{i < nt, r < M} qc[(t0 + i + 1) M + r] * D[r] * Y[i M + r]
// (deterministic: fixed grid, fixed in-block order; the host sums the partials in order)
template <typename T>
__global__ void __launch_bounds__(kRedThreads)
stress_dot_kernel(const T* __restrict__ qc, const T* __restrict__ D, const double* __restrict__ Y,
                  long long t0, long long nt, long long M, double* __restrict__ partials) {
    __shared__ double sh[kRedThreads / 32];
    const long long total = nt * M;
    double s = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / M, r = e - i * M;
        s += (double)qc[(t0 + i + 1) * M + r] * (double)D[r] * Y[e];
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// partials[4 b + 0] = sum phiA phiB, partials[4 b + 1] = sum (1 - phiA - phiB)
__global__ void __launch_bounds__(kRedThreads)
dxn_terms_kernel(const double* __restrict__ phiA, const double* __restrict__ phiB, long long M,
                 double* __restrict__ partials) {
    __shared__ double sh[kRedThreads / 32];
    double ab = 0.0, inc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
        ab += phiA[i] * phiB[i];
        inc += 1 - phiA[i] - phiB[i];
    }
    ab = block_sum(ab, sh);
    inc = block_sum(inc, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = ab;
        partials[2 * blockIdx.x + 1] = inc;
    }
}

}  // namespace crysscft
