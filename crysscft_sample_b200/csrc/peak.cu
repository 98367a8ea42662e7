// FP64 throughput probe: the denominator of the FP64 roofline reported by bench.py.
// A grid of 2 CTAs x 512 threads per SM runs independent chains of FP64 FMAs (SIMT)
// and of m8n8k4 FP64 tensor-core MMAs; both are timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/crysscft_b200.h"

namespace {

__global__ void peak_dfma(double* out, int iters) {
    double a[16];
    const double x = threadIdx.x * 1e-9, y = 1.0000001;
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = i * 1e-3;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < 16; ++i) a[i] = fma(a[i], y, x);
    double s = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) s += a[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void peak_dmma(double* out, int iters) {
    double d[8][2];
    const double av = threadIdx.x * 1e-9, bv = 1e-9;
#pragma unroll
    for (int i = 0; i < 8; ++i) d[i][0] = d[i][1] = 0;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(d[i][0]), "+d"(d[i][1])
                         : "d"(av), "d"(bv));
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += d[i][0] + d[i][1];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int scft_measure_fp64_peak(int device, double* tflops_simt, double* tflops_tensor) {
    if (!tflops_simt || !tflops_tensor) return SCFT_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SCFT_ERR_NO_DEVICE;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return SCFT_ERR_CUDA;
    const int threads = 512, blocks = 2 * sms, iters = 4096;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * (size_t)blocks * threads) != cudaSuccess) return SCFT_ERR_ALLOC;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms = 0.f;
    peak_dfma<<<blocks, threads>>>(out, 64);
    cudaEventRecord(e0);
    peak_dfma<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    *tflops_simt = 2.0 * 16 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
    peak_dmma<<<blocks, threads>>>(out, 64);
    cudaEventRecord(e0);
    peak_dmma<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    *tflops_tensor = 2.0 * 8 * 256 * iters * (double)blocks * (threads / 32) / (ms * 1e-3) / 1e12;
    const cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e == cudaSuccess ? SCFT_OK : SCFT_ERR_CUDA;
}
