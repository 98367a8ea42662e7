// Axis-pass kernels: apply a 1-D operator along one axis of a C-ordered 3-D grid,
// with the Boltzmann factor exp(-w ds/2) fused into the load of the first pass and
// into the store of the last pass of a triplet.
//
// A triplet of any of the three solvers is T = A_x (x) A_y (x) A_z on its physical
// grid (see operators.cpp), so one contour step q(s+1) = D T(D q(s)) with
// D = diag(exp(-w ds/2)) (src/crysSCFT_sample.cpp:387-395) is three passes:
//   z pass: t1[o][i]       = sum_j A_z[i][j] (D q)[o][j]          (o = x*ny + y)
//   y pass: t2[x][i][z]    = sum_j A_y[i][j] t1[x][j][z]
//   x pass: q'[i][yz]      = D * sum_j A_x[i][j] t2[j][yz]
// An operator that is a sum of Kronecker products runs the three passes once per
// term; the x passes after the first add into q' (ChainIO::accum) and the last one
// applies D.
// Each pass is a batch of small GEMMs tiled through shared memory.  Both contour
// chains of an SCFT iteration (forward q and backward q+) run in one launch
// (blockIdx.z selects the chain).
#pragma once
#include <cuda_runtime.h>

namespace crysscft {

template <typename T>
struct ChainIO {
    const T* in;
    T* out;
    const T* pre;   // multiply the input by pre[] elementwise (nullptr: no)
    const T* post;  // multiply the output by post[] elementwise (nullptr: no)
    int accum = 0;  // add the pass result to what out[] holds (before post)
};

template <typename T>
struct AxisPass {
    ChainIO<T> ch[2];
    const T* op;   // row-major n x n: out[i] = sum_j op[i*n + j] in[j]
    const T* opT;  // its transpose (row-major)
    int n;         // axis length
    long long outer;  // number of [n][inner] blocks (strided form) / number of rows (contiguous form)
    long long inner;  // axis stride (strided form)
};

__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }

// Strided axis (x or y): view [outer][n][inner], output tile = BM operator rows x BN inner columns.
template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
axis_strided_kernel(const AxisPass<T> p) {
    constexpr int NTX = BN / TN;
    constexpr int NT = NTX * (BM / TM);
    __shared__ __align__(16) T As[BK][BM + 2];  // As[k][m] = op[i0+m][k0+k]
    __shared__ __align__(16) T Bs[BK][BN + 2];  // Bs[k][c] = pre * in[o][k0+k][r0+c]

    const long long zc = blockIdx.z;
    const int chain = (int)(zc / p.outer);
    const long long o = zc - (long long)chain * p.outer;
    const int n = p.n;
    const long long inner = p.inner;
    const int i0 = blockIdx.y * BM;
    const long long r0 = (long long)blockIdx.x * BN;
    const ChainIO<T> io = p.ch[chain];
    const long long base = o * (long long)n * inner;
    const T* in = io.in + base;
    const T* pre = io.pre ? io.pre + base : nullptr;
    const int tid = threadIdx.x;
    const int tx = tid % NTX, ty = tid / NTX;

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    for (int k0 = 0; k0 < n; k0 += BK) {
        for (int e = tid; e < BM * BK; e += NT) {
            const int m = e / BK, k = e - (e / BK) * BK;
            const int gi = i0 + m, gk = k0 + k;
            As[k][m] = (gi < n && gk < n) ? p.op[(size_t)gi * n + gk] : T(0);
        }
        for (int e = tid; e < BK * BN; e += NT) {
            const int k = e / BN, c = e - (e / BN) * BN;
            const int gk = k0 + k;
            const long long gr = r0 + c;
            T v = T(0);
            if (gk < n && gr < inner) {
                const long long idx = (long long)gk * inner + gr;
                v = in[idx];
                if (pre) v = v * pre[idx];
            }
            Bs[k][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[k][ty * TM + i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[k][tx * TN + j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fma_t(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }

    T* out = io.out + base;
    const T* post = io.post ? io.post + base : nullptr;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gi = i0 + ty * TM + i;
        if (gi >= n) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const long long gr = r0 + tx * TN + j;
            if (gr >= inner) continue;
            const long long idx = (long long)gi * inner + gr;
            T v = acc[i][j];
            if (io.accum) v = v + out[idx];
            if (post) v = v * post[idx];
            out[idx] = v;
        }
    }
}

// Contiguous axis (z): rows of n contiguous elements; output tile = BM rows x BN operator rows.
template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
axis_contig_kernel(const AxisPass<T> p) {
    constexpr int NTX = BN / TN;
    constexpr int NT = NTX * (BM / TM);
    __shared__ __align__(16) T As[BK][BM + 2];  // As[k][m] = pre * in[o0+m][k0+k]
    __shared__ __align__(16) T Bs[BK][BN + 2];  // Bs[k][c] = opT[k0+k][i0+c] = op[i0+c][k0+k]

    const int chain = blockIdx.z;
    const int n = p.n;
    const long long rows = p.outer;
    const long long o0 = (long long)blockIdx.y * BM;
    const int i0 = blockIdx.x * BN;
    const ChainIO<T> io = p.ch[chain];
    const int tid = threadIdx.x;
    const int tx = tid % NTX, ty = tid / NTX;

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    for (int k0 = 0; k0 < n; k0 += BK) {
        for (int e = tid; e < BM * BK; e += NT) {
            const int m = e / BK, k = e - (e / BK) * BK;
            const long long go = o0 + m;
            const int gk = k0 + k;
            T v = T(0);
            if (go < rows && gk < n) {
                const long long idx = go * n + gk;
                v = io.in[idx];
                if (io.pre) v = v * io.pre[idx];
            }
            As[k][m] = v;
        }
        for (int e = tid; e < BK * BN; e += NT) {
            const int k = e / BN, c = e - (e / BN) * BN;
            const int gk = k0 + k, gi = i0 + c;
            Bs[k][c] = (gk < n && gi < n) ? p.opT[(size_t)gk * n + gi] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[k][ty * TM + i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[k][tx * TN + j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fma_t(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const long long go = o0 + ty * TM + i;
        if (go >= rows) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gi = i0 + tx * TN + j;
            if (gi >= n) continue;
            const long long idx = go * n + gi;
            T v = acc[i][j];
            if (io.accum) v = v + io.out[idx];
            if (io.post) v = v * io.post[idx];
            io.out[idx] = v;
        }
    }
}

}  // namespace crysscft
