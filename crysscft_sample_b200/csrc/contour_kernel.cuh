// Persistent whole-contour kernel (FP64): all steps of one or two propagator chains
// in one cooperative launch, one CTA per SM, the three per-axis operators resident in
// shared memory, FP64 tensor-core tiles (mma.sync m8n8k4 .f64, DMMA).
//
// One contour step q(s+1) = D T(D q(s)) (src/crysSCFT_sample.cpp:387-395) with
// T = A_x (x) A_y (x) A_z runs as two phases separated by a grid barrier:
//   phase P, one unit per (chain, x-plane): load the ny x nz plane times D, apply A_z
//            along rows and A_y along columns in shared memory, store to the chain's
//            exchange buffer;
//   phase Q, one unit per (chain, y-plane): load the nx x nz slab of the exchange
//            buffer, apply A_x along columns, multiply by D, store q(s+1).
// Centrosymmetric operators (PMMM and P1: A[n-1-i][n-1-j] = A[i][j]) are applied in
// even/odd form: u = x_j + x_{n-1-j}, v = x_j - x_{n-1-j}, p = E u, r = O v,
// y_i = p_i + r_i, y_{n-1-i} = p_i - r_i, which halves the multiply-adds.
//
// Grid barriers count arrivals on a counter that the host zeroes before each launch;
// every wait is bounded (spin limit), after which the kernel records an error and
// returns, so a lost block can never hang the GPU.
#pragma once
#include <cuda_runtime.h>

namespace crysscft {

constexpr int kContourThreads = 256;
constexpr int kContourMaxN = 64;

struct ContourArgs {
    double* q[2];           // contour storage of each chain
    const double* wds[2];   // Boltzmann factors of block A (segments < NsA) and block B
    double* xbuf[2];        // exchange buffer of each chain (space_size_phy)
    const double* ops;      // packed operators (see op_off / op_ld)
    int n[3];               // physical grid nx, ny, nz
    int eo[3];              // 1: even/odd (E then O blocks), 0: full n x n
    int op_off[3];          // offset (doubles) of each axis' operator block in ops
    int op_ld[3];           // leading dimension of each axis' matrices
    int op_half[3];         // offset from E to O (eo axes)
    int ops_total;          // doubles to stage into shared memory
    int nchain;             // 1 or 2
    long long slot0[2];     // first input slot of each chain
    int dir[2];             // +1 or -1
    long long NsA;          // segments with index < NsA use wds[0], the rest wds[1]
    int t_begin, t_end;     // steps of this launch
    unsigned* bar_count;    // zeroed by the host before each launch
    int* error;             // bit 0: barrier wait gave up
    long long spin_limit;
};

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Arrive, then wait until `target` arrivals are counted.  Returns false if this or any
// other block recorded an error (including a wait that ran out of spins).
__device__ __forceinline__ bool grid_barrier(unsigned* count, int* error, unsigned target, long long spin_limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        long long spins = 0;
        int ok = 1;
        while (ld_acquire_u32(count) < target) {
            if (++spins > spin_limit) {
                atomicOr(error, 1);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        if (*((volatile int*)error) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// rows x cols field slab between global (row stride gs, 16-byte aligned rows) and shared
// memory (row stride lf); optional elementwise factor w (same global indexing).
template <bool TO_SMEM>
__device__ __forceinline__ void move_slab(double* sm, int lf, double* gm, long long gs, const double* w, int rows,
                                          int cols) {
    const int per_row = cols >> 1;
    const int total = rows * per_row;
    constexpr int U = 8;
    for (int base = 0; base < total; base += kContourThreads * U) {
        double2 v[U];
        double2 f[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const int e = base + k * kContourThreads + threadIdx.x;
            if (e < total) {
                const int r = e / per_row, c = (e - r * per_row) * 2;
                if (TO_SMEM) v[k] = *reinterpret_cast<const double2*>(gm + r * gs + c);
                else v[k] = *reinterpret_cast<const double2*>(sm + r * lf + c);
                if (w) f[k] = __ldg(reinterpret_cast<const double2*>(w + r * gs + c));
            }
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const int e = base + k * kContourThreads + threadIdx.x;
            if (e < total) {
                const int r = e / per_row, c = (e - r * per_row) * 2;
                double2 x = v[k];
                if (w) {
                    x.x = x.x * f[k].x;
                    x.y = x.y * f[k].y;
                }
                if (TO_SMEM) *reinterpret_cast<double2*>(sm + r * lf + c) = x;
                else *reinterpret_cast<double2*>(gm + r * gs + c) = x;
            }
        }
    }
}

// G[r][i] = sum_j F[r][j] A[i][j]  (operator along the contiguous direction; R x C slab)
template <bool EO>
__device__ __forceinline__ void row_op(const double* F, double* G, int R, int C, int lf, const double* opE,
                                       const double* opO, int lo) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int NI = EO ? C / 2 : C;  // operator rows computed
    const int K = EO ? C / 2 : C;
    const int tm = R >> 3, tn = NI >> 3;
    const int bm = (tm + 1) >> 1, bn = (tn + 1) >> 1;
    for (int blk = warp; blk < bm * bn; blk += kContourThreads / 32) {
        const int mb = (blk / bn) * 2, nb = (blk % bn) * 2;
        const bool m1 = mb + 1 < tm, n1 = nb + 1 < tn;
        double dP[2][2][2], dR[2][2][2];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) dP[a][b][0] = dP[a][b][1] = dR[a][b][0] = dR[a][b][1] = 0.0;
        for (int k0 = 0; k0 < K; k0 += 4) {
            const int j = k0 + t;
            double aU[2], aV[2], bE[2], bO[2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int r = (mb + a) * 8 + g;
                if (a == 0 || m1) {
                    const double x0 = F[r * lf + j];
                    if (EO) {
                        const double x1 = F[r * lf + (C - 1 - j)];
                        aU[a] = x0 + x1;
                        aV[a] = x0 - x1;
                    } else {
                        aU[a] = x0;
                        aV[a] = 0.0;
                    }
                } else {
                    aU[a] = aV[a] = 0.0;
                }
            }
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int i = (nb + b) * 8 + g;
                if (b == 0 || n1) {
                    bE[b] = opE[i * lo + j];
                    bO[b] = EO ? opO[i * lo + j] : 0.0;
                } else {
                    bE[b] = bO[b] = 0.0;
                }
            }
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    if ((a == 0 || m1) && (b == 0 || n1)) {
                        dmma884(dP[a][b], aU[a], bE[b]);
                        if (EO) dmma884(dR[a][b], aV[a], bO[b]);
                    }
                }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if (!((a == 0 || m1) && (b == 0 || n1))) continue;
                const int r = (mb + a) * 8 + g;
                const int i = (nb + b) * 8 + 2 * t;
                if (EO) {
                    *reinterpret_cast<double2*>(G + r * lf + i) =
                        make_double2(dP[a][b][0] + dR[a][b][0], dP[a][b][1] + dR[a][b][1]);
                    *reinterpret_cast<double2*>(G + r * lf + (C - 2 - i)) =
                        make_double2(dP[a][b][1] - dR[a][b][1], dP[a][b][0] - dR[a][b][0]);
                } else {
                    *reinterpret_cast<double2*>(G + r * lf + i) = make_double2(dP[a][b][0], dP[a][b][1]);
                }
            }
    }
}

// G[i][c] = sum_j A[i][j] F[j][c]  (operator along the row direction; R x C slab)
template <bool EO>
__device__ __forceinline__ void col_op(const double* F, double* G, int R, int C, int lf, const double* opE,
                                       const double* opO, int lo) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int MI = EO ? R / 2 : R;
    const int K = EO ? R / 2 : R;
    const int tm = MI >> 3, tn = C >> 3;
    const int bm = (tm + 1) >> 1, bn = (tn + 1) >> 1;
    for (int blk = warp; blk < bm * bn; blk += kContourThreads / 32) {
        const int mb = (blk / bn) * 2, nb = (blk % bn) * 2;
        const bool m1 = mb + 1 < tm, n1 = nb + 1 < tn;
        double dP[2][2][2], dR[2][2][2];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) dP[a][b][0] = dP[a][b][1] = dR[a][b][0] = dR[a][b][1] = 0.0;
        for (int k0 = 0; k0 < K; k0 += 4) {
            const int j = k0 + t;
            double aE[2], aO[2], bU[2], bV[2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int i = (mb + a) * 8 + g;
                if (a == 0 || m1) {
                    aE[a] = opE[i * lo + j];
                    aO[a] = EO ? opO[i * lo + j] : 0.0;
                } else {
                    aE[a] = aO[a] = 0.0;
                }
            }
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int c = (nb + b) * 8 + g;
                if (b == 0 || n1) {
                    const double x0 = F[j * lf + c];
                    if (EO) {
                        const double x1 = F[(R - 1 - j) * lf + c];
                        bU[b] = x0 + x1;
                        bV[b] = x0 - x1;
                    } else {
                        bU[b] = x0;
                        bV[b] = 0.0;
                    }
                } else {
                    bU[b] = bV[b] = 0.0;
                }
            }
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    if ((a == 0 || m1) && (b == 0 || n1)) {
                        dmma884(dP[a][b], aE[a], bU[b]);
                        if (EO) dmma884(dR[a][b], aO[a], bV[b]);
                    }
                }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if (!((a == 0 || m1) && (b == 0 || n1))) continue;
                const int i = (mb + a) * 8 + g;
                const int c = (nb + b) * 8 + 2 * t;
                if (EO) {
                    *reinterpret_cast<double2*>(G + i * lf + c) =
                        make_double2(dP[a][b][0] + dR[a][b][0], dP[a][b][1] + dR[a][b][1]);
                    *reinterpret_cast<double2*>(G + (R - 1 - i) * lf + c) =
                        make_double2(dP[a][b][0] - dR[a][b][0], dP[a][b][1] - dR[a][b][1]);
                } else {
                    *reinterpret_cast<double2*>(G + i * lf + c) = make_double2(dP[a][b][0], dP[a][b][1]);
                }
            }
    }
}

__device__ __forceinline__ void apply_row_op(int eo, const double* F, double* G, int R, int C, int lf,
                                             const double* ops, int off, int ld, int half) {
    if (eo) row_op<true>(F, G, R, C, lf, ops + off, ops + off + half, ld);
    else row_op<false>(F, G, R, C, lf, ops + off, nullptr, ld);
}
__device__ __forceinline__ void apply_col_op(int eo, const double* F, double* G, int R, int C, int lf,
                                             const double* ops, int off, int ld, int half) {
    if (eo) col_op<true>(F, G, R, C, lf, ops + off, ops + off + half, ld);
    else col_op<false>(F, G, R, C, lf, ops + off, nullptr, ld);
}

__global__ void __launch_bounds__(kContourThreads, 1) contour_kernel_f64(const ContourArgs a) {
    extern __shared__ __align__(16) double smem[];
    const int nx = a.n[0], ny = a.n[1], nz = a.n[2];
    const int lf = nz + 4;
    const int rows = nx > ny ? nx : ny;
    const int ops_pad = (a.ops_total + 1) & ~1;
    double* sops = smem;
    double* F = smem + ops_pad;
    double* G = F + rows * lf;
    for (int i = threadIdx.x; i < a.ops_total; i += kContourThreads) sops[i] = a.ops[i];
    __syncthreads();

    const long long M = (long long)nx * ny * nz;
    const long long plane = (long long)ny * nz;
    const int unitsP = a.nchain * nx, unitsQ = a.nchain * ny;
    unsigned target = 0;
    for (int t = a.t_begin; t < a.t_end; ++t) {
        // ---- phase P: z then y on x-planes ----
        for (int u = blockIdx.x; u < unitsP; u += gridDim.x) {
            const int c = u / nx, x = u - c * nx;
            const int dir = a.dir[c];
            const long long in_slot = a.slot0[c] + (long long)dir * t;
            const long long seg = dir > 0 ? in_slot : in_slot - 1;
            const double* w = a.wds[seg < a.NsA ? 0 : 1];
            move_slab<true>(F, lf, a.q[c] + in_slot * M + x * plane, nz, w ? w + x * plane : nullptr, ny, nz);
            __syncthreads();
            apply_row_op(a.eo[2], F, G, ny, nz, lf, sops, a.op_off[2], a.op_ld[2], a.op_half[2]);
            __syncthreads();
            apply_col_op(a.eo[1], G, F, ny, nz, lf, sops, a.op_off[1], a.op_ld[1], a.op_half[1]);
            __syncthreads();
            move_slab<false>(F, lf, a.xbuf[c] + x * plane, nz, nullptr, ny, nz);
            __syncthreads();
        }
        target += gridDim.x;
        if (!grid_barrier(a.bar_count, a.error, target, a.spin_limit)) return;
        // ---- phase Q: x on y-planes, times D, store q(s+1) ----
        for (int u = blockIdx.x; u < unitsQ; u += gridDim.x) {
            const int c = u / ny, y = u - c * ny;
            const int dir = a.dir[c];
            const long long in_slot = a.slot0[c] + (long long)dir * t;
            const long long out_slot = in_slot + dir;
            const long long seg = dir > 0 ? in_slot : in_slot - 1;
            const double* w = a.wds[seg < a.NsA ? 0 : 1];
            move_slab<true>(F, lf, a.xbuf[c] + (long long)y * nz, plane, nullptr, nx, nz);
            __syncthreads();
            apply_col_op(a.eo[0], F, G, nx, nz, lf, sops, a.op_off[0], a.op_ld[0], a.op_half[0]);
            __syncthreads();
            move_slab<false>(G, lf, a.q[c] + out_slot * M + (long long)y * nz, plane,
                             w ? w + (long long)y * nz : nullptr, nx, nz);
            __syncthreads();
        }
        if (t + 1 < a.t_end) {
            target += gridDim.x;
            if (!grid_barrier(a.bar_count, a.error, target, a.spin_limit)) return;
        }
    }
}

}  // namespace crysscft
