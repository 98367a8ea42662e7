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
#include <cuda.h>  // CUtensorMap (type only)
#include <cuda_runtime.h>

namespace crysscft {

constexpr int kContourThreads = 256;
constexpr int kContourMaxN = 64;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copy an operator block (count values) into shared memory as 16-byte cp.async chunks,
// all in flight at once (a plain load/store loop serialises tens of global round trips
// per thread at every launch); the caller waits with cp_async_wait_all + a barrier.
template <typename T>
__device__ __forceinline__ void op_copy_async(T* sop, const T* op, int count) {
    const int bytes = count * (int)sizeof(T);
    if ((reinterpret_cast<unsigned long long>(op) & 15) == 0 && (smem_u32(sop) & 15) == 0 && (bytes & 15) == 0) {
        for (int i = threadIdx.x; i < bytes / 16; i += kContourThreads)
            cp_async16(reinterpret_cast<char*>(sop) + 16 * i, reinterpret_cast<const char*>(op) + 16 * i);
        cp_async_commit();
    } else {
        for (int i = threadIdx.x; i < count; i += kContourThreads) sop[i] = op[i];
    }
}

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
    unsigned* flags;        // alternating kernel: [chain][plane|slab][consumer][producer] last finished phase + 1, zeroed by the host
    // alternating kernel, fused phi (null: off): sums of q(s) q+(s) per chain, block A|B,
    // layout plane|slab and tile, in panel order ([chain][block][layout][tile][N * N]), and
    // per chain and unit: U/2 once the q stores of phases < U/2 have landed (zeroed by the host)
    double* phi_acc;
    unsigned* done;
    // alternating kernel: Boltzmann and staging tiles in 8-column panels ([z / 8][row][z % 8],
    // rows y in plane tiles, x in slab tiles), [0] plane and [1] slab view; contour store of
    // each chain as (z % 8, row, z / 8, tile, slot), Boltzmann factors of blocks A and B
    // as (z % 8, row, z / 8, tile)
    alignas(64) CUtensorMap tm_pq[2][2];
    alignas(64) CUtensorMap tm_pw[2][2];
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
            if (spins > 256) __nanosleep(32);
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
    op_copy_async(sops, a.ops, a.ops_total);
    cp_async_wait_all();
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

// ---------------------------------------------------------------------------
// Compile-time specialised form of the same kernel for common grids: every size,
// stride and operator offset is a constant, so the tile loops unroll completely.
// ---------------------------------------------------------------------------
namespace crysscft {

template <int N, bool EO>
struct AxisShape {
    static constexpr int K = EO ? N / 2 : N;       // contraction length
    static constexpr int LD = K + 4;               // operator leading dimension
    static constexpr int HALF = EO ? K * LD : 0;   // E -> O offset
    static constexpr int SIZE = EO ? 2 * K * LD : N * LD;
};

// G[r][i] = sum_j F[r][j] A[i][j] on an R x C slab (leading dimension LF)
template <int R, int C, int LF, bool EO>
__device__ __forceinline__ void row_op_ct(const double* __restrict__ F, double* __restrict__ G,
                                          const double* __restrict__ opE) {
    using S = AxisShape<C, EO>;
    const double* opO = opE + S::HALF;
    constexpr int NI = S::K, K = S::K;
    constexpr int TM = R / 8, TN = NI / 8;
    constexpr int BM = (TM + 1) / 2, BN = (TN + 1) / 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int blk = warp; blk < BM * BN; blk += kContourThreads / 32) {
        const int mb = (blk / BN) * 2, nb = (blk % BN) * 2;
        const bool m1 = (TM % 2 == 0) || (mb + 1 < TM);
        const bool n1 = (TN % 2 == 0) || (nb + 1 < TN);
        double dP[2][2][2] = {}, dR[2][2][2] = {};
        const double* Fr0 = F + (mb * 8 + g) * LF + t;
        const double* Fr1 = Fr0 + 8 * LF;
        const double* E0 = opE + (nb * 8 + g) * S::LD + t;
        const double* E1 = E0 + 8 * S::LD;
        const double* O0 = opO + (nb * 8 + g) * S::LD + t;
        const double* O1 = O0 + 8 * S::LD;
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 4) {
            double aU[2], aV[2];
            {
                const double x0 = Fr0[k0];
                const double x1 = EO ? Fr0[C - 1 - 2 * t - k0] : 0.0;
                aU[0] = EO ? x0 + x1 : x0;
                aV[0] = x0 - x1;
            }
            if (m1) {
                const double x0 = Fr1[k0];
                const double x1 = EO ? Fr1[C - 1 - 2 * t - k0] : 0.0;
                aU[1] = EO ? x0 + x1 : x0;
                aV[1] = x0 - x1;
            } else {
                aU[1] = aV[1] = 0.0;
            }
            const double bE0 = E0[k0];
            const double bE1 = n1 ? E1[k0] : 0.0;
            dmma884(dP[0][0], aU[0], bE0);
            if (n1) dmma884(dP[0][1], aU[0], bE1);
            if (m1) dmma884(dP[1][0], aU[1], bE0);
            if (m1 && n1) dmma884(dP[1][1], aU[1], bE1);
            if (EO) {
                const double bO0 = O0[k0];
                const double bO1 = n1 ? O1[k0] : 0.0;
                dmma884(dR[0][0], aV[0], bO0);
                if (n1) dmma884(dR[0][1], aV[0], bO1);
                if (m1) dmma884(dR[1][0], aV[1], bO0);
                if (m1 && n1) dmma884(dR[1][1], aV[1], bO1);
            }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if ((a == 1 && !m1) || (b == 1 && !n1)) continue;
                const int r = (mb + a) * 8 + g;
                const int i = (nb + b) * 8 + 2 * t;
                if (EO) {
                    *reinterpret_cast<double2*>(G + r * LF + i) =
                        make_double2(dP[a][b][0] + dR[a][b][0], dP[a][b][1] + dR[a][b][1]);
                    *reinterpret_cast<double2*>(G + r * LF + (C - 2 - i)) =
                        make_double2(dP[a][b][1] - dR[a][b][1], dP[a][b][0] - dR[a][b][0]);
                } else {
                    *reinterpret_cast<double2*>(G + r * LF + i) = make_double2(dP[a][b][0], dP[a][b][1]);
                }
            }
    }
}

// Where col_op_ct writes its result G[i][c]: kToSmem, a shared-memory slab (row stride LF);
// kToGlobal, the global exchange buffer (row stride gs), straight from the MMA
// accumulators, so the stores overlap the other warps' tiles.
// kFinish (two-level kernel): the result y finishes a contour step: q = y W0 goes to the
// panel staging tile qs (stored from there by TMA) and, if start, q W1 to the slab G.
enum ColEpilogue { kToSmem = 0, kToGlobal = 1, kFinish = 2 };

struct ColOut {
    double* G;
    long long gs;  // kToGlobal: row stride of G
    const double* w0 = nullptr;  // kFinish: Boltzmann tiles of the finished / next step (panels)
    const double* w1 = nullptr;
    double* qs = nullptr;        // kFinish: staging tile of q (panels)
    int start = 0;               // kFinish: a next step follows
};

// element (i, c) of a tile with PR rows stored in 8-column panels
template <int PR>
__device__ __forceinline__ int panel_index(int i, int c) {
    return ((c >> 3) * PR + i) * 8 + (c & 7);
}

template <int LF, int EPI, int PR = 0>
__device__ __forceinline__ void col_store(const ColOut& o, int i, int c, double v0, double v1) {
    if constexpr (EPI == kToSmem) {
        *reinterpret_cast<double2*>(o.G + i * LF + c) = make_double2(v0, v1);
    } else if constexpr (EPI == kToGlobal) {
        *reinterpret_cast<double2*>(o.G + i * o.gs + c) = make_double2(v0, v1);
    } else {
        const int pi = panel_index<PR>(i, c);
        const double2 w0 = *reinterpret_cast<const double2*>(o.w0 + pi);
        v0 = v0 * w0.x;
        v1 = v1 * w0.y;
        *reinterpret_cast<double2*>(o.qs + pi) = make_double2(v0, v1);
        if (o.start) {
            const double2 w1 = *reinterpret_cast<const double2*>(o.w1 + pi);
            *reinterpret_cast<double2*>(o.G + i * LF + c) = make_double2(v0 * w1.x, v1 * w1.y);
        }
    }
}

// G[i][c] = sum_j A[i][j] F[j][c] on an R x C slab (leading dimension LF); EPI selects
// where the result goes (ColEpilogue)
template <int R, int C, int LF, bool EO, int EPI = kToSmem>
__device__ __forceinline__ void col_op_ct(const double* __restrict__ F, const ColOut& out,
                                          const double* __restrict__ opE) {
    using S = AxisShape<R, EO>;
    const double* opO = opE + S::HALF;
    constexpr int MI = S::K, K = S::K;
    constexpr int TM = MI / 8, TN = C / 8;
    constexpr int BM = (TM + 1) / 2, BN = (TN + 1) / 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int blk = warp; blk < BM * BN; blk += kContourThreads / 32) {
        const int mb = (blk / BN) * 2, nb = (blk % BN) * 2;
        const bool m1 = (TM % 2 == 0) || (mb + 1 < TM);
        const bool n1 = (TN % 2 == 0) || (nb + 1 < TN);
        double dP[2][2][2] = {}, dR[2][2][2] = {};
        const double* E0 = opE + (mb * 8 + g) * S::LD + t;
        const double* E1 = E0 + 8 * S::LD;
        const double* O0 = opO + (mb * 8 + g) * S::LD + t;
        const double* O1 = O0 + 8 * S::LD;
        const double* Fc0 = F + t * LF + nb * 8 + g;         // F[j][c], j = k0 + t
        const double* Fm0 = F + (R - 1 - t) * LF + nb * 8 + g;  // F[R-1-j][c]
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 4) {
            double bU[2], bV[2];
            {
                const double x0 = Fc0[k0 * LF];
                const double x1 = EO ? Fm0[-k0 * LF] : 0.0;
                bU[0] = EO ? x0 + x1 : x0;
                bV[0] = x0 - x1;
            }
            if (n1) {
                const double x0 = Fc0[k0 * LF + 8];
                const double x1 = EO ? Fm0[-k0 * LF + 8] : 0.0;
                bU[1] = EO ? x0 + x1 : x0;
                bV[1] = x0 - x1;
            } else {
                bU[1] = bV[1] = 0.0;
            }
            const double aE0 = E0[k0];
            const double aE1 = m1 ? E1[k0] : 0.0;
            dmma884(dP[0][0], aE0, bU[0]);
            if (n1) dmma884(dP[0][1], aE0, bU[1]);
            if (m1) dmma884(dP[1][0], aE1, bU[0]);
            if (m1 && n1) dmma884(dP[1][1], aE1, bU[1]);
            if (EO) {
                const double aO0 = O0[k0];
                const double aO1 = m1 ? O1[k0] : 0.0;
                dmma884(dR[0][0], aO0, bV[0]);
                if (n1) dmma884(dR[0][1], aO0, bV[1]);
                if (m1) dmma884(dR[1][0], aO1, bV[0]);
                if (m1 && n1) dmma884(dR[1][1], aO1, bV[1]);
            }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if ((a == 1 && !m1) || (b == 1 && !n1)) continue;
                const int i = (mb + a) * 8 + g;
                const int c = (nb + b) * 8 + 2 * t;
                if (EO) {
                    col_store<LF, EPI, R>(out, i, c, dP[a][b][0] + dR[a][b][0], dP[a][b][1] + dR[a][b][1]);
                    col_store<LF, EPI, R>(out, R - 1 - i, c, dP[a][b][0] - dR[a][b][0], dP[a][b][1] - dR[a][b][1]);
                } else {
                    col_store<LF, EPI, R>(out, i, c, dP[a][b][0], dP[a][b][1]);
                }
            }
    }
}

// col_op_ct into a shared-memory slab G
template <int R, int C, int LF, bool EO>
__device__ __forceinline__ void col_op_ct(const double* __restrict__ F, double* __restrict__ G,
                                          const double* __restrict__ opE) {
    const ColOut o{G, 0};
    col_op_ct<R, C, LF, EO, kToSmem>(F, o, opE);
}

// ---- two even/odd levels (PMMM operators, n = 64 and 128) -----------------------------
// For the PMMM operator the even half E = (A[i][j] + A[i][n-1-j]) / 2 is itself
// centrosymmetric (it keeps only even frequencies: a DCT pair of half the size), so p = E u
// splits again: ue = u_j + u_{h-1-j}, uo = u_j - u_{h-1-j} (j < h/2), pe = EE ue,
// po = EO uo, p_i = pe_i + po_i, p_{h-1-i} = pe_i - po_i.  The odd half O stays dense.
// Per warp: 16 rows (or columns) x 8 pair indices i and their three mirrors; 3/4 of the
// DMMA of one level.  Operator block: [EE | EO] (h/2 x h/2, ld h/2 + 4), then O (h x h,
// ld h + 4).
template <int N>
struct AxisShapeEO2 {
    static constexpr int H = N / 2, H2 = N / 4;
    static constexpr int LD2 = H2 + 4, LD = H + 4;
    static constexpr int OFF_EO = H2 * LD2, OFF_O = 2 * H2 * LD2;
    static constexpr int SIZE = OFF_O + H * LD;
    static constexpr int GROUPS = H2 / 8;  // groups of 8 pair indices
};

// G[r][i] = sum_j F[r][j] A[i][j] on an R x C slab (two even/odd levels); warp =
// (16-row block, group of 8 pair indices), (R / 16) x (C / 32) warps
template <int R, int C, int LF>
__device__ __forceinline__ void row_op_eo2(const double* __restrict__ F, double* __restrict__ G,
                                           const double* __restrict__ op) {
    using S = AxisShapeEO2<C>;
    static_assert((R / 16) * S::GROUPS == kContourThreads / 32 && R % 16 == 0 && S::H2 % 8 == 0,
                  "one warp per 16 rows x 8 pair indices");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rb = warp / S::GROUPS, hh = warp % S::GROUPS;
    const double* EEp = op + (8 * hh + g) * S::LD2 + t;
    const double* EOp = EEp + S::OFF_EO;
    const double* OA = op + S::OFF_O + (8 * hh + g) * S::LD + t;
    const double* OB = op + S::OFF_O + (S::H - 1 - 8 * hh - g) * S::LD + t;
    const double* Fr0 = F + (rb * 16 + g) * LF;
    const double* Fr1 = Fr0 + 8 * LF;
    double pe[2][2] = {}, po[2][2] = {}, rA[2][2] = {}, rB[2][2] = {};
#pragma unroll
    for (int k0 = 0; k0 < S::H2; k0 += 4) {
        const int j = k0 + t;
        const double s0 = Fr0[j] + Fr0[C - 1 - j], d0 = Fr0[S::H - 1 - j] + Fr0[S::H + j];
        const double s1 = Fr1[j] + Fr1[C - 1 - j], d1 = Fr1[S::H - 1 - j] + Fr1[S::H + j];
        const double bE = EEp[k0], bO = EOp[k0];
        dmma884(pe[0], s0 + d0, bE);
        dmma884(pe[1], s1 + d1, bE);
        dmma884(po[0], s0 - d0, bO);
        dmma884(po[1], s1 - d1, bO);
    }
#pragma unroll
    for (int k0 = 0; k0 < S::H; k0 += 4) {
        const int j = k0 + t;
        const double v0 = Fr0[j] - Fr0[C - 1 - j], v1 = Fr1[j] - Fr1[C - 1 - j];
        const double bA = OA[k0], bB = OB[k0];
        dmma884(rA[0], v0, bA);
        dmma884(rA[1], v1, bA);
        dmma884(rB[0], v0, bB);
        dmma884(rB[1], v1, bB);
    }
    const int ip = 8 * hh + 2 * t;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        double* Gr = G + (rb * 16 + a * 8 + g) * LF;
        const double p10 = pe[a][0] + po[a][0], p11 = pe[a][1] + po[a][1];
        const double p20 = pe[a][0] - po[a][0], p21 = pe[a][1] - po[a][1];
        *reinterpret_cast<double2*>(Gr + ip) = make_double2(p10 + rA[a][0], p11 + rA[a][1]);
        *reinterpret_cast<double2*>(Gr + C - 2 - ip) = make_double2(p11 - rA[a][1], p10 - rA[a][0]);
        *reinterpret_cast<double2*>(Gr + S::H - 2 - ip) = make_double2(p21 + rB[a][1], p20 + rB[a][0]);
        *reinterpret_cast<double2*>(Gr + S::H + ip) = make_double2(p20 - rB[a][0], p21 - rB[a][1]);
    }
}

// G[i][c] = sum_j A[i][j] F[j][c] on an R x C slab (two even/odd levels); EPI as col_op_ct;
// warp = (16-column block, group of 8 pair indices), (C / 16) x (R / 32) warps
template <int R, int C, int LF, int EPI>
__device__ __forceinline__ void col_op_eo2(const double* __restrict__ F, const ColOut& out,
                                           const double* __restrict__ op) {
    using S = AxisShapeEO2<R>;
    static_assert((C / 16) * S::GROUPS == kContourThreads / 32 && C % 16 == 0 && S::H2 % 8 == 0,
                  "one warp per 16 columns x 8 pair indices");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int cb = warp / S::GROUPS, hh = warp % S::GROUPS;
    const double* EEp = op + (8 * hh + g) * S::LD2 + t;
    const double* EOp = EEp + S::OFF_EO;
    const double* OA = op + S::OFF_O + (8 * hh + g) * S::LD + t;
    const double* OB = op + S::OFF_O + (S::H - 1 - 8 * hh - g) * S::LD + t;
    const double* Fc = F + cb * 16 + g;  // column c = cb*16 + b*8 + g
    double pe[2][2] = {}, po[2][2] = {}, rA[2][2] = {}, rB[2][2] = {};
#pragma unroll
    for (int k0 = 0; k0 < S::H2; k0 += 4) {
        const int j = k0 + t;
        const double aE = EEp[k0], aO = EOp[k0];
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double* f = Fc + b * 8;
            const double s = f[j * LF] + f[(R - 1 - j) * LF], d = f[(S::H - 1 - j) * LF] + f[(S::H + j) * LF];
            dmma884(pe[b], aE, s + d);
            dmma884(po[b], aO, s - d);
        }
    }
#pragma unroll
    for (int k0 = 0; k0 < S::H; k0 += 4) {
        const int j = k0 + t;
        const double aA = OA[k0], aB = OB[k0];
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double* f = Fc + b * 8;
            const double v = f[j * LF] - f[(R - 1 - j) * LF];
            dmma884(rA[b], aA, v);
            dmma884(rB[b], aB, v);
        }
    }
    const int ip = 8 * hh + g;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        const int c = cb * 16 + b * 8 + 2 * t;
        const double p10 = pe[b][0] + po[b][0], p11 = pe[b][1] + po[b][1];
        const double p20 = pe[b][0] - po[b][0], p21 = pe[b][1] - po[b][1];
        col_store<LF, EPI, R>(out, ip, c, p10 + rA[b][0], p11 + rA[b][1]);
        col_store<LF, EPI, R>(out, R - 1 - ip, c, p10 - rA[b][0], p11 - rA[b][1]);
        col_store<LF, EPI, R>(out, S::H - 1 - ip, c, p20 + rB[b][0], p21 + rB[b][1]);
        col_store<LF, EPI, R>(out, S::H + ip, c, p20 - rB[b][0], p21 - rB[b][1]);
    }
}

// R x C slab between global (row stride gs) and shared memory (row stride LF), optional factor w
template <bool TO_SMEM, int R, int C, int LF>
__device__ __forceinline__ void move_slab_ct(double* sm, double* gm, long long gs, const double* w) {
    constexpr int PER_ROW = C / 2;
    constexpr int TOTAL = R * PER_ROW;
    constexpr int U = (TOTAL + kContourThreads - 1) / kContourThreads;
    double2 v[U], f[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
        const int e = k * kContourThreads + threadIdx.x;
        if (TOTAL % kContourThreads == 0 || e < TOTAL) {
            const int r = e / PER_ROW, c = (e % PER_ROW) * 2;
            if (TO_SMEM) v[k] = *reinterpret_cast<const double2*>(gm + r * gs + c);
            else v[k] = *reinterpret_cast<const double2*>(sm + r * LF + c);
            if (w) f[k] = __ldg(reinterpret_cast<const double2*>(w + r * gs + c));
        }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
        const int e = k * kContourThreads + threadIdx.x;
        if (TOTAL % kContourThreads == 0 || e < TOTAL) {
            const int r = e / PER_ROW, c = (e % PER_ROW) * 2;
            double2 x = v[k];
            if (w) {
                x.x = x.x * f[k].x;
                x.y = x.y * f[k].y;
            }
            if (TO_SMEM) *reinterpret_cast<double2*>(sm + r * LF + c) = x;
            else *reinterpret_cast<double2*>(gm + r * gs + c) = x;
        }
    }
}

template <int NX, int NY, int NZ, bool EX, bool EY, bool EZ>
__global__ void __launch_bounds__(kContourThreads, 1) contour_kernel_ct(const ContourArgs a) {
    extern __shared__ __align__(16) double smem[];
    constexpr int LF = NZ + 4;
    constexpr int ROWS = NX > NY ? NX : NY;
    constexpr int OFFX = 0;
    constexpr int OFFY = AxisShape<NX, EX>::SIZE;
    constexpr int OFFZ = OFFY + AxisShape<NY, EY>::SIZE;
    constexpr int OPS = OFFZ + AxisShape<NZ, EZ>::SIZE;
    constexpr int OPS_PAD = (OPS + 1) & ~1;
    double* sops = smem;
    double* F = smem + OPS_PAD;
    double* G = F + ROWS * LF;
    op_copy_async(sops, a.ops, OPS);
    cp_async_wait_all();
    __syncthreads();

    constexpr long long M = (long long)NX * NY * NZ;
    constexpr long long PLANE = (long long)NY * NZ;
    const int unitsP = a.nchain * NX, unitsQ = a.nchain * NY;
    unsigned target = 0;
    for (int t = a.t_begin; t < a.t_end; ++t) {
        for (int u = blockIdx.x; u < unitsP; u += gridDim.x) {
            const int c = u >= NX ? 1 : 0, x = u - c * NX;
            const int dir = c ? a.dir[1] : a.dir[0];
            const long long in_slot = (c ? a.slot0[1] : a.slot0[0]) + (long long)dir * t;
            const long long seg = dir > 0 ? in_slot : in_slot - 1;
            const double* w = seg < a.NsA ? a.wds[0] : a.wds[1];
            double* q = c ? a.q[1] : a.q[0];
            double* xb = c ? a.xbuf[1] : a.xbuf[0];
            move_slab_ct<true, NY, NZ, LF>(F, q + in_slot * M + x * PLANE, NZ, w ? w + x * PLANE : nullptr);
            __syncthreads();
            row_op_ct<NY, NZ, LF, EZ>(F, G, sops + OFFZ);
            __syncthreads();
            col_op_ct<NY, NZ, LF, EY>(G, F, sops + OFFY);
            __syncthreads();
            move_slab_ct<false, NY, NZ, LF>(F, xb + x * PLANE, NZ, nullptr);
            __syncthreads();
        }
        target += gridDim.x;
        if (!grid_barrier(a.bar_count, a.error, target, a.spin_limit)) return;
        for (int u = blockIdx.x; u < unitsQ; u += gridDim.x) {
            const int c = u >= NY ? 1 : 0, y = u - c * NY;
            const int dir = c ? a.dir[1] : a.dir[0];
            const long long in_slot = (c ? a.slot0[1] : a.slot0[0]) + (long long)dir * t;
            const long long out_slot = in_slot + dir;
            const long long seg = dir > 0 ? in_slot : in_slot - 1;
            const double* w = seg < a.NsA ? a.wds[0] : a.wds[1];
            double* q = c ? a.q[1] : a.q[0];
            double* xb = c ? a.xbuf[1] : a.xbuf[0];
            move_slab_ct<true, NX, NZ, LF>(F, xb + (long long)y * NZ, PLANE, nullptr);
            __syncthreads();
            col_op_ct<NX, NZ, LF, EX>(F, G, sops + OFFX);
            __syncthreads();
            move_slab_ct<false, NX, NZ, LF>(G, q + out_slot * M + (long long)y * NZ, PLANE,
                                            w ? w + (long long)y * NZ : nullptr);
            __syncthreads();
        }
        if (t + 1 < a.t_end) {
            target += gridDim.x;
            if (!grid_barrier(a.bar_count, a.error, target, a.spin_limit)) return;
        }
    }
}

}  // namespace crysscft

// ---------------------------------------------------------------------------
// Alternating-layout schedule (cubic grids): the three axis operators commute, so
// the phase that finishes step k can also start step k+1 on the same data layout.
//   plane phase (units (chain, x)):  [z y]  D  store q  D  [y]  -> exchange buffer XP
//   slab phase  (units (chain, y)):  [z x]  D  store q  D  [x]  -> exchange buffer XS
// (step k is started with y on planes and finished with z and x on slabs, or started with
// x on slabs and finished with z and y on planes: three operations per phase, and both
// phases begin with the row operation A_z)
// Phase k (k = 0..U) finishes step k-1 (k >= 1) and starts step k (k < U); plane
// phases have even k.  One exchange per step and no grid barrier: a unit waits only for
// the release flags of the units whose rows it reads.  The Boltzmann-factor tiles of the
// next phase are loaded by TMA as soon as the current ones are consumed; the last axis
// operation of a phase applies D in its epilogue and finished q(s) tiles leave by TMA
// stores, so neither sits on the critical path.
// ---------------------------------------------------------------------------
namespace crysscft {

// ---- TMA (cp.async.bulk.tensor) and mbarriers ---------------------------------------
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of `bar` with the given parity to complete; false after `limit` polls.
// Polls allowed for draining this block's own bulk copies on an error exit, independent
// of the caller's wait limit (a copy from valid memory completes in microseconds).
constexpr long long kDrainSpins = 1LL << 24;

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
    long long spins = 0;
    while (!mbar_test(bar, parity)) {
        if (++spins > limit) return false;
    }
    return true;
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the source shared memory of this thread's bulk stores may be overwritten after this
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the bulk-copy engine
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// tiled TMA: the 4-D box at (c0, c1, c2, c3) into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
// tiled TMA: shared memory to the 5-D box at (c0, .., c4), tracked by bulk groups
__device__ __forceinline__ void tma_store_5d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3,
                                             int c4) {
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5, %6}], [%1];"
                 ::"l"(map), "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
                 : "memory");
}
// tiled TMA: the 5-D box at (c0, .., c4) into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}
// the 5-D box at (c0, .., c4) of a tensor map into L2 (no shared memory, no completion)
__device__ __forceinline__ void tma_prefetch_l2_5d(const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4) {
    asm volatile("cp.async.bulk.prefetch.tensor.5d.L2.global.tile [%0, {%1, %2, %3, %4, %5}];"
                 ::"l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
                 : "memory");
}
// every bulk group of this thread but the newest one (three) has completed (writes performed)
__device__ __forceinline__ void bulk_wait_but_newest() { asm volatile("cp.async.bulk.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_newest3() { asm volatile("cp.async.bulk.wait_group 3;" ::: "memory"); }
// orders this thread's generic-proxy accesses of global memory with its bulk copies
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
// bulk reduction: dst[i] += src[i] for `bytes` / 8 doubles, shared to global, tracked by bulk groups
__device__ __forceinline__ void bulk_reduce_add_f64(double* dst, const void* src, unsigned bytes) {
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;"
                 ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
// N x N tile from global (row stride gs) into shared memory (row stride LF) with cp.async
template <int N, int LF>
__device__ __forceinline__ void tile_fetch(double* sm, const double* gm, long long gs) {
    constexpr int PER_ROW = N / 2;
    constexpr int TOTAL = N * PER_ROW;
#pragma unroll 4
    for (int e = threadIdx.x; e < TOTAL; e += kContourThreads) {
        const int r = e / PER_ROW, c = (e - r * PER_ROW) * 2;
        cp_async16(sm + r * LF + c, gm + r * gs + c);
    }
}

// T <- T * W (T row stride LF, W in 8-column panels)
template <int N, int LF>
__device__ __forceinline__ void tile_scale_panel(double* T, const double* W) {
    constexpr int PER_ROW = N / 2;
    constexpr int TOTAL = N * PER_ROW;
#pragma unroll 4
    for (int e = threadIdx.x; e < TOTAL; e += kContourThreads) {
        const int r = e / PER_ROW, c = (e - r * PER_ROW) * 2;
        double2 v = *reinterpret_cast<double2*>(T + r * LF + c);
        const double2 w = *reinterpret_cast<const double2*>(W + panel_index<N>(r, c));
        v.x = v.x * w.x;
        v.y = v.y * w.y;
        *reinterpret_cast<double2*>(T + r * LF + c) = v;
    }
}

// Shared-memory carve-up of the alternating kernel: operators, two padded work tiles
// (row stride LF, conflict-free MMA fragments), and three N x N tiles in 8-column panels
// filled and drained by TMA (Boltzmann factors W0/W1, q staging tile QS); the last axis
// operation of a phase reads and writes the panels from its MMA accumulators, where two
// rows x 8 columns per quarter-warp fall on distinct banks.
template <int N, bool EO, bool EO2 = false>
struct AltShape {
    static constexpr int LF = N + 4;
    static constexpr int AX = EO2 ? AxisShapeEO2<N>::SIZE : AxisShape<N, EO>::SIZE;  // per-axis operator block
    static constexpr int OPS = 3 * AX;
    static constexpr int OPS_PAD = (OPS + 15) & ~15;        // 128-byte aligned tiles after it
    static constexpr int TILE = (N * LF + 15) & ~15;
    static constexpr int WT = N * N;
    // + 128: the carve-up starts at the first 128-byte boundary of the dynamic window
    static constexpr size_t SMEM = (size_t)(OPS_PAD + 2 * TILE + 3 * WT) * sizeof(double) + 128;
};

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Preconditions of the bulk/TMA copies, checked once per launch before any is issued:
// bit 3 of the returned word: a shared-memory tile not 128-byte aligned; bit 4: a TMA
// descriptor not 64-byte aligned.  0 when every copy may be issued.
__device__ __forceinline__ int tma_alignment_error(const void* const* tiles, int ntiles, const CUtensorMap* maps,
                                                   int nmaps) {
    int e = 0;
    for (int i = 0; i < ntiles; ++i)
        if (smem_u32(tiles[i]) & 127u) e |= 8;
    for (int i = 0; i < nmaps; ++i)
        if (reinterpret_cast<uintptr_t>(&maps[i]) & 63u) e |= 16;
    return e;
}

template <int N, bool EO, bool EO2 = false>
__global__ void __launch_bounds__(kContourThreads, 1) contour_alt_kernel(const __grid_constant__ ContourArgs a) {
    static_assert(!EO2 || (EO && N == 64), "two even/odd levels: n = 64");
    using S = AltShape<N, EO, EO2>;
    constexpr int LF = S::LF;
    constexpr int OFFY = S::AX;
    constexpr int OFFZ = 2 * S::AX;
    constexpr int TPR = kContourThreads / N;         // threads per tile row (rows * TPR <= block)
    constexpr int CPT = (N / 2 + TPR - 1) / TPR;     // 16-byte chunks per thread and row
    constexpr unsigned TILE_BYTES = N * N * sizeof(double);
    static_assert(TPR >= 1, "tile rows must not exceed the block");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // the dynamic window is only guaranteed 16-byte alignment; TMA tiles need 128
    double* smem = reinterpret_cast<double*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
    double* sops = smem;
    double* T0 = smem + S::OPS_PAD;
    double* T1 = T0 + S::TILE;
    double* W0 = T1 + S::TILE;  // D of the step being finished
    double* W1 = W0 + S::WT;    // D of the step being started
    double* QS = W1 + S::WT;    // finished q(s+1), drained by bulk stores
    __shared__ __align__(8) unsigned long long s_bar;  // completion of the W0/W1 bulk loads
    __shared__ __align__(8) unsigned long long s_xbar; // fused phi: the other chain's slot tile
    __shared__ int s_fail;

    constexpr long long M = (long long)N * N * N;
    constexpr long long PLANE = (long long)N * N;
    const int units = a.nchain * N;
    const int u = blockIdx.x;  // one unit per block: the host launches units <= SMs blocks
    if (units > (int)gridDim.x) {
        if (threadIdx.x == 0) atomicOr(a.error, 4);
        return;
    }
    if (u >= units) return;
    const int warp = threadIdx.x >> 5;
    const bool fphi = a.phi_acc != nullptr;  // the host sets it only for two chains
    {
        const void* tiles[4] = {W0, W1, QS, T1};
        const int e = tma_alignment_error(tiles, fphi ? 4 : 3, &a.tm_pq[0][0], 4) |
                      tma_alignment_error(tiles, 0, &a.tm_pw[0][0], 4);
        if (e) {
            if (threadIdx.x == 0) atomicOr(a.error, e);
            return;
        }
    }
    op_copy_async(sops, a.ops, S::OPS);
    cp_async_wait_all();
    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(&s_bar, 1);
        mbar_init(&s_xbar, 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int U = a.t_end;  // steps 0..U-1 of both chains (t_begin is 0)
    const int c = u >= N ? 1 : 0, p = u - c * N;
    const int dir = c ? a.dir[1] : a.dir[0];
    const long long slot0 = c ? a.slot0[1] : a.slot0[0];
    // Fused phi.  The phase that finishes slot s of this chain sums q(s) q+(s) over the
    // unit's tile when the other chain finished slot s at least two phases earlier (the
    // second half of the contour: chain 0 the slots above U/2, chain 1 those below).  The
    // other chain's tile of slot s is bulk-loaded into T1 (free between the finishing
    // operation and the next phase's A_z); after this phase's release the products replace
    // q(s) in QS (its store has read it) and one bulk add (cp.reduce.async.bulk) puts them
    // into the unit's accumulator tile of the slot's block and the layout.  Per-element
    // atomics were measured slower: 4096 FP64 L2 atomics per unit and phase slowed the
    // exchange more than the separate phi pass costs.  A tile's bulk adds are issued only
    // after the previous one has completed, so the sums run in phase order (deterministic).
    // The host enables this only for chain 0 forward from slot 0 and chain 1 backward from
    // slot U, U even: then kp = U - k, and the slots read are those stored before U/2.
    // Slots 0, NsA (trapezoid weights), U/2 (both chains finish it in the same phase) and
    // U are left to the finishing kernel.
    const int co = 1 - c;
    double* acc_unit = fphi ? a.phi_acc + (size_t)c * 4 * M + (size_t)p * PLANE : nullptr;
    auto x_active = [&](int k) -> bool {
        const long long s = slot0 + (long long)dir * k, kq = (s - a.slot0[co]) * a.dir[co];
        return fphi && k >= 1 && k <= U && kq >= 1 && kq <= k - 2 && ((k - kq) & 1) == 0 && s != a.NsA;
    };
    unsigned xpar = 0;   // parity of the pending phase of s_xbar
    unsigned x_seen = 0; // thread 0: the other unit's landed-store count last acquired
    bool x_pend = false; // this thread gave up waiting for an issued slot-tile load
    double* q = c ? a.q[1] : a.q[0];
    double* XP = c ? a.xbuf[1] : a.xbuf[0];  // written by plane phases
    double* XS = XP + M;                     // written by slab phases
    // flags[chain][producing layout][consumer][producer]: every consumer polls its own
    // N flags (one cache line per 32), written by the producers (push), so the waits of
    // different blocks never share a line
    unsigned* fl_plane = a.flags + (size_t)c * 2 * N * N;  // written by plane units
    unsigned* fl_slab = fl_plane + (size_t)N * N;           // written by slab units

    // block of the Boltzmann factor exp(-w ds/2) of step s: A (0) for segments < NsA, else B (1)
    auto blk_of = [&](int s) -> int {
        const long long in_slot = slot0 + (long long)dir * s;
        const long long seg = dir > 0 ? in_slot : in_slot - 1;
        return seg < a.NsA ? 0 : 1;
    };
    // warp 0: bulk-load the Boltzmann tiles of phase k (W0 = D of step k-1, W1 = D of step k)
    auto issue_w = [&](int k) {
        const bool plane = (k & 1) == 0;
        const unsigned bytes = ((k >= 1) + (k < U)) * TILE_BYTES;
        if ((threadIdx.x & 31) == 0) mbar_expect_tx(&s_bar, bytes);
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {  // 8-column panels, the layout the finishing epilogue reads
            if (k >= 1) tma_load_4d(W0, &a.tm_pw[blk_of(k - 1)][plane ? 0 : 1], 0, 0, 0, p, &s_bar);
            if (k < U) tma_load_4d(W1, &a.tm_pw[blk_of(k)][plane ? 0 : 1], 0, 0, 0, p, &s_bar);
        }
    };
    unsigned wpar = 0;  // parity of the pending W phase of s_bar
    // error exit: let this block's bulk copies finish (bounded), then return
    auto drain = [&](bool w_pending) {
        if (w_pending) mbar_wait(&s_bar, wpar, kDrainSpins);
        if (x_pend) mbar_wait(&s_xbar, xpar, kDrainSpins);
        if (warp == 0) bulk_wait_all();
    };

    // axis operations on shared-memory tiles (two even/odd levels when EO2)
    auto row_z = [&](const double* F, double* G) {
        if constexpr (EO2) row_op_eo2<N, N, LF>(F, G, sops + OFFZ);
        else row_op_ct<N, N, LF, EO>(F, G, sops + OFFZ);
    };
    auto col_smem = [&](const double* F, double* G, int off) {
        if constexpr (EO2) col_op_eo2<N, N, LF, kToSmem>(F, ColOut{G, 0}, sops + off);
        else col_op_ct<N, N, LF, EO>(F, G, sops + off);
    };
    auto col_global = [&](const double* F, const ColOut& o, int off) {
        if constexpr (EO2) col_op_eo2<N, N, LF, kToGlobal>(F, o, sops + off);
        else col_op_ct<N, N, LF, EO, kToGlobal>(F, o, sops + off);
    };

    if (warp == 0) issue_w(0);
    for (int k = 0; k <= U; ++k) {
        const bool plane = (k & 1) == 0;
        const long long off = plane ? (long long)p * PLANE : (long long)p * N;
        const long long gs = plane ? N : PLANE;
        // fused phi: slot finished in this phase, and the phase kp in which the other chain
        // finished (stored) the same slot on the same layout and tile
        const long long s_fin = slot0 + (long long)dir * k;
        const long long kp = (s_fin - a.slot0[co]) * a.dir[co];
        const bool xact = x_active(k);
        if (k == 0) {
            tile_fetch<N, LF>(T0, q + slot0 * M + off, gs);
        } else {
            // row r of this tile was produced by unit r of the other layout in phase k-1:
            // wait for its flag, then fetch the row (waits and copies overlap)
            const int r = threadIdx.x / TPR, sub = threadIdx.x - r * TPR;
            if (r < N) {
                const unsigned* f = (plane ? fl_slab : fl_plane) + (size_t)p * N + r;
                long long spins = 0;
                while (ld_acquire_u32(f) < (unsigned)k) {
                    if (++spins > a.spin_limit) {
                        atomicOr(a.error, 1);
                        s_fail = 1;
                        break;
                    }
                    if (spins > 64) __nanosleep(20);
                }
                const double* src = (plane ? XS : XP) + off + r * gs;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int ch = sub + j * TPR;
                    if (ch < N / 2) cp_async16(T0 + r * LF + 2 * ch, src + 2 * ch);
                }
            }
        }
        cp_async_commit();
        cp_async_wait_all();
        if (EO2 && k >= 1) {
            static_assert(!EO2 || (TPR == 4 && AxisShapeEO2<N>::GROUPS == 2),
                          "warp w fetches rows 8w..8w+7; row_op_eo2 gives warps 2b, 2b+1 rows 16b..16b+15");
            // the first operation of both layouts (A_z along rows) of warps 2b, 2b+1 reads
            // only rows 16b..16b+15, which these two warps fetched: they start as soon as
            // their own producers' rows are in, while other rows are still arriving.  A wait
            // that ran out is caught at the block barrier after the operation.
            asm volatile("bar.sync %0, 64;" ::"r"(1 + (warp >> 1)) : "memory");
        } else {
            __syncthreads();
            if (s_fail) {
                drain(true);
                return;
            }
        }
        double* cur = T0;
        double* oth = T1;
        if (k >= 1) {
            // finish step k-1: A_z, then the layout's column axis (A_y on planes, A_x on
            // slabs), whose epilogue applies D, writes q(s+1) to the panel staging tile and
            // D q(s+1) to the work tile
            row_z(cur, oth);
            if (warp == 0) bulk_wait_read();  // the previous q store has left QS
            if (!mbar_wait(&s_bar, wpar, a.spin_limit)) s_fail = 1;
            __syncthreads();
            if (s_fail) {
                if (threadIdx.x == 0) atomicOr(a.error, 2);
                drain(true);
                return;
            }
            wpar ^= 1u;
            ColOut fo{cur, 0};
            fo.w0 = W0;
            fo.w1 = W1;
            fo.qs = QS;
            fo.start = k < U;
            if constexpr (EO2) col_op_eo2<N, N, LF, kFinish>(oth, fo, sops + (plane ? OFFY : 0));
            else col_op_ct<N, N, LF, EO, kFinish>(oth, fo, sops + (plane ? OFFY : 0));
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {  // the thread that commits and waits on bulk groups
                tma_store_5d(&a.tm_pq[c][plane ? 0 : 1], QS, 0, 0, 0, p, (int)(slot0 + (long long)dir * k));
                bulk_commit();
                if (fphi) {
                    if (xact) {  // T1 was last read by the finishing operation (fenced above)
                        // the other unit releases once; after the first acquire that saw it, no
                        // further round trip to L2 on warp 0's way to the phase's last operation
                        const unsigned* df = a.done + (size_t)co * N + p;
                        long long spins = 0;
                        while (x_seen < (unsigned)(kp + 1)) {
                            x_seen = ld_acquire_u32(df);
                            if (x_seen >= (unsigned)(kp + 1)) break;
                            if (++spins > a.spin_limit) break;
                            if (spins > 64) __nanosleep(32);
                        }
                        if (spins > a.spin_limit) {
                            atomicOr(a.error, 32);
                            s_fail = 1;  // no load issued; the block leaves after the next barrier
                        } else {
                            fence_async_global();
                            mbar_expect_tx(&s_xbar, TILE_BYTES);
                            tma_load_5d(T1, &a.tm_pq[co][plane ? 0 : 1], 0, 0, 0, p, (int)s_fin, &s_xbar);
                        }
                    }
                    // the next phase's tile into L2 now (the old slots are in HBM); it was
                    // stored at least three phases ago, and L2 is coherent with that store
                    if (x_active(k + 1))
                        tma_prefetch_l2_5d(&a.tm_pq[co][plane ? 1 : 0], 0, 0, 0, p, (int)(s_fin + dir));

                }
            }
        }
        if (k == 0) {
            if (!mbar_wait(&s_bar, wpar, a.spin_limit)) s_fail = 1;
            __syncthreads();
            if (s_fail) {  // every thread leaves here: the W load still lands in this block's memory first
                if (threadIdx.x == 0) atomicOr(a.error, 2);
                drain(true);
                return;
            }
            wpar ^= 1u;
            tile_scale_panel<N, LF>(cur, W1);
            __syncthreads();
        }
        if (k < U) {
            // W0/W1 are free: prefetch the next phase's factors (in a phase with the fused phi
            // sums after them, so the bulk copies the sums wait for go first)
            if (warp == 0 && !xact) issue_w(k + 1);
            // start step k on this layout with its column axis; the epilogue writes the
            // exchange buffer, which the other layout finishes (A_z, then its own axis) next phase
            const ColOut xo{(plane ? XP : XS) + off, gs};
            col_global(cur, xo, plane ? OFFY : 0);
            __syncthreads();
            if (xact && s_fail) {  // thread 0 gave up on the other chain's store: no load in flight
                drain(false);
                return;
            }
            if (threadIdx.x < N) {  // tell consumer threadIdx.x that tile p of phase k is out
                __threadfence();
                st_release_u32((plane ? fl_plane : fl_slab) + (size_t)threadIdx.x * N + p, (unsigned)(k + 1));
            }
            if (fphi && threadIdx.x == 0 && 2 * k == U) {
                // the other chain reads only slots this chain stored before the midpoint
                // phase (kp <= U/2 - 1 above): one release, once those stores have landed
                // (every bulk group but this phase's q store has completed).  A release in
                // every phase, right after the q store was issued, cost 0.15 ms per iteration.
                bulk_wait_but_newest();
                fence_async_global();
                st_release_u32(a.done + (size_t)c * N + p, (unsigned)k);
            }
        }
        if (fphi && k == 0) {  // zero the accumulator tiles, long before the first bulk add
            for (int t4 = 0; t4 < 4; ++t4)
                for (int i = threadIdx.x; i < N * N; i += kContourThreads) acc_unit[(size_t)t4 * M + i] = 0.0;
            fence_async_global();
        }
        if (xact) {  // fused phi: QS holds q(s) of this chain, T1 the other chain's, same panels
            if (threadIdx.x == 0) bulk_wait_read();  // the q(s) store has read QS
            if (mbar_wait(&s_xbar, xpar, a.spin_limit)) {
                xpar ^= 1u;
            } else {
                x_pend = true;
                s_fail = 1;
                atomicOr(a.error, 2);
            }
            __syncthreads();
            if (s_fail) {  // the next phase's factors are not requested yet
                drain(false);
                return;
            }
            // QS <- q(s) q+(s), then one bulk add into the accumulator tile; the next phase's
            // wait for QS to be read (before its finishing operation) covers it.  The barrier
            // after the products also ends the phase.
            for (int i = 2 * threadIdx.x; i < N * N; i += 2 * kContourThreads) {
                double2 v = *reinterpret_cast<double2*>(QS + i);
                const double2 w = *reinterpret_cast<const double2*>(T1 + i);
                v.x *= w.x;
                v.y *= w.y;
                *reinterpret_cast<double2*>(QS + i) = v;
            }
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                // the add of two phases back (same layout, possibly the same tile) has
                // completed: at most this phase's store and the last phase's store and add
                // are pending, so the adds into one tile apply in phase order
                bulk_wait_newest3();
                bulk_reduce_add_f64(acc_unit + (size_t)((s_fin < a.NsA ? 0 : 2) + (plane ? 0 : 1)) * M, QS,
                                    TILE_BYTES);
                bulk_commit();
            }
            if (warp == 0) issue_w(k + 1);  // an active phase is never the last (kp >= 1)
        } else {
            __syncthreads();
            if (fphi && s_fail) {
                drain(k < U);
                return;
            }
        }
    }
    if (warp == 0) bulk_wait_all();
}

}  // namespace crysscft
