// Axis passes on the tensor cores for large cubic grids (n = 96, 128), where the
// whole-contour kernels do not fit in shared memory: one persistent launch per pass
// (z, y or x) over both contour chains, the axis operator resident in shared memory
// (even/odd form when centrosymmetric), DMMA tiles from the contour kernel
// (row_op_ct / col_op_ct; two even/odd levels, row_op_eo2 / col_op_eo2, for 128-point
// PMMM axes), and the next tile prefetched into registers while the current one is on
// the tensor cores.  The Boltzmann factor exp(-w ds/2) of the
// contour step is applied on the z-pass input (pre) and the x-pass output (post),
// as in the per-axis SIMT kernels (axis_kernels.cuh) these replace for such grids.
//
//   z pass: rows of n contiguous values, tile = kRowsZ rows x n      (row_op_ct)
//   y pass: for one x, tile = n (y) x kColsYX (z) with row stride n   (col_op_ct)
//   x pass: for one y, tile = n (x) x kColsYX (z) with row stride n^2 (col_op_ct)
// FP64 runs on DMMA (axis_dmma_kernel); the FP32 precision form on 3xTF32 split products
// (axis_tf32_kernel, row_op_f32 / col_op_f32).
#pragma once
#include <cuda_runtime.h>

#include "contour_kernel.cuh"
#include "contour_kernel_f32.cuh"

namespace crysscft {

constexpr int kRowsZ = 32;
constexpr int kColsYX = 32;

// L2 eviction priorities of the pass traffic.  At 256^3 the two chains' working set (the
// Boltzmann factors, the field a pass reads and the one it writes) is close to the L2
// size, and the contour slices written every step stream through it.  A pass's output
// is read by the next pass (evict_last); its input is dead once read (evict_first, which
// also demotes the line the previous pass kept); the Boltzmann factors are reused every
// step (evict_last).  hints == 0 issues the plain cache-global forms.
// Drop the 128-byte L2 line at a (128-byte aligned) without writing it back: for a pass
// input that no one reads again (the triplet's intermediate fields), so that evicting
// it costs no DRAM write.
__device__ __forceinline__ void l2_discard_line(const void* a) {
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(a) : "memory");
}

__device__ __forceinline__ unsigned long long l2_policy(bool last) {
    unsigned long long p;
    if (last) asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double2 ld_cg_policy(const double* a, unsigned long long pol) {
    double2 v;
    asm volatile("ld.global.cg.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ld_nc_policy(const double* a, unsigned long long pol) {
    double2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_cg_policy(double* a, double2 v, unsigned long long pol) {
    asm volatile("st.global.cg.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ float4 ld_cg_policy(const float* a, unsigned long long pol) {
    float4 v;
    asm volatile("ld.global.cg.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_nc_policy(const float* a, unsigned long long pol) {
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_cg_policy(float* a, float4 v, unsigned long long pol) {
    asm volatile("st.global.cg.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(a), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}

struct AxisPassD {
    const double* in[2];
    double* out[2];
    const double* pre[2];   // z pass: input *= pre (nullptr: none)
    const double* post[2];  // x pass: output *= post (nullptr: none)
    const double* op;       // this axis' packed operator (AxisShape<N, EO> or AxisShapeEO2<N> layout)
    int nchain;
    int hints;              // 1: L2 eviction priorities on the pass traffic (see l2_policy)
    int discard_in;         // 1: the input is dead once read (a triplet intermediate): drop its
                            // L2 lines after the tile is loaded (y and x passes)
};

template <int N, bool EO, bool EO2 = false>
struct AxisDmmaShape {
    static_assert(!EO2 || (EO && N == 128), "two even/odd levels: 128-point even/odd axes");
    static constexpr int OP_VALUES = EO2 ? AxisShapeEO2<N>::SIZE : AxisShape<N, EO>::SIZE;
    static constexpr int OPS = (OP_VALUES + 15) & ~15;
    static constexpr int LFZ = N + 4;       // z tile: kRowsZ x N
    static constexpr int LFC = kColsYX + 4;  // y/x tile: N x kColsYX
    static constexpr int TILE = (N * LFC > kRowsZ * LFZ ? N * LFC : kRowsZ * LFZ);
    static constexpr int TILE_PAD = (TILE + 15) & ~15;
    static constexpr size_t SMEM = (size_t)(OPS + 2 * TILE_PAD) * sizeof(double);
    static constexpr int PER_THREAD = N * kColsYX / 2 / kContourThreads;  // double2 per thread and tile
    static_assert(N * kColsYX == kRowsZ * N, "z and y/x tiles hold the same number of values");
    static_assert(PER_THREAD * 2 * kContourThreads == N * kColsYX, "tile not a multiple of the block");
};

// element (r, c) of tile `t` (double2 granularity: c even) and its global offset
template <int N, int AX>
struct AxisTiling {
    static constexpr long long M = (long long)N * N * N;
    static constexpr int TILES_PER_CHAIN = (AX == 2) ? (N * N / kRowsZ) : (N * (N / kColsYX));
    // global offset of the tile's origin within its chain and the row stride
    __device__ static long long origin(int t) {
        if (AX == 2) return (long long)t * kRowsZ * N;
        const int a = t / (N / kColsYX), zb = t - a * (N / kColsYX);
        return AX == 1 ? (long long)a * N * N + zb * kColsYX : (long long)a * N + zb * kColsYX;
    }
    static constexpr long long ROW_STRIDE = AX == 2 ? N : (AX == 1 ? N : (long long)N * N);
    static constexpr int ROW_LEN = AX == 2 ? N : kColsYX;  // values per tile row
};

template <int N, bool EO, int AX, bool EO2 = false>
__global__ void __launch_bounds__(kContourThreads, 1) axis_dmma_kernel(const AxisPassD p) {
    using S = AxisDmmaShape<N, EO, EO2>;
    using TL = AxisTiling<N, AX>;
    constexpr int LF = AX == 2 ? S::LFZ : S::LFC;
    constexpr int RL = TL::ROW_LEN;
    constexpr int PT = S::PER_THREAD;
    extern __shared__ __align__(16) double axs[];
    double* sop = axs;
    double* F = axs + S::OPS;
    double* G = F + S::TILE_PAD;
    op_copy_async(sop, p.op, S::OP_VALUES);

    const int tiles = p.nchain * TL::TILES_PER_CHAIN;
    const unsigned long long pol_first = l2_policy(false), pol_last = l2_policy(true);
    double2 v[PT], w[PT];
    // fetch tile t into registers (input x pre for the z pass; post for the x pass)
    auto fetch = [&](int t) {
        const int c = t / TL::TILES_PER_CHAIN;
        const long long o = TL::origin(t - c * TL::TILES_PER_CHAIN);
        const double* in = p.in[c] + o;
        const double* aux = AX == 2 ? p.pre[c] : (AX == 0 ? p.post[c] : nullptr);
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            const int e = (k * kContourThreads + threadIdx.x) * 2;
            const int r = e / RL, cc = e - r * RL;
            const long long g = r * TL::ROW_STRIDE + cc;
            if (p.hints) {
                v[k] = ld_cg_policy(in + g, pol_first);
                if (aux) w[k] = ld_nc_policy(aux + o + g, pol_last);
            } else {
                v[k] = __ldcg(reinterpret_cast<const double2*>(in + g));
                if (aux) w[k] = __ldg(reinterpret_cast<const double2*>(aux + o + g));
            }
        }
    };
    int t = blockIdx.x;
    if (t < tiles) fetch(t);  // in flight with the operator copies
    cp_async_wait_all();      // the operator; the loop's first barrier publishes it
    for (; t < tiles; t += gridDim.x) {
        const int c = t / TL::TILES_PER_CHAIN;
        const long long o = TL::origin(t - c * TL::TILES_PER_CHAIN);
        const bool pre = AX == 2 && p.pre[c] != nullptr;
        const bool post = AX == 0 && p.post[c] != nullptr;
        __syncthreads();  // the previous tile's G has been stored, F may be overwritten
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            const int e = (k * kContourThreads + threadIdx.x) * 2;
            const int r = e / RL, cc = e - r * RL;
            double2 x = v[k];
            if (pre) {
                x.x *= w[k].x;
                x.y *= w[k].y;
            }
            *reinterpret_cast<double2*>(F + r * LF + cc) = x;
        }
        double2 wpost[PT];
        if (post) {
#pragma unroll
            for (int k = 0; k < PT; ++k) wpost[k] = w[k];
        }
        __syncthreads();
        if (AX != 2 && p.discard_in) {
            // every load of this tile has returned (its values are in F): drop the input's
            // lines, two 128-byte lines per tile row of kColsYX doubles
            constexpr int LINES = N * (kColsYX * (int)sizeof(double) / 128);
            if (threadIdx.x < LINES) {
                const int r = threadIdx.x / (LINES / N), h = threadIdx.x - r * (LINES / N);
                l2_discard_line(p.in[c] + o + r * TL::ROW_STRIDE + h * (128 / (int)sizeof(double)));
            }
        }
        if (t + (int)gridDim.x < tiles) fetch(t + gridDim.x);  // in flight during the MMAs
        if constexpr (AX == 2) {
            if constexpr (EO2) row_op_eo2<kRowsZ, N, LF>(F, G, sop);
            else row_op_ct<kRowsZ, N, LF, EO>(F, G, sop);
        } else {
            if constexpr (EO2) col_op_eo2<N, kColsYX, LF, kToSmem>(F, ColOut{G, 0}, sop);
            else col_op_ct<N, kColsYX, LF, EO>(F, G, sop);
        }
        __syncthreads();
        double* out = p.out[c] + o;
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            const int e = (k * kContourThreads + threadIdx.x) * 2;
            const int r = e / RL, cc = e - r * RL;
            double2 y = *reinterpret_cast<const double2*>(G + r * LF + cc);
            if (post) {
                y.x *= wpost[k].x;
                y.y *= wpost[k].y;
            }
            if (p.hints) st_cg_policy(out + r * TL::ROW_STRIDE + cc, y, pol_last);
            else __stcg(reinterpret_cast<double2*>(out + r * TL::ROW_STRIDE + cc), y);
        }
    }
}

// ---- FP32 (3xTF32) form ---------------------------------------------------------
struct AxisPassF {
    const float* in[2];
    float* out[2];
    const float* pre[2];
    const float* post[2];
    const float* op;  // this axis' packed TF32 hi/lo operator (AxisShapeF<N, EO> layout)
    int nchain;
    int hints;        // as AxisPassD::hints
    int discard_in;   // as AxisPassD::discard_in
};

template <int N, bool EO>
struct AxisTf32Shape {
    static constexpr int OPS = (AxisShapeF<N, EO>::SIZE + 31) & ~31;
    static constexpr int LFZ = N + 4;
    static constexpr int LFC = kColsYX + 4;
    static constexpr int TILE = (N * LFC > kRowsZ * LFZ ? N * LFC : kRowsZ * LFZ);
    static constexpr int TILE_PAD = (TILE + 31) & ~31;
    static constexpr size_t SMEM = (size_t)(OPS + 2 * TILE_PAD) * sizeof(float);
    static constexpr int PER_THREAD = N * kColsYX / 4 / kContourThreads;  // float4 per thread and tile
    static_assert(PER_THREAD * 4 * kContourThreads == N * kColsYX, "tile not a multiple of the block");
};

template <int N, bool EO, int AX>
__global__ void __launch_bounds__(kContourThreads) axis_tf32_kernel(const AxisPassF p) {
    using S = AxisTf32Shape<N, EO>;
    using TL = AxisTiling<N, AX>;
    constexpr int LF = AX == 2 ? S::LFZ : S::LFC;
    constexpr int RL = TL::ROW_LEN;
    constexpr int PT = S::PER_THREAD;
    extern __shared__ __align__(16) float axf[];
    float* sop = axf;
    float* F = axf + S::OPS;
    float* G = F + S::TILE_PAD;
    op_copy_async(sop, p.op, AxisShapeF<N, EO>::SIZE);

    const int tiles = p.nchain * TL::TILES_PER_CHAIN;
    const unsigned long long pol_first = l2_policy(false), pol_last = l2_policy(true);
    float4 v[PT], w[PT];
    auto fetch = [&](int t) {
        const int c = t / TL::TILES_PER_CHAIN;
        const long long o = TL::origin(t - c * TL::TILES_PER_CHAIN);
        const float* in = p.in[c] + o;
        const float* aux = AX == 2 ? p.pre[c] : (AX == 0 ? p.post[c] : nullptr);
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            const int e = (k * kContourThreads + threadIdx.x) * 4;
            const int r = e / RL, cc = e - r * RL;
            const long long g = r * TL::ROW_STRIDE + cc;
            if (p.hints) {
                v[k] = ld_cg_policy(in + g, pol_first);
                if (aux) w[k] = ld_nc_policy(aux + o + g, pol_last);
            } else {
                v[k] = __ldcg(reinterpret_cast<const float4*>(in + g));
                if (aux) w[k] = __ldg(reinterpret_cast<const float4*>(aux + o + g));
            }
        }
    };
    int t = blockIdx.x;
    if (t < tiles) fetch(t);  // in flight with the operator copies
    cp_async_wait_all();      // the operator; the loop's first barrier publishes it
    for (; t < tiles; t += gridDim.x) {
        const int c = t / TL::TILES_PER_CHAIN;
        const long long o = TL::origin(t - c * TL::TILES_PER_CHAIN);
        const bool pre = AX == 2 && p.pre[c] != nullptr;
        const bool post = AX == 0 && p.post[c] != nullptr;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            const int e = (k * kContourThreads + threadIdx.x) * 4;
            const int r = e / RL, cc = e - r * RL;
            float4 x = v[k];
            if (pre) {
                x.x *= w[k].x;
                x.y *= w[k].y;
                x.z *= w[k].z;
                x.w *= w[k].w;
            }
            *reinterpret_cast<float4*>(F + r * LF + cc) = x;
        }
        float4 wpost[PT];
        if (post) {
#pragma unroll
            for (int k = 0; k < PT; ++k) wpost[k] = w[k];
        }
        __syncthreads();
        if (AX != 2 && p.discard_in) {  // as in axis_dmma_kernel: one 128-byte line per tile row
            static_assert(kColsYX * sizeof(float) == 128, "one line per FP32 tile row");
            if (threadIdx.x < N) l2_discard_line(p.in[c] + o + threadIdx.x * TL::ROW_STRIDE);
        }
        if (t + (int)gridDim.x < tiles) fetch(t + gridDim.x);
        if constexpr (AX == 2) row_op_f32<kRowsZ, N, LF, EO>(F, G, sop);
        else col_op_f32<N, kColsYX, LF, EO>(F, G, sop);
        __syncthreads();
        float* out = p.out[c] + o;
#pragma unroll
        for (int k = 0; k < PT; ++k) {
            const int e = (k * kContourThreads + threadIdx.x) * 4;
            const int r = e / RL, cc = e - r * RL;
            float4 y = *reinterpret_cast<const float4*>(G + r * LF + cc);
            if (post) {
                y.x *= wpost[k].x;
                y.y *= wpost[k].y;
                y.z *= wpost[k].z;
                y.w *= wpost[k].w;
            }
            if (p.hints) st_cg_policy(out + r * TL::ROW_STRIDE + cc, y, pol_last);
            else __stcg(reinterpret_cast<float4*>(out + r * TL::ROW_STRIDE + cc), y);
        }
    }
}

}  // namespace crysscft
