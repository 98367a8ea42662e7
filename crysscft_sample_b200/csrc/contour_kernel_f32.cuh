// FP32 form of the alternating-layout contour kernel (precision form of the triplets).
//
// Same schedule as contour_alt_kernel (plane phases [A_z A_y], slab phases [A_x],
// per-consumer release flags, TMA tiles), with FP32 contour slices and
// Boltzmann factors.  The axis products run on the tensor cores as 3xTF32 split
// products (mma.sync m16n8k8 .tf32, FP32 accumulate): every operand x is split
// into hi = tf32(x) and lo = tf32(x - hi) and a*b ~ a_lo b_hi + a_hi b_lo + a_hi b_hi,
// which keeps FP32-level accuracy (the dropped a_lo b_lo term is ~2^-22 relative).
// Operators are split on the host; field values are split on the fly.
#pragma once
#include <cuda_runtime.h>

#include "contour_kernel.cuh"

namespace crysscft {

__device__ __forceinline__ unsigned f32_to_tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
    hi = f32_to_tf32(x);
    lo = f32_to_tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// The tensor cores round the FP32 result of an MMA toward zero, so accumulating a whole
// contraction in the MMA accumulator biases every axis product low by a few units in
// the last place, and the bias compounds along the contour (measured: -6e-7 relative
// per contour step at n = 64).  Mode 0 accumulates on the tensor core; mode 1 gives
// every k-group of three MMAs a zero accumulator and adds the partials with
// round-to-nearest FP32 adds; mode 2 also adds back half a unit in the last place of
// each partial, the mean error of rounding toward zero; mode 3 adds back the mean of
// that half unit over log-uniform mantissas with one FMA.  Measured at 128^3 PMMM,
// Ns = 200 (contour slot 200 mean relative error; |dF/F| after 90 FP32 + 10 FP64
// iterations): mode 0 -1.5e-4, 1.0e-7; mode 1 -2.5e-5, 4.0e-9; mode 2 +2e-7, 2.9e-10;
// mode 3 -8.9e-6, 2.6e-8.  Mode 1 is the fastest one that meets |dF/F| <= 1e-8.
#ifndef CRYSSCFT_TF32_ACCUM
#define CRYSSCFT_TF32_ACCUM 1
#endif

// v + sign(v) * ulp(v) / 2 for normal v (zero and tiny values unchanged)
__device__ __forceinline__ float add_half_ulp(float v) {
    const unsigned e = __float_as_uint(v) & 0x7f800000u;
    if (e <= (24u << 23)) return v;
    return v + copysignf(__uint_as_float(e - (24u << 23)), v);
}

// d += (ahi + alo)(bhi + blo) without the lo*lo term, small terms first
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const unsigned (&ah)[4], const unsigned (&al)[4],
                                           const unsigned (&bh)[2], const unsigned (&bl)[2]) {
#if CRYSSCFT_TF32_ACCUM == 0
    mma_tf32(d, al[0], al[1], al[2], al[3], bh[0], bh[1]);
    mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bl[0], bl[1]);
    mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bh[0], bh[1]);
#else
    float t[4] = {0.f, 0.f, 0.f, 0.f};
    mma_tf32(t, al[0], al[1], al[2], al[3], bh[0], bh[1]);
    mma_tf32(t, ah[0], ah[1], ah[2], ah[3], bl[0], bl[1]);
    mma_tf32(t, ah[0], ah[1], ah[2], ah[3], bh[0], bh[1]);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
#if CRYSSCFT_TF32_ACCUM == 2
        t[e] = add_half_ulp(t[e]);
        d[e] += t[e];
#elif CRYSSCFT_TF32_ACCUM == 3
        // mean of ulp(v)/2 over a log-uniform mantissa is (1/(2 ln 2)) 2^-24 |v|
        d[e] = fmaf(t[e], 4.2995662e-08f, d[e] + t[e]);
#else
        d[e] += t[e];
#endif
    }
#endif
}

// Per-axis operator block in FP32: [hi part][lo part], each E then O (even/odd) or A (full).
template <int N, bool EO>
struct AxisShapeF {
    static constexpr int K = EO ? N / 2 : N;
    static constexpr int LD = K + 4;
    static constexpr int HALF = EO ? K * LD : 0;            // E -> O
    static constexpr int PART = EO ? 2 * K * LD : N * LD;   // hi -> lo
    static constexpr int SIZE = 2 * PART;
};

// G[r][i] = sum_j F[r][j] A[i][j] on an R x C slab: m16 tiles over r, n8 tiles over i
template <int R, int C, int LF, bool EO>
__device__ __forceinline__ void row_op_f32(const float* __restrict__ F, float* __restrict__ G,
                                           const float* __restrict__ op) {
    using S = AxisShapeF<C, EO>;
    constexpr int NI = S::K, K = S::K, LD = S::LD;
    constexpr int TM = R / 16, TN = NI / 8;
    constexpr int BN = (TN + 1) / 2;  // blocks of 1 x 2 tiles
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int blk = warp; blk < TM * BN; blk += kContourThreads / 32) {
        const int m0 = (blk / BN) * 16, nb = (blk % BN) * 2;
        const bool n1 = (TN % 2 == 0) || (nb + 1 < TN);
        float dP[2][4] = {}, dR[2][4] = {};
        const float* Fr0 = F + (m0 + g) * LF;
        const float* Fr1 = Fr0 + 8 * LF;
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 8) {
            unsigned uh[4], ul[4], vh[4], vl[4];
            {
                const int j0 = k0 + t, j1 = k0 + t + 4;
                const float x[4] = {Fr0[j0], Fr1[j0], Fr0[j1], Fr1[j1]};
                if (EO) {
                    const float y[4] = {Fr0[C - 1 - j0], Fr1[C - 1 - j0], Fr0[C - 1 - j1], Fr1[C - 1 - j1]};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        split_tf32(x[e] + y[e], uh[e], ul[e]);
                        split_tf32(x[e] - y[e], vh[e], vl[e]);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) split_tf32(x[e], uh[e], ul[e]);
                }
            }
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if (b == 1 && !n1) continue;
                const int i = (nb + b) * 8 + g;
                const float* Eh = op + i * LD + k0 + t;
                const float* El = Eh + S::PART;
                unsigned bh[2] = {__float_as_uint(Eh[0]), __float_as_uint(Eh[4])};
                unsigned bl[2] = {__float_as_uint(El[0]), __float_as_uint(El[4])};
                mma_3xtf32(dP[b], uh, ul, bh, bl);
                if (EO) {
                    const float* Oh = Eh + S::HALF;
                    const float* Ol = El + S::HALF;
                    unsigned ch[2] = {__float_as_uint(Oh[0]), __float_as_uint(Oh[4])};
                    unsigned cl[2] = {__float_as_uint(Ol[0]), __float_as_uint(Ol[4])};
                    mma_3xtf32(dR[b], vh, vl, ch, cl);
                }
            }
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            if (b == 1 && !n1) continue;
            const int i = (nb + b) * 8 + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = m0 + g + 8 * h;
                const float p0 = dP[b][2 * h], p1 = dP[b][2 * h + 1];
                if (EO) {
                    const float r0 = dR[b][2 * h], r1 = dR[b][2 * h + 1];
                    *reinterpret_cast<float2*>(G + r * LF + i) = make_float2(p0 + r0, p1 + r1);
                    *reinterpret_cast<float2*>(G + r * LF + (C - 2 - i)) = make_float2(p1 - r1, p0 - r0);
                } else {
                    *reinterpret_cast<float2*>(G + r * LF + i) = make_float2(p0, p1);
                }
            }
        }
    }
}

// Destination of col_op_f32 (ColEpilogue of the FP64 kernel): a shared slab or the global
// exchange buffer.
struct ColOutF {
    float* G;
    long long gs;
    const float* w0 = nullptr;  // kFinish: Boltzmann tiles of the finished / next step (panels)
    const float* w1 = nullptr;
    float* qs = nullptr;        // kFinish: staging tile of q (panels)
    int start = 0;              // kFinish: a next step follows
};

template <int LF, int EPI, int PR = 0>
__device__ __forceinline__ void col_store_f32(const ColOutF& o, int i, int c, float v0, float v1) {
    if constexpr (EPI == kToSmem) {
        *reinterpret_cast<float2*>(o.G + i * LF + c) = make_float2(v0, v1);
    } else if constexpr (EPI == kToGlobal) {
        *reinterpret_cast<float2*>(o.G + i * o.gs + c) = make_float2(v0, v1);
    } else {  // kFinish, as col_store
        const int pi = panel_index<PR>(i, c);
        const float2 w0 = *reinterpret_cast<const float2*>(o.w0 + pi);
        v0 = v0 * w0.x;
        v1 = v1 * w0.y;
        *reinterpret_cast<float2*>(o.qs + pi) = make_float2(v0, v1);
        if (o.start) {
            const float2 w1 = *reinterpret_cast<const float2*>(o.w1 + pi);
            *reinterpret_cast<float2*>(o.G + i * LF + c) = make_float2(v0 * w1.x, v1 * w1.y);
        }
    }
}

// G[i][c] = sum_j A[i][j] F[j][c] on an R x C slab: m16 tiles over i, n8 tiles over c
template <int R, int C, int LF, bool EO, int EPI = kToSmem>
__device__ __forceinline__ void col_op_f32(const float* __restrict__ F, const ColOutF& out,
                                           const float* __restrict__ op) {
    using S = AxisShapeF<R, EO>;
    constexpr int MI = S::K, K = S::K, LD = S::LD;
    constexpr int TM = MI / 16, TN = C / 8;
    constexpr int BN = (TN + 1) / 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int blk = warp; blk < TM * BN; blk += kContourThreads / 32) {
        const int m0 = (blk / BN) * 16, nb = (blk % BN) * 2;
        const bool n1 = (TN % 2 == 0) || (nb + 1 < TN);
        float dP[2][4] = {}, dR[2][4] = {};
        const float* Eh0 = op + (m0 + g) * LD + t;
        const float* Eh1 = Eh0 + 8 * LD;
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 8) {
            unsigned ah[4] = {__float_as_uint(Eh0[k0]), __float_as_uint(Eh1[k0]), __float_as_uint(Eh0[k0 + 4]),
                              __float_as_uint(Eh1[k0 + 4])};
            unsigned al[4] = {__float_as_uint(Eh0[k0 + S::PART]), __float_as_uint(Eh1[k0 + S::PART]),
                              __float_as_uint(Eh0[k0 + 4 + S::PART]), __float_as_uint(Eh1[k0 + 4 + S::PART])};
            unsigned oh[4], ol[4];
            if (EO) {
                oh[0] = __float_as_uint(Eh0[k0 + S::HALF]);
                oh[1] = __float_as_uint(Eh1[k0 + S::HALF]);
                oh[2] = __float_as_uint(Eh0[k0 + 4 + S::HALF]);
                oh[3] = __float_as_uint(Eh1[k0 + 4 + S::HALF]);
                ol[0] = __float_as_uint(Eh0[k0 + S::HALF + S::PART]);
                ol[1] = __float_as_uint(Eh1[k0 + S::HALF + S::PART]);
                ol[2] = __float_as_uint(Eh0[k0 + 4 + S::HALF + S::PART]);
                ol[3] = __float_as_uint(Eh1[k0 + 4 + S::HALF + S::PART]);
            }
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if (b == 1 && !n1) continue;
                const int c = (nb + b) * 8 + g;
                const int j0 = k0 + t, j1 = k0 + t + 4;
                const float x0 = F[j0 * LF + c], x1 = F[j1 * LF + c];
                unsigned uh[2], ul[2];
                if (EO) {
                    const float y0 = F[(R - 1 - j0) * LF + c], y1 = F[(R - 1 - j1) * LF + c];
                    unsigned vh[2], vl[2];
                    split_tf32(x0 + y0, uh[0], ul[0]);
                    split_tf32(x1 + y1, uh[1], ul[1]);
                    split_tf32(x0 - y0, vh[0], vl[0]);
                    split_tf32(x1 - y1, vh[1], vl[1]);
                    mma_3xtf32(dP[b], ah, al, uh, ul);
                    mma_3xtf32(dR[b], oh, ol, vh, vl);
                } else {
                    split_tf32(x0, uh[0], ul[0]);
                    split_tf32(x1, uh[1], ul[1]);
                    mma_3xtf32(dP[b], ah, al, uh, ul);
                }
            }
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            if (b == 1 && !n1) continue;
            const int c = (nb + b) * 8 + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = m0 + g + 8 * h;
                const float p0 = dP[b][2 * h], p1 = dP[b][2 * h + 1];
                if (EO) {
                    const float r0 = dR[b][2 * h], r1 = dR[b][2 * h + 1];
                    col_store_f32<LF, EPI, R>(out, i, c, p0 + r0, p1 + r1);
                    col_store_f32<LF, EPI, R>(out, R - 1 - i, c, p0 - r0, p1 - r1);
                } else {
                    col_store_f32<LF, EPI, R>(out, i, c, p0, p1);
                }
            }
        }
    }
}

// col_op_f32 into a shared-memory slab G
template <int R, int C, int LF, bool EO>
__device__ __forceinline__ void col_op_f32(const float* __restrict__ F, float* __restrict__ G,
                                           const float* __restrict__ op) {
    const ColOutF o{G, 0};
    col_op_f32<R, C, LF, EO, kToSmem>(F, o, op);
}

// N x N FP32 tile from global (row stride gs) into shared memory (row stride LF) with cp.async
template <int N, int LF>
__device__ __forceinline__ void tile_fetch_f32(float* sm, const float* gm, long long gs) {
    constexpr int PER_ROW = N / 4;
    constexpr int TOTAL = N * PER_ROW;
#pragma unroll 4
    for (int e = threadIdx.x; e < TOTAL; e += kContourThreads) {
        const int r = e / PER_ROW, c = (e - r * PER_ROW) * 4;
        cp_async16(sm + r * LF + c, gm + r * gs + c);
    }
}

// T <- T * W (T row stride LF, W in 8-column panels)
template <int N, int LF>
__device__ __forceinline__ void tile_scale_f32(float* T, const float* W) {
    constexpr int PER_ROW = N / 4;
    constexpr int TOTAL = N * PER_ROW;
#pragma unroll 4
    for (int e = threadIdx.x; e < TOTAL; e += kContourThreads) {
        const int r = e / PER_ROW, c = (e - r * PER_ROW) * 4;
        float4 v = *reinterpret_cast<float4*>(T + r * LF + c);
        const float4 w = *reinterpret_cast<const float4*>(W + panel_index<N>(r, c));
        v.x *= w.x;
        v.y *= w.y;
        v.z *= w.z;
        v.w *= w.w;
        *reinterpret_cast<float4*>(T + r * LF + c) = v;
    }
}

// Shared memory: operators, two padded work tiles, the four Boltzmann-factor tiles of
// this block's unit (blocks A and B, plane and slab layout; loaded once per launch by
// TMA) and the q staging tile, both in 8-column panels (the finishing epilogue's layout).
template <int N, bool EO>
struct AltShapeF {
    static constexpr int LF = N + 4;
    static constexpr int OPS = 3 * AxisShapeF<N, EO>::SIZE;
    static constexpr int OPS_PAD = (OPS + 31) & ~31;  // 128-byte aligned tiles after it
    static constexpr int TILE = (N * LF + 31) & ~31;
    static constexpr int WT = N * N;
    // + 128: the carve-up starts at the first 128-byte boundary of the dynamic window
    static constexpr size_t SMEM = (size_t)(OPS_PAD + 2 * TILE + 5 * WT) * sizeof(float) + 128;
    // with the fused phi sums: the other chain's tile (FP32) and the products (FP64)
    static constexpr size_t SMEM_FUSED = SMEM + (size_t)WT * (sizeof(float) + sizeof(double));
};

struct ContourArgsF {
    float* q[2];
    const float* wds[2];
    float* xbuf[2];        // 2 x space_size_phy per chain
    const float* ops;      // packed FP32 operators (hi/lo), x then y then z
    int nchain;
    long long slot0[2];
    int dir[2];
    long long NsA;
    int t_end;
    int* error;
    long long spin_limit;
    unsigned* flags;       // [chain][plane|slab][consumer][producer], zeroed by the host
    double* phi_acc;       // fused phi sums (null: off; the launch then has SMEM_FUSED), as ContourArgs
    unsigned* done;
    alignas(64) CUtensorMap tm_pq[2][2];  // panel tiles, as ContourArgs::tm_pq / tm_pw
    alignas(64) CUtensorMap tm_pw[2][2];
};

template <int N, bool EO>
__global__ void __launch_bounds__(kContourThreads, 1) contour_alt_kernel_f32(const __grid_constant__ ContourArgsF a) {
    using S = AltShapeF<N, EO>;
    constexpr int LF = S::LF;
    constexpr int OFFY = AxisShapeF<N, EO>::SIZE;
    constexpr int OFFZ = 2 * AxisShapeF<N, EO>::SIZE;
    constexpr int TPR = kContourThreads / N;
    constexpr int CPT = (N / 4 + TPR - 1) / TPR;
    constexpr unsigned TILE_BYTES = N * N * sizeof(float);
    static_assert(TPR >= 1, "tile rows must not exceed the block");
    extern __shared__ __align__(128) unsigned char smemf_raw[];
    // the dynamic window is only guaranteed 16-byte alignment; TMA tiles need 128
    float* smemf = reinterpret_cast<float*>(smemf_raw + ((128u - (smem_u32(smemf_raw) & 127u)) & 127u));
    float* sops = smemf;
    float* T0 = smemf + S::OPS_PAD;
    float* T1 = T0 + S::TILE;
    float* WP = T1 + S::TILE;  // [block A, block B] plane-layout factors of this unit
    float* WS = WP + 2 * S::WT;  // [block A, block B] slab-layout factors
    float* QS = WS + 2 * S::WT;  // finished q(s+1), drained by bulk stores
    float* XF = QS + S::WT;      // fused phi: the other chain's tile of the slot
    double* PD = reinterpret_cast<double*>(XF + S::WT);  // fused phi: the products, bulk-added
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ __align__(8) unsigned long long s_xbar;
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
    const int c = u >= N ? 1 : 0, p = u - c * N;
    const int dir = c ? a.dir[1] : a.dir[0];
    const long long slot0 = c ? a.slot0[1] : a.slot0[0];
    float* q = c ? a.q[1] : a.q[0];
    float* XP = c ? a.xbuf[1] : a.xbuf[0];
    float* XS = XP + M;
    // flags[chain][producing layout][consumer][producer]: every consumer polls its own
    // N flags (one cache line per 32), written by the producers (push), so the waits of
    // different blocks never share a line
    unsigned* fl_plane = a.flags + (size_t)c * 2 * N * N;  // written by plane units
    unsigned* fl_slab = fl_plane + (size_t)N * N;           // written by slab units
    const int U = a.t_end;
    const bool fphi = a.phi_acc != nullptr;
    {
        const void* tiles[7] = {WP, WP + S::WT, WS, WS + S::WT, QS, XF, PD};
        const int e = tma_alignment_error(tiles, fphi ? 7 : 5, &a.tm_pq[0][0], 4) |
                      tma_alignment_error(tiles, 0, &a.tm_pw[0][0], 4);
        if (e) {
            if (threadIdx.x == 0) atomicOr(a.error, e);
            return;
        }
    }
    // Fused phi, as in the FP64 alternating kernel (contour_kernel.cuh): in the second half of
    // the contour the phase that finishes slot s bulk-loads the other chain's tile of slot s,
    // forms the products in FP64 (exact for FP32 factors) and bulk-adds them into the FP64
    // accumulator tile of the slot's block and the layout, in phase order.
    const int co = 1 - c;
    double* acc_unit = fphi ? a.phi_acc + (size_t)c * 4 * M + (size_t)p * PLANE : nullptr;
    auto x_active = [&](int k) -> bool {
        const long long s = slot0 + (long long)dir * k, kq = (s - a.slot0[co]) * a.dir[co];
        return fphi && k >= 1 && k <= U && kq >= 1 && kq <= k - 2 && ((k - kq) & 1) == 0 && s != a.NsA;
    };
    unsigned xpar = 0, x_seen = 0;
    bool x_pend = false;

    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(&s_bar, 1);
        mbar_init(&s_xbar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == 0) {
        // the unit's Boltzmann factors of both blocks in both layouts, once per launch
        if ((threadIdx.x & 31) == 0) mbar_expect_tx(&s_bar, 4 * TILE_BYTES);
        __syncwarp();
        if ((threadIdx.x & 31) == 0)  // in 8-column panels, the layout the finishing epilogue reads
            for (int b = 0; b < 2; ++b) {
                tma_load_4d(WP + b * S::WT, &a.tm_pw[b][0], 0, 0, 0, p, &s_bar);
                tma_load_4d(WS + b * S::WT, &a.tm_pw[b][1], 0, 0, 0, p, &s_bar);
            }
    }
    op_copy_async(sops, a.ops, S::OPS);
    cp_async_wait_all();
    // block (0: A, 1: B) of the Boltzmann factor of step s
    auto blk_of = [&](int s) -> int {
        const long long in_slot = slot0 + (long long)dir * s;
        const long long seg = dir > 0 ? in_slot : in_slot - 1;
        return seg < a.NsA ? 0 : 1;
    };
    if (!mbar_wait(&s_bar, 0, a.spin_limit)) s_fail = 1;
    __syncthreads();
    if (s_fail) {  // every thread leaves here: the factor tiles still land in this block's memory first
        if (threadIdx.x == 0) {
            atomicOr(a.error, 2);
            mbar_wait(&s_bar, 0, kDrainSpins);
        }
        return;
    }

    for (int k = 0; k <= U; ++k) {
        const bool plane = (k & 1) == 0;
        const long long off = plane ? (long long)p * PLANE : (long long)p * N;
        const long long gs = plane ? N : PLANE;
        const float* Wl = plane ? WP : WS;
        if (k == 0) {
            tile_fetch_f32<N, LF>(T0, q + slot0 * M + off, gs);
        } else {
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
                const float* src = (plane ? XS : XP) + off + r * gs;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int ch = sub + j * TPR;
                    if (ch < N / 4) cp_async16(T0 + r * LF + 4 * ch, src + 4 * ch);
                }
            }
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        if (s_fail) {
            if (x_pend) mbar_wait(&s_xbar, xpar, kDrainSpins);
            if (warp == 0) bulk_wait_all();
            return;
        }
        const long long s_fin = slot0 + (long long)dir * k;
        const long long kp = (s_fin - a.slot0[co]) * a.dir[co];
        const bool xact = x_active(k);
        float* cur = T0;
        float* oth = T1;
        if (k >= 1) {
            // finish step k-1: the axis ops this layout owns; the last one's epilogue applies
            // D, writes q(s+1) to the panel staging tile and D q(s+1) to the work tile
            if (plane) row_op_f32<N, N, LF, EO>(cur, oth, sops + OFFZ);
            if (warp == 0) bulk_wait_read();  // the previous q store has left QS
            __syncthreads();
            ColOutF fo{plane ? cur : oth, 0};
            fo.w0 = Wl + blk_of(k - 1) * S::WT;
            fo.w1 = Wl + (k < U ? blk_of(k) : 0) * S::WT;
            fo.qs = QS;
            fo.start = k < U;
            col_op_f32<N, N, LF, EO, kFinish>(plane ? oth : cur, fo, sops + (plane ? OFFY : 0));
            if (!plane) {
                float* tmp = cur;
                cur = oth;
                oth = tmp;
            }
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tma_store_5d(&a.tm_pq[c][plane ? 0 : 1], QS, 0, 0, 0, p, (int)(slot0 + (long long)dir * k));
                bulk_commit();
                if (xact) {  // XF was last read by the previous product pass (block barriers since)
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
                        tma_load_5d(XF, &a.tm_pq[co][plane ? 0 : 1], 0, 0, 0, p, (int)s_fin, &s_xbar);
                    }
                }
            }
        } else {
            tile_scale_f32<N, LF>(cur, Wl + blk_of(0) * S::WT);
            __syncthreads();
        }
        if (k < U) {
            // start step k; the last op's epilogue writes the exchange buffer
            const ColOutF xo{(plane ? XP : XS) + off, gs};
            if (plane) {
                row_op_f32<N, N, LF, EO>(cur, oth, sops + OFFZ);
                __syncthreads();
                col_op_f32<N, N, LF, EO, kToGlobal>(oth, xo, sops + OFFY);
            } else {
                col_op_f32<N, N, LF, EO, kToGlobal>(cur, xo, sops);
            }
            __syncthreads();
            if (xact && s_fail) {  // thread 0 gave up on the other chain's store: no load in flight
                if (warp == 0) bulk_wait_all();
                return;
            }
            if (threadIdx.x < N) {  // tell consumer threadIdx.x that tile p of phase k is out
                __threadfence();
                st_release_u32((plane ? fl_plane : fl_slab) + (size_t)threadIdx.x * N + p, (unsigned)(k + 1));
            }
            if (fphi && threadIdx.x == 0 && 2 * k == U) {  // the stores before the midpoint have landed
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
        if (xact) {
            if (threadIdx.x == 0) bulk_wait_read();  // the last bulk add has read PD
            if (mbar_wait(&s_xbar, xpar, a.spin_limit)) {
                xpar ^= 1u;
            } else {
                x_pend = true;
                s_fail = 1;
                atomicOr(a.error, 2);
            }
            __syncthreads();
            if (s_fail) {
                if (x_pend) mbar_wait(&s_xbar, xpar, kDrainSpins);
                if (warp == 0) bulk_wait_all();
                return;
            }
            for (int i = 2 * threadIdx.x; i < N * N; i += 2 * kContourThreads) {
                const float2 v = *reinterpret_cast<const float2*>(QS + i);
                const float2 w = *reinterpret_cast<const float2*>(XF + i);
                *reinterpret_cast<double2*>(PD + i) = make_double2((double)v.x * w.x, (double)v.y * w.y);
            }
            fence_async_smem();
            __syncthreads();  // also ends the phase
            if (threadIdx.x == 0) {
                bulk_wait_newest3();  // the add into this tile two phases back has completed
                bulk_reduce_add_f64(acc_unit + (size_t)((s_fin < a.NsA ? 0 : 2) + (plane ? 0 : 1)) * M, PD,
                                    N * N * (unsigned)sizeof(double));
                bulk_commit();
            }
        } else {
            __syncthreads();
        }
    }
    if (warp == 0) bulk_wait_all();
}

}  // namespace crysscft
