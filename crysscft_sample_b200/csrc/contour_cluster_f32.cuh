// FP32 precision form of the whole-contour kernel on thread-block clusters (64^3 grids).
//
// An FP32 contour chain of a 64^3 grid is 1 MB: it fits in the shared memory of one
// 16-CTA cluster, so each chain runs on its own cluster and the transposition every
// contour step needs goes through distributed shared memory (DSMEM) with one hardware
// cluster barrier per step, instead of global-memory exchange buffers and release flags.
// CTA r of a cluster owns the x-planes 4r..4r+3 (plane layout P[x][y][z]) and the
// y-slabs 4r..4r+3 (slab layout S[y][x][z]).  Phases alternate between the layouts:
//
//   plane phase:  [A_y]  D  store q  D  [A_y] [A_z]  -> push z-lines into the slab owners
//   slab phase:   [A_x]  D  store q  D  [A_x] [A_z]  -> push z-lines into the plane owners
//
// The first axis operation finishes the previous contour step, the other two start the
// next one (the three axis operators commute), so every step costs one cluster barrier.
// The two operations of one orientation keep the line in registers between them.
//
// Axis operations run on the 5th-generation tensor cores (tcgen05.mma kind::f16,
// M = 128 lines, N = 32, K = 16), in even/odd form (u = x_j + x_{63-j}, v = x_j - x_{63-j},
// p = E u, r = O v, y_i = p_i + r_i, y_{63-i} = p_i - r_i).  Each line is scaled by a power of
// two so its largest value lies in [1, 2), and every FP32 operand x is split into two fp16
// parts x = hi + 2^-12 lo (hi = fp16(x), lo = fp16((x - hi) 2^12)); the operators are split
// the same way on the host.  a b ~ a_hi b_hi + 2^-12 (a_lo b_hi + a_hi b_lo), the same
// 22-bit parts and the same dropped lo*lo term as 3xTF32 splitting, at the f16 tensor rate.
// The A operand (the split line) lives in tensor memory (TMEM), the operator parts in
// shared memory.  The tensor cores round an MMA's FP32 result toward zero: the large
// hi*hi products of the two K-steps therefore go to separate zero-initialised
// accumulators (one truncation each, then a round-to-nearest add), and the small parts to
// a third one whose truncation is 2^-12 smaller.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "contour_kernel.cuh"

namespace crysscft {

constexpr int kClN = 64;                        // grid side
constexpr int kClCtas = 16;                     // CTAs per cluster (one chain)
constexpr int kClThreads = 256;                 // 8 warps: two blocks of 128 lines
constexpr int kClPlanes = kClN / kClCtas;       // planes (slabs) per CTA
constexpr int kClField = kClPlanes * kClN * kClN;  // floats per layout buffer (64 KB)
constexpr int kClOpMat = 32 * 32;               // fp16 values of one 32 x 32 operator part
constexpr int kClOpAxis = 4 * kClOpMat;         // [E_hi | E_lo | O_hi | O_lo] per axis
// shared memory: P, S, the Boltzmann-factor tile, the three axes' operator parts
constexpr size_t kClSmem = (size_t)3 * kClField * sizeof(float) + (size_t)3 * kClOpAxis * sizeof(__half) + 1024;

struct ClusterArgsF {
    float* q[2];           // contour stores of the two chains ((U + 1) slices of n^3)
    const float* wds[2];   // exp(-w ds / 2) of blocks A and B
    const __half* ops;     // 3 x kClOpAxis fp16 values, axes x, y, z (pack_operator_h16)
    long long slot0[2];
    int dir[2];
    long long NsA;
    int U;                 // contour steps per chain
    int* error;            // bit 1: a wait ran out; bit 2: launch shape
    long long spin_limit;
};

// ---- tcgen05 -----------------------------------------------------------------------
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc512(unsigned* dst) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(dst)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc512(unsigned taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(taddr) : "memory");
}
// D[tmem] (+)= A[tmem] * B[smem]^T, M = 128, N = 32, K = 16, fp16 inputs, FP32 accumulate
__device__ __forceinline__ void mma_f16_ts(unsigned d, unsigned a, unsigned long long bdesc, unsigned accumulate) {
    constexpr unsigned kIdesc = (1u << 4) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %4, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(accumulate), "r"(kIdesc)
        : "memory");
}
// Bounded wait on an mbarrier phase with the non-blocking test (try_wait may suspend the
// thread for a hardware-chosen time inside one poll, so a poll count would not bound the
// wait's length, and a limit of one poll would not reliably run out)
__device__ __forceinline__ bool cl_mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
    long long spins = 0;
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (++spins > limit) return false;
        if (spins > 64) __nanosleep(20);
    }
}
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// shared-memory descriptor of a canonical K-major operand without swizzle: 8-row groups
// `sbo` bytes apart, 16-byte K chunks 128 bytes apart (sm100 descriptor version 1)
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned sbo) {
    return (unsigned long long)((saddr >> 4) & 0x3FFF) | ((unsigned long long)(128u >> 4) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tmem_st16(unsigned taddr, const unsigned (&r)[16]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
                 ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
                 "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
                 : "memory");
}
__device__ __forceinline__ void tmem_ld8(unsigned taddr, float (&v)[8]) {
    unsigned r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---- clusters ------------------------------------------------------------------------
__device__ __forceinline__ unsigned cluster_ctarank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_id_x() {
    unsigned r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned dsmem_addr(const void* local, unsigned rank) {
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_dsmem_v4(unsigned addr, float a, float b, float c, float d) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}
// every CTA of the cluster arrives once per call: the writes before it (DSMEM included)
// are visible to all CTAs after it
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// untiled bulk copy global -> shared, completing on `bar`
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// position of (line-major index a*64 + b, element z) in a swizzled P/S buffer: the 16-byte
// chunk index of z is XORed with b % 16, so lines along b (fixed a, z) and lines along z
// (fixed a, b) are both read without bank conflicts
__device__ __forceinline__ int cl_idx(int a, int b, int z) {
    return ((a * kClN + b) << 6) + ((((z >> 2) ^ (b & 15)) << 2) | (z & 3));
}

// ---- one axis operation on 256 lines (two M = 128 blocks) ----------------------------
// TMEM columns of block k (k = 0, 1): 256 k + {0: P_hi0, 32: P_hi1, 64: P_small, 96: R_hi0,
// 128: R_hi1, 160: R_small, 192: u_hi, 208: u_lo, 224: v_hi, 240: v_lo}
struct ClOp {
    unsigned tmem;               // allocation base (lane 0, column 0)
    unsigned long long* bar;     // [2] MMA completion of blocks 0 and 1
    long long limit;
};

// v: the line (64 values along the operator's axis) in, the result out.  opaxis: the
// axis's [E_hi | E_lo | O_hi | O_lo] parts in shared memory.  Every thread of the CTA calls
// it; `skip` is the same on all of them (an earlier failure: nothing is issued).  Returns
// false when this thread's wait for the products ran out (the line is then left as it was).
__device__ __forceinline__ bool cl_axis_op(float (&v)[64], const __half* opaxis, const ClOp& o, unsigned (&ph)[2],
                                           bool skip) {
    const int tid = threadIdx.x, warp = tid >> 5;
    const int blk = warp >> 2;
    const unsigned lane_base = (unsigned)((warp & 3) * 32) << 16;
    const unsigned cb = o.tmem + (unsigned)(blk * 256);
    // scale by 2^-e so that max |v| lies in [1, 2): exact, undone after the products
    float mx = 0.f;
#pragma unroll
    for (int j = 0; j < 64; ++j) mx = fmaxf(mx, fabsf(v[j]));
    const unsigned ex = (__float_as_uint(mx) >> 23) & 0xffu;
    const bool scaled = ex >= 1u && ex <= 253u;
    const float sc = scaled ? __uint_as_float((254u - ex) << 23) : 1.0f;
    const float inv = scaled ? __uint_as_float(ex << 23) : 1.0f;
    if (!skip) {
        unsigned uh[16], ul[16], vh[16], vl[16];
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            float a[2], b[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                a[e] = (v[j + e] + v[63 - j - e]) * sc;
                b[e] = (v[j + e] - v[63 - j - e]) * sc;
            }
            __half ah[2], al[2], bh[2], bl[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                ah[e] = __float2half_rn(a[e]);
                al[e] = __float2half_rn((a[e] - __half2float(ah[e])) * 4096.0f);
                bh[e] = __float2half_rn(b[e]);
                bl[e] = __float2half_rn((b[e] - __half2float(bh[e])) * 4096.0f);
            }
            uh[j / 2] = (unsigned)__half_as_ushort(ah[0]) | ((unsigned)__half_as_ushort(ah[1]) << 16);
            ul[j / 2] = (unsigned)__half_as_ushort(al[0]) | ((unsigned)__half_as_ushort(al[1]) << 16);
            vh[j / 2] = (unsigned)__half_as_ushort(bh[0]) | ((unsigned)__half_as_ushort(bh[1]) << 16);
            vl[j / 2] = (unsigned)__half_as_ushort(bl[0]) | ((unsigned)__half_as_ushort(bl[1]) << 16);
        }
        tmem_st16(cb + lane_base + 192, uh);
        tmem_st16(cb + lane_base + 208, ul);
        tmem_st16(cb + lane_base + 224, vh);
        tmem_st16(cb + lane_base + 240, vl);
        tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (skip) return true;
    if (tid == 0) {
        const unsigned sop = smem_u32(opaxis);
        constexpr unsigned kSbo = 512;     // 32 K values = 4 chunks of 128 bytes per 8 rows
        constexpr unsigned kMat = kClOpMat * sizeof(__half);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const unsigned c = o.tmem + (unsigned)(k * 256);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const unsigned long long eh = umma_desc(sop + 0 * kMat + s * 256, kSbo);
                const unsigned long long el = umma_desc(sop + 1 * kMat + s * 256, kSbo);
                const unsigned long long oh = umma_desc(sop + 2 * kMat + s * 256, kSbo);
                const unsigned long long ol = umma_desc(sop + 3 * kMat + s * 256, kSbo);
                const unsigned as = (unsigned)(s * 8);
                mma_f16_ts(c + 0 + s * 32, c + 192 + as, eh, 0u);   // P_hi_s = u_hi E_hi (K-step s)
                mma_f16_ts(c + 64, c + 208 + as, eh, s);            // P_small += u_lo E_hi
                mma_f16_ts(c + 64, c + 192 + as, el, 1u);           //          + u_hi E_lo
                mma_f16_ts(c + 96 + s * 32, c + 224 + as, oh, 0u);  // R_hi_s = v_hi O_hi
                mma_f16_ts(c + 160, c + 240 + as, oh, s);           // R_small += v_lo O_hi
                mma_f16_ts(c + 160, c + 224 + as, ol, 1u);          //          + v_hi O_lo
            }
            mma_commit(&o.bar[k]);
        }
    }
    // wait for this block's products (bounded)
    const bool ok = cl_mbar_wait(&o.bar[blk], ph[blk], o.limit);
    ph[0] ^= 1u;
    ph[1] ^= 1u;
    if (!ok) return false;
    tc_fence_after();
    constexpr float kSmall = 1.0f / 4096.0f;
#pragma unroll
    for (int i0 = 0; i0 < 32; i0 += 8) {
        float p0[8], p1[8], ps[8], r0[8], r1[8], rs[8];
        const unsigned t = cb + lane_base + (unsigned)i0;
        tmem_ld8(t + 0, p0);
        tmem_ld8(t + 32, p1);
        tmem_ld8(t + 64, ps);
        tmem_ld8(t + 96, r0);
        tmem_ld8(t + 128, r1);
        tmem_ld8(t + 160, rs);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const float p = fmaf(ps[e], kSmall, p0[e] + p1[e]);
            const float r = fmaf(rs[e], kSmall, r0[e] + r1[e]);
            v[i0 + e] = (p + r) * inv;
            v[63 - i0 - e] = (p - r) * inv;
        }
    }
    tc_fence_before();
    return true;
}

// block (0: A, 1: B) of the Boltzmann factor of contour step s of a chain
__device__ __forceinline__ int cl_block_of(long long slot0, int dir, long long NsA, int s) {
    const long long in_slot = slot0 + (long long)dir * s;
    const long long seg = dir > 0 ? in_slot : in_slot - 1;
    return seg < NsA ? 0 : 1;
}

// Issue the Boltzmann-factor tile of a phase: plane layout = the CTA's 4 x-planes (one
// contiguous 64 KB copy), slab layout = rows y = 4r..4r+3 of every x-plane (64 x 1 KB),
// stored as [x][y - 4r][z].
__device__ __forceinline__ void cl_load_d(float* Db, const float* w, bool plane, unsigned r,
                                          unsigned long long* bar) {
    constexpr unsigned kBytes = kClField * sizeof(float);
    mbar_expect_tx(bar, kBytes);
    if (plane) {
        bulk_load(Db, w + (size_t)r * kClPlanes * kClN * kClN, kBytes, bar);
    } else {
        for (int x = 0; x < kClN; ++x)
            bulk_load(Db + x * kClPlanes * kClN, w + (size_t)x * kClN * kClN + (size_t)r * kClPlanes * kClN,
                      kBytes / kClN, bar);
    }
}

__global__ void __launch_bounds__(kClThreads, 1) contour_cluster_kernel_f32(const __grid_constant__ ClusterArgsF a) {
    extern __shared__ __align__(1024) unsigned char cl_raw[];
    unsigned char* base = cl_raw + ((1024u - (smem_u32(cl_raw) & 1023u)) & 1023u);
    float* P = reinterpret_cast<float*>(base);
    float* S = P + kClField;
    float* Db = S + kClField;
    __half* sop = reinterpret_cast<__half*>(Db + kClField);
    __shared__ __align__(8) unsigned long long s_bar_mma[2];
    __shared__ __align__(8) unsigned long long s_bar_d;
    __shared__ unsigned s_tmem;

    constexpr long long M = (long long)kClN * kClN * kClN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned r = cluster_ctarank();
    const int c = (int)cluster_id_x();
    if (gridDim.x != 2 * kClCtas || c > 1) {  // launch shape fixed by the host: 2 clusters of 16
        if (tid == 0) atomicOr(a.error, 4);
        return;  // every CTA takes this branch (the condition is uniform over the grid)
    }
    const long long slot0 = a.slot0[c];
    const int dir = a.dir[c];
    float* q = a.q[c];
    // a thread's line: 32 w + lane -> (a_, t_) with a_ = the local plane/slab, t_ its position
    const int la = warp >> 1;
    const int lt = (warp & 1) * 32 + lane;

    if (tid == 0) {
        mbar_init(&s_bar_mma[0], 1);
        mbar_init(&s_bar_mma[1], 1);
        mbar_init(&s_bar_d, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc512(&s_tmem);
    // the operators of the three axes (24 KB) with 16-byte cp.async chunks
    for (int e = tid; e < 3 * kClOpAxis / 8; e += kClThreads) cp_async16(sop + 8 * e, a.ops + 8 * e);
    cp_async_commit();
    cp_async_wait_all();
    fence_async_smem();  // the tensor cores read the operator parts through the async proxy
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const ClOp op{s_tmem, s_bar_mma, a.spin_limit};
    unsigned ph[2] = {0u, 0u};
    unsigned dph = 0;                 // parity of the next Boltzmann-tile completion
    bool d_pending = false;           // thread 0: a tile copy is in flight
    bool mma_issued = false;          // some MMA was issued (thread 0 drains them on failure)
    bool failed = false;              // uniform over the CTA (combined at every barrier)
    if (tid == 0) {
        cl_load_d(Db, a.wds[cl_block_of(slot0, dir, a.NsA, 0)], true, r, &s_bar_d);
        d_pending = true;
    }
    // no CTA writes into another's shared memory before all of them are running
    cluster_sync_all();

    float v[64];
    for (int j = 0; j <= a.U; ++j) {
        const bool plane = (j & 1) == 0;
        float* buf = plane ? P : S;
        const __half* opA = sop + (plane ? 1 : 0) * kClOpAxis;  // A_y (plane) or A_x (slab)
        const __half* opZ = sop + 2 * kClOpAxis;
        // global offset of element b of this thread's strided line: plane: (x = 4r + la,
        // y = b, z = lt); slab: (x = b, y = 4r + la, z = lt)
        const long long g0 = plane ? ((long long)(r * kClPlanes + la) * kClN * kClN + lt)
                                   : ((long long)(r * kClPlanes + la) * kClN + lt);
        const long long gstride = plane ? kClN : (long long)kClN * kClN;
        bool bad = false;
        // ---- finish step j - 1 (or load q(0))
        if (j == 0) {
            const float* src = q + slot0 * M + g0;
#pragma unroll
            for (int b = 0; b < 64; ++b) v[b] = src[b * gstride];
        } else {
#pragma unroll
            for (int b = 0; b < 64; ++b) v[b] = buf[cl_idx(la, b, lt)];
            mma_issued |= !failed;
            bad |= !cl_axis_op(v, opA, op, ph, failed);
        }
        // ---- D, store q(j), D
        if (!failed) {
            if (cl_mbar_wait(&s_bar_d, dph, a.spin_limit)) {
                if (tid == 0) d_pending = false;  // a copy that did not land is drained at exit
                dph ^= 1u;
            } else {
                bad = true;
            }
        }
        if (!failed && !bad) {
            const int bcur = j >= 1 ? cl_block_of(slot0, dir, a.NsA, j - 1) : -1;
            const int bnext = j < a.U ? cl_block_of(slot0, dir, a.NsA, j) : -1;
            // the tile holds block bnext for j = 0 and block bcur after; a different next
            // block (once per chain, where it crosses from A to B) is read from global memory
            const float* wn = (j >= 1 && bnext >= 0 && bnext != bcur) ? a.wds[bnext] : nullptr;
            float* dst = q + (slot0 + (long long)dir * j) * M + g0;
#pragma unroll
            for (int b = 0; b < 64; ++b) {
                const float d = plane ? Db[(la * kClN + b) * kClN + lt] : Db[(b * kClPlanes + la) * kClN + lt];
                float x = v[b];
                if (j >= 1) {
                    x *= d;
                    dst[b * gstride] = x;
                }
                if (bnext >= 0) x *= wn ? wn[g0 + b * gstride] : d;
                v[b] = x;
            }
        }
        failed = __syncthreads_or(failed || bad) != 0;  // also: the tile has been read by every thread
        if (j == a.U) break;
        if (tid == 0 && !failed) {
            fence_async_smem();
            cl_load_d(Db, a.wds[cl_block_of(slot0, dir, a.NsA, j)], !plane, r, &s_bar_d);
            d_pending = true;
        }
        // ---- start step j: the strided axis again, from registers, then A_z
        mma_issued |= !failed;
        bad |= !cl_axis_op(v, opA, op, ph, failed);
        if (!failed && !bad) {
#pragma unroll
            for (int b = 0; b < 64; ++b) buf[cl_idx(la, b, lt)] = v[b];
        }
        failed = __syncthreads_or(failed || bad) != 0;
        // z-lines: line (la, lt) of the buffer, 16 swizzled 16-byte chunks
#pragma unroll
        for (int cz = 0; cz < 16; ++cz) {
            const float4 t = *reinterpret_cast<const float4*>(buf + ((la * kClN + lt) << 6) + ((cz ^ (lt & 15)) << 2));
            v[4 * cz] = t.x;
            v[4 * cz + 1] = t.y;
            v[4 * cz + 2] = t.z;
            v[4 * cz + 3] = t.w;
        }
        bad |= !cl_axis_op(v, opZ, op, ph, failed);
        // push the z-line (la, lt) to its owner in the other layout: plane -> slab owner of
        // y = lt (row (y % 4, x = 4r + la)); slab -> plane owner of x = lt (row (x % 4, y = 4r + la))
        if (!failed && !bad) {
            float* other = plane ? S : P;
            const int row_a = lt & 3, row_b = (int)r * kClPlanes + la;
            const unsigned dst = dsmem_addr(other + ((row_a * kClN + row_b) << 6), (unsigned)(lt >> 2));
#pragma unroll
            for (int cz = 0; cz < 16; ++cz)
                st_dsmem_v4(dst + (unsigned)(((cz ^ (row_b & 15)) << 2) * sizeof(float)), v[4 * cz], v[4 * cz + 1],
                            v[4 * cz + 2], v[4 * cz + 3]);
        }
        failed = __syncthreads_or(failed || bad) != 0;
        cluster_sync_all();
    }
    // leave: products and tile copies still in flight after a failure land first (bounded),
    // then TMEM goes back
    if (failed && tid == 0) {
        atomicOr(a.error, 2);
        if (mma_issued) {
            // tcgen05.commit tracks every earlier MMA of this thread: the last commit of
            // each block covers them all (its parity is the one before the last toggle)
            mbar_wait(&s_bar_mma[0], ph[0] ^ 1u, kDrainSpins);
            mbar_wait(&s_bar_mma[1], ph[1] ^ 1u, kDrainSpins);
        }
        if (d_pending) mbar_wait(&s_bar_d, dph, kDrainSpins);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc512(s_tmem);
    cluster_sync_all();  // no CTA leaves while another may still address its shared memory
}

}  // namespace crysscft
