// Field kernels of one SCFT iteration (FP64 fields; contour slices of type T).
//
//  prep    : calc_ksi (src/crysSCFT_sample.cpp:341-346), array_exp (:315-322) for the
//            two Boltzmann factors, and the initial slices q(0) = 1, q+(end) = 1 (:483)
//  Q       : array_average of q+_A(0) (:324-331, :494)
//  phi     : integrate_phi, trapezoid weights (:348-360), both blocks
//  energy  : the sums of print_energy (:398-424) and the max incompressibility
//  update  : calc_new_fields, simple mixing (:362-371)
//  anderson: Anderson mixing in place of calc_new_fields (no counterpart in the reference)
//
// Reductions are deterministic: a fixed grid writes per-block partials, the last
// block to finish (atomic ticket, no waiting) reduces them in a fixed order.
#pragma once
#include <cuda_runtime.h>

namespace crysscft {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 592;  // 4 x 148 SMs

// Layout of the per-iteration record written by energy_kernel (doubles).
// HIST_RES: rms of the mixing residual r = (xN phiB + ksi - wA, xN phiA + ksi - wB) over both fields
enum { HIST_F = 0, HIST_EH, HIST_E0, HIST_E1, HIST_EK, HIST_MAXINC, HIST_Q, HIST_FLAGS, HIST_RES, HIST_STRIDE };

struct IterState {
    double Q;            // partition function of the current iteration
    unsigned ticket_q;   // last-block tickets
    unsigned ticket_e;
    unsigned iteration;  // iterations completed since the counter was reset
    int error;           // bit 0: Q <= 0 or not finite, bit 1: F not finite
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
// block-wide sum / max over kRedThreads threads; result valid in thread 0
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (kRedThreads / 32) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}
__device__ __forceinline__ double block_max(double v, double* sh) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (kRedThreads / 32) ? sh[lane] : 0.0;
        r = warp_max(r);
    }
    return r;
}

template <typename T>
__global__ void prep_kernel(const double* __restrict__ wA, const double* __restrict__ wB,
                            double* __restrict__ ksi, T* __restrict__ wAds, T* __restrict__ wBds,
                            T* __restrict__ q_first, T* __restrict__ qc_last, double xN, double ds,
                            long long M) {
    const double index = -ds / 2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        const double a = wA[i], b = wB[i];
        ksi[i] = 0.5 * (a + b - xN);
        wAds[i] = (T)(1. * exp(index * a));
        wBds[i] = (T)(1. * exp(index * b));
        q_first[i] = T(1);
        qc_last[i] = T(1);
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads)
q_reduce_kernel(const T* __restrict__ qc0, long long M, double* __restrict__ partials,
                IterState* st) {
    __shared__ double sh[kRedThreads / 32];
    __shared__ bool last;
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x)
        s += (double)qc0[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = s;
        __threadfence();
        const unsigned t = atomicAdd(&st->ticket_q, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double r = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) r += __ldcg(&partials[i]);
    r = block_sum(r, sh);
    if (threadIdx.x == 0) {
        const double Q = r / (double)M;
        st->Q = Q;
        st->ticket_q = 0;
        if (!(Q > 0.0) || !isfinite(Q)) st->error |= 1;
    }
}

// phi_A = sum_{u=0}^{NsA} w_u fA/(NsA Q) q[u] q+[u];  phi_B over u = NsA..NsA+NsB.
// q (forward chain) and qc (backward chain) hold U+1 = NsA+NsB+1 slices of M.  Each thread
// takes two neighbouring points (16-byte loads for FP64) and the slice loop is unrolled so
// several slices' loads are in flight; the sum runs over the slices in order.  The stored
// contour is read once, with streaming loads (it is larger than L2).
template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};

template <typename T>
__device__ __forceinline__ void phi_point_pair(const T* __restrict__ q, const T* __restrict__ qc, long long M,
                                               long long i, long long s0, long long ns, double c, double& a0,
                                               double& a1) {
    using P = typename Pair<T>::type;
#pragma unroll 4
    for (long long s = 0; s <= ns; ++s) {
        double factor = s == 0 ? 0.5 : (s == ns ? 0.5 : 1);
        factor *= c;
        const long long o = (s0 + s) * M + i;
        const P x = __ldcs(reinterpret_cast<const P*>(q + o));
        const P y = __ldcs(reinterpret_cast<const P*>(qc + o));
        a0 += factor * (double)x.x * (double)y.x;
        a1 += factor * (double)x.y * (double)y.y;
    }
}

template <typename T>
__global__ void phi_kernel(const T* __restrict__ q, const T* __restrict__ qc, double* __restrict__ phiA,
                           double* __restrict__ phiB, const IterState* st, double fA, long long NsA,
                           long long NsB, long long M) {
    const double Q = st->Q;
    const double fB = 1 - fA;
    const double cA = fA / (NsA * Q);
    const double cB = fB / (NsB * Q);
    if (M & 1) {  // odd M: pairs would straddle slices unaligned; one point per thread
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
             i += (long long)gridDim.x * blockDim.x) {
            double a = 0.0, b = 0.0;
            for (long long s = 0; s <= NsA; ++s) {
                double factor = s == 0 ? 0.5 : (s == NsA ? 0.5 : 1);
                factor *= cA;
                a += factor * (double)q[s * M + i] * (double)qc[s * M + i];
            }
            for (long long s = 0; s <= NsB; ++s) {
                double factor = s == 0 ? 0.5 : (s == NsB ? 0.5 : 1);
                factor *= cB;
                const long long u = NsA + s;
                b += factor * (double)q[u * M + i] * (double)qc[u * M + i];
            }
            phiA[i] = a;
            phiB[i] = b;
        }
        return;
    }
    const long long pairs = M / 2;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < pairs;
         j += (long long)gridDim.x * blockDim.x) {
        const long long i = 2 * j;
        double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
        phi_point_pair<T>(q, qc, M, i, 0, NsA, cA, a0, a1);
        phi_point_pair<T>(q, qc, M, i, NsA, NsB, cB, b0, b1);
        *reinterpret_cast<double2*>(phiA + i) = make_double2(a0, a1);
        *reinterpret_cast<double2*>(phiB + i) = make_double2(b0, b1);
    }
}

// phi from the alternating contour kernel's fused sums (cubic grid n^3, U = NsA + NsB even).
// acc[c][block][layout][tile][panel element] holds, for chain c, the sum of q(s) q+(s) over
// the slots s of the block that the chain finished in that layout, except slots 0, NsA,
// U/2 and U; those are added here with the trapezoid weights of integrate_phi
// (src/crysSCFT_sample.cpp:348-360: 1/2 at both ends of each block, 1 inside).  The panel
// element of grid point (x, y, z) is (z / 8) * 8n + row * 8 + z % 8, with row y in plane
// tile x and row x in slab tile y.
template <typename T>
__global__ void phi_fused_finish_kernel(const double* __restrict__ acc, const T* __restrict__ q,
                                        const T* __restrict__ qc, double* __restrict__ phiA,
                                        double* __restrict__ phiB, const IterState* st, double fA, long long NsA,
                                        long long NsB, int n) {
    const long long n2 = (long long)n * n, M = n2 * n, U = NsA + NsB;
    const double Q = st->Q;
    const double cA = fA / (NsA * Q), cB = (1 - fA) / (NsB * Q);
    long long sp[4] = {0, NsA, U / 2, U};
    int nsp = 4;
    if (U / 2 == NsA) {  // the midpoint is the block boundary
        sp[2] = U;
        nsp = 3;
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i / n2), y = (int)((i / n) % n), z = (int)(i % n);
        const long long zp = (long long)(z >> 3) * 8 * n + (z & 7);
        const long long ep = x * n2 + zp + y * 8;  // plane tile x, row y
        const long long es = y * n2 + zp + x * 8;  // slab tile y, row x
        double a = 0.0, b = 0.0;
        for (int c = 0; c < 2; ++c) {
            const double* t = acc + (size_t)c * 4 * M;
            a += t[ep] + t[M + es];
            b += t[2 * M + ep] + t[3 * M + es];
        }
        for (int j = 0; j < nsp; ++j) {
            const long long s = sp[j];
            const double w = (double)q[s * M + i] * (double)qc[s * M + i];
            if (s <= NsA) a += (s == 0 || s == NsA ? 0.5 : 1.0) * w;
            if (s >= NsA) b += (s == NsA || s == U ? 0.5 : 1.0) * w;
        }
        phiA[i] = cA * a;
        phiB[i] = cB * b;
    }
}

__global__ void __launch_bounds__(kRedThreads)
energy_kernel(const double* __restrict__ wA, const double* __restrict__ wB,
              const double* __restrict__ phiA, const double* __restrict__ phiB,
              const double* __restrict__ ksi, double xN, long long M, double* __restrict__ partials,
              IterState* st, double* __restrict__ hist, unsigned hist_cap) {
    __shared__ double sh[kRedThreads / 32];
    __shared__ bool last;
    double e1 = 0.0, eh = 0.0, ek = 0.0, mx = 0.0, rr = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        const double pa = phiA[i], pb = phiB[i];
        const double a = wA[i], b = wB[i], x = ksi[i];
        e1 += -a * pa - b * pb;
        eh += xN * pa * pb;
        const double temp = 1 - pa - pb;
        ek += -x * temp;
        mx = fmax(mx, fabs(temp));
        const double ra = xN * pb + x - a, rb = xN * pa + x - b;
        rr += ra * ra + rb * rb;
    }
    e1 = block_sum(e1, sh);
    eh = block_sum(eh, sh);
    ek = block_sum(ek, sh);
    mx = block_max(mx, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        partials[5 * blockIdx.x + 0] = e1;
        partials[5 * blockIdx.x + 1] = eh;
        partials[5 * blockIdx.x + 2] = ek;
        partials[5 * blockIdx.x + 3] = mx;
        partials[5 * blockIdx.x + 4] = rr;
        __threadfence();
        const unsigned t = atomicAdd(&st->ticket_e, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double r1 = 0.0, rh = 0.0, rk = 0.0, rm = 0.0, rs = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        r1 += __ldcg(&partials[5 * i + 0]);
        rh += __ldcg(&partials[5 * i + 1]);
        rk += __ldcg(&partials[5 * i + 2]);
        rm = fmax(rm, __ldcg(&partials[5 * i + 3]));
        rs += __ldcg(&partials[5 * i + 4]);
    }
    r1 = block_sum(r1, sh);
    rh = block_sum(rh, sh);
    rk = block_sum(rk, sh);
    rm = block_max(rm, sh);
    rs = block_sum(rs, sh);
    if (threadIdx.x == 0) {
        const double Q = st->Q;
        const double fe_entropic_0 = -log(Q);
        const double fe_entropic_1 = r1 / (double)M;
        const double fe_enthalpic = rh / (double)M;
        const double fe_ksi = rk / (double)M;
        const double F = fe_entropic_0 + fe_entropic_1 + fe_enthalpic + fe_ksi;
        if (!isfinite(F)) st->error |= 2;
        double* h = hist + (size_t)(st->iteration % hist_cap) * HIST_STRIDE;
        h[HIST_F] = F;
        h[HIST_EH] = fe_enthalpic;
        h[HIST_E0] = fe_entropic_0;
        h[HIST_E1] = fe_entropic_1;
        h[HIST_EK] = fe_ksi;
        h[HIST_MAXINC] = rm;
        h[HIST_Q] = Q;
        h[HIST_FLAGS] = (double)st->error;
        h[HIST_RES] = sqrt(rs / (2.0 * (double)M));
        st->ticket_e = 0;
    }
}

__global__ void update_kernel(double* __restrict__ wA, double* __restrict__ wB,
                              const double* __restrict__ phiA, const double* __restrict__ phiB,
                              const double* __restrict__ ksi, double xN, double acc, long long M,
                              IterState* st) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        wA[i] += acc * (xN * phiB[i] + ksi[i] - wA[i]);
        wB[i] += acc * (xN * phiA[i] + ksi[i] - wB[i]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->iteration += 1;
}

// ---------------------------------------------------------------------------
// Anderson mixing (replaces calc_new_fields when enabled; no counterpart in the
// reference).  The iterate w = (wA, wB) and residual r = (xN phiB + ksi - wA,
// xN phiA + ksi - wB) of every iteration go into a ring of history + 1 slots of 2M
// doubles; gram[a][b] = <r_a, r_b> is kept per ring slot.  With D_j = r_0 - r_j
// (0 the current iterate, j the j-th previous) the update solves
// sum_j <D_i, D_j> c_j = <D_i, r_0> and sets
// w <- w_0 + sum_j c_j (w_j - w_0) + beta (r_0 + sum_j c_j (r_j - r_0)).
// ---------------------------------------------------------------------------
constexpr int kAndersonMax = 32;

struct AndersonState {
    int count;    // previous iterates in the ring (<= history)
    int head;     // ring slot of the current iterate
    int k;        // previous iterates this iteration's update uses
    int restart;  // the last solve was singular: history restarted
    int slot[kAndersonMax + 1];  // slot[0] current, slot[j] the j-th previous
    double c[kAndersonMax];
    double gram[(kAndersonMax + 1) * (kAndersonMax + 1)];
    unsigned ticket;
};

// W[head] <- (wA, wB), R[head] <- residual
__global__ void anderson_record_kernel(const double* __restrict__ wA, const double* __restrict__ wB,
                                       const double* __restrict__ phiA, const double* __restrict__ phiB,
                                       const double* __restrict__ ksi, double xN, long long M,
                                       double* __restrict__ W, double* __restrict__ R, const AndersonState* as) {
    const long long base = (long long)as->head * 2 * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x) {
        const double a = wA[i], b = wB[i], x = ksi[i];
        W[base + i] = a;
        W[base + M + i] = b;
        R[base + i] = xN * phiB[i] + x - a;
        R[base + M + i] = xN * phiA[i] + x - b;
    }
}

// gram[head][s_j] = gram[s_j][head] = <R[head], R[s_j]>, j = 0..count (deterministic:
// per-block partials, the last block reduces them in block order)
__global__ void __launch_bounds__(kRedThreads)
anderson_dots_kernel(const double* __restrict__ R, long long M, int slots, double* __restrict__ partials,
                     AndersonState* as) {
    __shared__ double sh[kRedThreads / 32];
    __shared__ bool last;
    const int head = as->head, count = as->count;
    const long long n2 = 2 * M;
    const double* r0 = R + (long long)head * n2;
    for (int j = 0; j <= count; ++j) {
        const int sj = (head - j + slots) % slots;
        const double* rj = R + (long long)sj * n2;
        double d = 0.0;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2;
             i += (long long)gridDim.x * blockDim.x)
            d += r0[i] * rj[i];
        d = block_sum(d, sh);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * (kAndersonMax + 1) + j] = d;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(&as->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int j = 0; j <= count; ++j) {
        double r = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
            r += __ldcg(&partials[(size_t)b * (kAndersonMax + 1) + j]);
        r = block_sum(r, sh);
        if (threadIdx.x == 0) {
            const int sj = (head - j + slots) % slots;
            as->gram[head * (kAndersonMax + 1) + sj] = r;
            as->gram[sj * (kAndersonMax + 1) + head] = r;
        }
    }
    if (threadIdx.x == 0) as->ticket = 0;
}

// One thread: the k x k normal equations by Gaussian elimination with partial pivoting;
// a pivot below 1e-13 of the largest diagonal entry restarts the history (simple step).
// Then advances the ring.
__global__ void anderson_solve_kernel(AndersonState* as, int history) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int slots = history + 1;
    const int n = as->head, k = as->count;
    constexpr int G = kAndersonMax + 1;
    int s[kAndersonMax + 1];
    for (int j = 0; j <= k; ++j) s[j] = (n - j + slots) % slots;
    const double* g = as->gram;
    double U[kAndersonMax][kAndersonMax], V[kAndersonMax];
    const double g00 = g[n * G + n];
    double scale = 0.0;
    for (int i = 1; i <= k; ++i) {
        V[i - 1] = g00 - g[n * G + s[i]];
        for (int j = 1; j <= k; ++j) U[i - 1][j - 1] = g00 - g[n * G + s[j]] - g[s[i] * G + n] + g[s[i] * G + s[j]];
        scale = fmax(scale, fabs(U[i - 1][i - 1]));
    }
    bool singular = false;
    for (int col = 0; col < k && !singular; ++col) {
        int piv = col;
        for (int r = col + 1; r < k; ++r)
            if (fabs(U[r][col]) > fabs(U[piv][col])) piv = r;
        if (!(fabs(U[piv][col]) > 1e-13 * scale)) {
            singular = true;
            break;
        }
        if (piv != col) {
            for (int j = 0; j < k; ++j) {
                const double t = U[col][j];
                U[col][j] = U[piv][j];
                U[piv][j] = t;
            }
            const double t = V[col];
            V[col] = V[piv];
            V[piv] = t;
        }
        for (int r = col + 1; r < k; ++r) {
            const double f = U[r][col] / U[col][col];
            for (int j = col; j < k; ++j) U[r][j] -= f * U[col][j];
            V[r] -= f * V[col];
        }
    }
    if (!singular) {
        for (int r = k - 1; r >= 0; --r) {
            double acc = 0.0;
            for (int j = r + 1; j < k; ++j) acc += U[r][j] * as->c[j];
            as->c[r] = (V[r] - acc) / U[r][r];
        }
    }
    as->k = singular ? 0 : k;
    as->restart = singular ? 1 : 0;
    for (int j = 0; j <= k; ++j) as->slot[j] = s[j];
    const int kept = singular ? 0 : k;
    as->count = kept + 1 < history ? kept + 1 : history;
    as->head = (n + 1) % slots;
}

// (wA, wB) <- w_0 + sum_j c_j (w_j - w_0) + beta (r_0 + sum_j c_j (r_j - r_0))
__global__ void anderson_update_kernel(double* __restrict__ wA, double* __restrict__ wB,
                                       const double* __restrict__ W, const double* __restrict__ R,
                                       long long M, const AndersonState* as, double beta, IterState* st) {
    const int k = as->k;
    const long long n2 = 2 * M;
    const double* w0 = W + (long long)as->slot[0] * n2;
    const double* r0 = R + (long long)as->slot[0] * n2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2;
         i += (long long)gridDim.x * blockDim.x) {
        const double w = w0[i], r = r0[i];
        double dw = 0.0, dr = 0.0;
        for (int j = 1; j <= k; ++j) {
            const long long o = (long long)as->slot[j] * n2 + i;
            const double c = as->c[j - 1];
            dw += c * (W[o] - w);
            dr += c * (R[o] - r);
        }
        const double out = (w + dw) + beta * (r + dr);
        if (i < M) wA[i] = out;
        else wB[i - M] = out;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->iteration += 1;
}

// dst[i] = src[i] (type conversion allowed)
template <typename D, typename S>
__global__ void convert_kernel(D* __restrict__ dst, const S* __restrict__ src, long long M) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (D)src[i];
}

}  // namespace crysscft
