// Axis passes by fast Fourier transform (the "butterfly" form of the triplets, FP64 and FP32).
//
// Every per-axis operator of the three solvers is a real circulant with an even
// spectrum g, applied to an extension of the line and restricted back:
//   P1   (src/solver_p1.h:184-202):   the line itself, n points, g_k = exp(-ds (2 pi min(k, n-k) / L)^2)
//   PMMM (src/solver_Pmmm.h:194-215): DCT-II -> g -> DCT-III equals the 2n-point circulant on the
//        mirror extension [x_0..x_{n-1}, x_{n-1}..x_0] (mirrors between grid points), first n kept
//   3m   (src/solver_3m.h:281-324), zero translations: the full-grid (2n-point) circulant on the
//        mirror-symmetric extension of the even sub-lattice, z[2i] = x_i, z[2i+1] = x_{n-1-i},
//        even points kept
// with 1/NF folded into g (NF = the transform length).  Two real lines x1, x2 share one complex
// transform (z = ext(x1) + i ext(x2)); since g is real and even,
//   A x1 - i A x2 = FFT(conj(g . FFT(z)))
// so the inverse transform is a second forward one.  Each NF-point FFT (NF = 16 T, T = 4, 8, 16)
// is a four-step decomposition: T threads of a pair each hold 16 values x[T m + t]; a 16-point
// DFT in registers (radix 4 x 4), the twiddles W_NF^(t k1), one transposition through shared
// memory, then T-point DFTs (16 / T columns per thread).  The result lands in the same
// distribution (thread t holds index T m + t), which is what the second transform reads, so
// the two transforms need two shared-memory exchanges in total.  The Boltzmann factor is
// fused into the load (pre) and the store (post) as in the dense passes.
#pragma once
#include <cuda_runtime.h>

namespace crysscft {

constexpr int kFftThreads = 256;

// complex type of a real type
template <typename T> struct CplxOf;
template <> struct CplxOf<double> { using type = double2; };
template <> struct CplxOf<float> { using type = float2; };

template <typename T>
struct AxisFftPass {
    using C = typename CplxOf<T>::type;
    const T* in[2];
    T* out[2];
    const T* pre[2];         // input *= pre (nullptr: none)
    const T* post[2];        // output *= post (nullptr: none)
    const C* tw;             // NF twiddles exp(-2 pi i m / NF)
    const T* g;              // NF spectrum values, 1/NF included
    long long outer, inner;  // lines (o, i), element j of line (o, i) at o n inner + j inner + i
    int nchain;
};

template <int N, int NF, int EXT, typename R = double>
struct FftShape {
    static_assert(NF == 64 || NF == 128 || NF == 256, "transform lengths 64, 128, 256");
    static_assert((EXT == 0 && NF == N) || (EXT != 0 && NF == 2 * N), "P1: NF = n; PMMM, 3m: NF = 2n");
    static constexpr int T = NF / 16;               // threads per line pair
    static constexpr int PAIRS = kFftThreads / T;
    static constexpr int LINES = 2 * PAIRS;
    static constexpr int XROW = T + 1;              // exchange row (padded against bank conflicts)
    static constexpr int LS = N + 1;                // tile line stride: lines along l hit distinct banks
    static constexpr size_t TILE_BYTES = (size_t)LINES * LS * sizeof(R);
    static constexpr size_t XCH_BYTES = (size_t)PAIRS * 16 * XROW * 2 * sizeof(R);
    static constexpr size_t BUF_BYTES = TILE_BYTES > XCH_BYTES ? TILE_BYTES : XCH_BYTES;
    static constexpr size_t SMEM = BUF_BYTES + (size_t)NF * 3 * sizeof(R);
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 mul_minus_i(double2 a) { return make_double2(a.y, -a.x); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 mul_minus_i(float2 a) { return make_float2(a.y, -a.x); }
template <typename C> __device__ __forceinline__ C cmake(double x, double y);
template <> __device__ __forceinline__ double2 cmake<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 cmake<float2>(double x, double y) { return make_float2((float)x, (float)y); }

// in-place 4-point DFT (W4 = -i)
template <typename C>
__device__ __forceinline__ void dft4(C& a, C& b, C& c, C& d) {
    const C t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = mul_minus_i(csub(b, d));
    a = cadd(t0, t2);
    c = csub(t0, t2);
    b = cadd(t1, t3);
    d = csub(t1, t3);
}

// W16^j = exp(-2 pi i j / 16) for the products m2 k1 of a radix-4 x 4 16-point DFT
template <typename C>
__device__ __forceinline__ C w16(int j) {
    constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, h = 0.70710678118654752440;
    switch (j) {
        case 0: return cmake<C>(1.0, 0.0);
        case 1: return cmake<C>(c1, -s1);
        case 2: return cmake<C>(h, -h);
        case 3: return cmake<C>(s1, -c1);
        case 4: return cmake<C>(0.0, -1.0);
        case 6: return cmake<C>(-h, -h);
        default: return cmake<C>(-c1, s1);  // j = 9
    }
}

// out[k] = sum_m x[m] W16^(m k), k = k1 + 4 k2, m = 4 m1 + m2
template <typename C>
__device__ __forceinline__ void dft16(const C (&x)[16], C (&out)[16]) {
    C y[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) y[i] = x[i];
#pragma unroll
    for (int m2 = 0; m2 < 4; ++m2) dft4(y[m2], y[4 + m2], y[8 + m2], y[12 + m2]);  // -> y[4 k1 + m2]
#pragma unroll
    for (int m2 = 1; m2 < 4; ++m2)
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) y[4 * k1 + m2] = cmul(y[4 * k1 + m2], w16<C>(m2 * k1));
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4(y[4 * k1], y[4 * k1 + 1], y[4 * k1 + 2], y[4 * k1 + 3]);  // -> y[4 k1 + k2]
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) out[k1 + 4 * k2] = y[4 * k1 + k2];
}

// R-point DFT (R = 4, 8, 16) of x[0..R-1] in place
template <int R, typename C>
__device__ __forceinline__ void dft_small(C* x) {
    if constexpr (R == 4) {
        dft4(x[0], x[1], x[2], x[3]);
    } else if constexpr (R == 8) {
        // m = 2 m1 + m2: two 4-point DFTs, W8^k1 on the odd one, radix-2 combine
        C e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
        dft4(e[0], e[1], e[2], e[3]);
        dft4(o[0], o[1], o[2], o[3]);
        constexpr double h = 0.70710678118654752440;
        x[0] = cadd(e[0], o[0]);
        x[4] = csub(e[0], o[0]);
        const C t1 = cmul(o[1], cmake<C>(h, -h));
        x[1] = cadd(e[1], t1);
        x[5] = csub(e[1], t1);
        const C t2 = mul_minus_i(o[2]);
        x[2] = cadd(e[2], t2);
        x[6] = csub(e[2], t2);
        const C t3 = cmul(o[3], cmake<C>(-h, -h));
        x[3] = cadd(e[3], t3);
        x[7] = csub(e[3], t3);
    } else {
        C in[16], out[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) in[i] = x[i];
        dft16(in, out);
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = out[i];
    }
}

// NF-point forward FFT of one line pair, z[m] = x[T m + t] in, X[T m + t] out.
// xch: this pair's exchange rows (16 x XROW), tw: the NF twiddles (shared memory).
template <int NF, typename Cx>
__device__ __forceinline__ void fft_pair(Cx (&z)[16], Cx* xch, const Cx* tw, int t) {
    constexpr int T = NF / 16, XROW = T + 1, C = 16 / T;
    Cx y[16];
    dft16(z, y);  // y[k1] = sum_{n1} x[T n1 + t] W16^(n1 k1)
    // twiddles W_NF^(t k1) as a running product of W_NF^t (one table read per thread: the
    // strided reads tw[t k1] collided on the shared-memory banks); <= 15 products, ~1e-15
    const Cx wt = tw[t];
    Cx w = wt;
    xch[t] = y[0];
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) {
        xch[k1 * XROW + t] = cmul(y[k1], w);
        w = cmul(w, wt);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const int k1 = t + T * c;
        Cx col[T];
#pragma unroll
        for (int n2 = 0; n2 < T; ++n2) col[n2] = xch[k1 * XROW + n2];
        dft_small<T>(col);  // col[k2] = X[k1 + 16 k2]
#pragma unroll
        for (int k2 = 0; k2 < T; ++k2) z[c + C * k2] = col[k2];  // index k1 + 16 k2 = t + T (c + C k2)
    }
    __syncthreads();  // the exchange rows may be written again
}

template <int N, int NF, int EXT, typename R = double>
__global__ void __launch_bounds__(kFftThreads) axis_fft_kernel(const AxisFftPass<R> p) {
    using S = FftShape<N, NF, EXT, R>;
    using Cx = typename CplxOf<R>::type;
    constexpr int T = S::T, LINES = S::LINES, LS = S::LS;
    constexpr int PER = LINES * N / kFftThreads;  // tile values per thread
    // loads in flight per thread and chunk (measured on B200: 16 for 256-point FP64 lines and
    // for FP32, where the registers allow it at the same occupancy; 8 for 128-point FP64
    // lines, where 16 lowered occupancy and was 9 % slower)
    constexpr int CHMAX = (N >= 256 || sizeof(R) == 4) ? 16 : 8;
    constexpr int CH = PER < CHMAX ? PER : CHMAX;
    static_assert(LINES * N % kFftThreads == 0 && PER % CH == 0, "whole chunks per thread");
    extern __shared__ __align__(16) unsigned char fft_raw[];
    __shared__ long long s_base[LINES];  // offset of element 0 of each line of the tile (-1: none)
    R* buf = reinterpret_cast<R*>(fft_raw);
    Cx* xch = reinterpret_cast<Cx*>(fft_raw);  // aliases the tile between its uses
    Cx* stw = reinterpret_cast<Cx*>(fft_raw + S::BUF_BYTES);
    R* sg = reinterpret_cast<R*>(stw + NF);
    const int tid = threadIdx.x;
    for (int e = tid; e < NF; e += kFftThreads) {
        stw[e] = p.tw[e];
        sg[e] = p.g[e];
    }
    const int pair = tid / T, t = tid - (tid / T) * T;
    const long long lines = p.outer * p.inner;  // per chain
    const long long tiles_per_chain = (lines + LINES - 1) / LINES;
    const long long tiles = tiles_per_chain * p.nchain;
    const long long stride_line = (long long)N * p.inner;
    const bool contiguous = p.inner == 1;
    const long long inner = p.inner;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int c = (int)(tile / tiles_per_chain);
        const long long L0 = (tile - (long long)c * tiles_per_chain) * LINES;
        const R* in = p.in[c];
        const R* pre = p.pre[c];
        __syncthreads();  // the previous tile's stores have read the buffer and the line offsets
        // line offsets of this tile: one division per line, not per element
        for (int l = tid; l < LINES; l += kFftThreads) {
            const long long L = L0 + l;
            long long b = -1;
            if (L < lines) {
                const long long o = L / inner;
                b = o * stride_line + (L - o * inner);
            }
            s_base[l] = b;
        }
        __syncthreads();
        // load the tile (buf[l][j]), coalesced along j for contiguous lines, along l otherwise;
        // the loads of a chunk are all issued before its shared-memory stores, so their
        // latencies overlap
#pragma unroll 1
        for (int k0 = 0; k0 < PER; k0 += CH) {
            R v[CH], w[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = tid + (k0 + k) * kFftThreads;
                const int l = contiguous ? e / N : e % LINES;
                const int j = contiguous ? e % N : e / LINES;
                const long long b = s_base[l];
                const long long idx = b + (long long)j * inner;
                v[k] = b >= 0 ? __ldg(in + idx) : R(0);
                w[k] = (b >= 0 && pre) ? __ldg(pre + idx) : R(1);
            }
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = tid + (k0 + k) * kFftThreads;
                const int l = contiguous ? e / N : e % LINES;
                const int j = contiguous ? e % N : e / LINES;
                buf[l * LS + j] = v[k] * w[k];
            }
        }
        __syncthreads();
        Cx z[16];
        const R* l1 = buf + (2 * pair) * LS;
        const R* l2 = l1 + LS;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int k = T * m + t;
            int e;
            if constexpr (EXT == 0) e = k;
            else if constexpr (EXT == 1) e = k < N ? k : 2 * N - 1 - k;
            else e = (k & 1) ? N - 1 - (k >> 1) : (k >> 1);
            z[m].x = l1[e];
            z[m].y = l2[e];
        }
        __syncthreads();  // the tile is read: its memory becomes the exchange rows
        Cx* my = xch + (size_t)pair * 16 * S::XROW;
        fft_pair<NF>(z, my, stw, t);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const R gk = sg[T * m + t];
            z[m].x = z[m].x * gk;
            z[m].y = -z[m].y * gk;
        }
        fft_pair<NF>(z, my, stw, t);
        // results: A x1 = Re, A x2 = -Im, at the kept points of the extension
        R* o1 = buf + (2 * pair) * LS;
        R* o2 = o1 + LS;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int k = T * m + t;
            if constexpr (EXT == 0) {
                o1[k] = z[m].x;
                o2[k] = -z[m].y;
            } else if constexpr (EXT == 1) {
                if (k < N) {
                    o1[k] = z[m].x;
                    o2[k] = -z[m].y;
                }
            } else {
                if (!(k & 1)) {
                    o1[k >> 1] = z[m].x;
                    o2[k >> 1] = -z[m].y;
                }
            }
        }
        __syncthreads();
        R* out = p.out[c];
        const R* post = p.post[c];
#pragma unroll 1
        for (int k0 = 0; k0 < PER; k0 += CH) {
            R w[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = tid + (k0 + k) * kFftThreads;
                const int l = contiguous ? e / N : e % LINES;
                const int j = contiguous ? e % N : e / LINES;
                const long long b = s_base[l];
                w[k] = (b >= 0 && post) ? __ldg(post + b + (long long)j * inner) : R(1);
            }
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = tid + (k0 + k) * kFftThreads;
                const int l = contiguous ? e / N : e % LINES;
                const int j = contiguous ? e % N : e / LINES;
                const long long b = s_base[l];
                if (b >= 0) out[b + (long long)j * inner] = buf[l * LS + j] * w[k];
            }
        }
    }
}

}  // namespace crysscft
