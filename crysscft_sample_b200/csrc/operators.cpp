// Per-axis diffusion operators of the three solvers.
//
// On its physical grid, each reference triplet (forward transform -> multiply by
// exp(-k^2 ds) -> backward transform -> normalise) is a linear map that factors
// into a Kronecker product A_x (x) A_y (x) A_z of three small dense matrices,
// because the transforms are separable and exp(-(kx^2+ky^2+kz^2) ds) is a product
// of per-axis factors.  This file builds each 1-D factor in long double from the
// reference's own definitions of K:
//
//  PMMM (src/solver_Pmmm.h:159-186, triplet :125-143, :194-215): REDFT10 along the
//    axis, multiply by g_k = exp(-ds (2 pi k / L)^2), k < n, REDFT01, times 1/(2n)
//    (the 1/(NxNyNz) of :128-142 is the product of the three 1/(2n)):
//      A[j][j'] = (1/n) sum_k c_k g_k cos(pi k (2j+1)/2n) cos(pi k (2j'+1)/2n),
//      c_0 = 1, c_k = 2.
//  P1 (src/solver_p1.h:142-172, :83-93, :184-202): r2c, K with k = 2 pi min(i, N-i)/L,
//    c2r, times 1/N per axis: a symmetric circulant
//      A[i][j] = c[(i - j) mod N],  c[d] = (1/N) sum_{k<N} g_{min(k,N-k)} cos(2 pi k d / N).
//  3M with zero mirror translations (src/solver_3m.h:184-255, :281-324): the 2x2y2z
//    algorithm applies, on the even sub-lattice f[2i], the full-grid periodic operator
//    to the mirror-symmetric extension f[N-1-2i] = f[2i] (mirrors between grid points),
//      A[i][i'] = c[(2i - 2i') mod N] + c[(2i + 2i' + 1 - N) mod N],  N = 2n.
//
// Trigonometric arguments are reduced exactly with integer arithmetic before cosl.
#include "operators.h"

#include <cmath>

namespace crysscft {

static const long double kPi = 3.141592653589793238462643383279502884L;

// g_k = exp(-ds (2 pi k / L)^2): the per-axis factor of K (src/solver_Pmmm.h:380-393,
// src/solver_p1.h:149-165, src/solver_3m.h:197-231)
static long double gauss(long k, long double L, long double ds) {
    long double kk = 2.0L * kPi * (long double)k / L;
    return expl(-ds * kk * kk);
}

std::vector<long double> pmmm_axis_operator(int n, long double L, long double ds) {
    // cos(pi m / (2n)) for m mod 4n
    const long period = 4L * n;
    std::vector<long double> ctab(period);
    for (long m = 0; m < period; ++m) ctab[m] = cosl(kPi * (long double)m / (2.0L * n));
    std::vector<long double> g(n);
    for (int k = 0; k < n; ++k) g[k] = gauss(k, L, ds) * (k == 0 ? 1.0L : 2.0L);
    std::vector<long double> A((size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int jp = 0; jp < n; ++jp) {
            long double acc = 0.0L;
            for (int k = 0; k < n; ++k) {
                long double a = ctab[((long)k * (2 * j + 1)) % period];
                long double b = ctab[((long)k * (2 * jp + 1)) % period];
                acc += g[k] * a * b;
            }
            A[(size_t)j * n + jp] = acc / (long double)n;
        }
    return A;
}

std::vector<long double> circulant_kernel(int N, long double L, long double ds) {
    std::vector<long double> ctab(N);
    for (int m = 0; m < N; ++m) ctab[m] = cosl(2.0L * kPi * (long double)m / (long double)N);
    std::vector<long double> g(N);
    for (int k = 0; k < N; ++k) g[k] = gauss(k < N - k ? k : N - k, L, ds);
    std::vector<long double> c(N);
    for (int d = 0; d < N; ++d) {
        long double acc = 0.0L;
        for (int k = 0; k < N; ++k) acc += g[k] * ctab[((long)k * d) % N];
        c[d] = acc / (long double)N;
    }
    return c;
}

std::vector<long double> p1_axis_operator(int N, long double L, long double ds) {
    std::vector<long double> c = circulant_kernel(N, L, ds);
    std::vector<long double> A((size_t)N * N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) A[(size_t)i * N + j] = c[((i - j) % N + N) % N];
    return A;
}

std::vector<long double> m3_axis_operator(int N, long double L, long double ds) {
    const int n = N / 2;
    std::vector<long double> c = circulant_kernel(N, L, ds);
    std::vector<long double> A((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int ip = 0; ip < n; ++ip) {
            long d1 = ((2L * i - 2L * ip) % N + N) % N;
            long d2 = ((2L * i + 2L * ip + 1 - N) % N + N) % N;
            A[(size_t)i * n + ip] = c[d1] + c[d2];
        }
    return A;
}

}  // namespace crysscft

// ---------------------------------------------------------------------------
// Cell-length derivatives.  Every operator above is linear in its spectral factor
// g_k = exp(-ds (2 pi k / L)^2), and dg_k/dL = g_k * 2 ds (2 pi k)^2 / L^3, so the
// derivative operator is the same construction with g replaced by dg/dL.
// ---------------------------------------------------------------------------
namespace crysscft {

static long double dgauss_dL(long k, long double L, long double ds) {
    const long double kk = 2.0L * kPi * (long double)k;
    return gauss(k, L, ds) * 2.0L * ds * kk * kk / (L * L * L);
}

std::vector<long double> pmmm_axis_operator_dL(int n, long double L, long double ds) {
    const long period = 4L * n;
    std::vector<long double> ctab(period);
    for (long m = 0; m < period; ++m) ctab[m] = cosl(kPi * (long double)m / (2.0L * n));
    std::vector<long double> g(n);
    for (int k = 0; k < n; ++k) g[k] = dgauss_dL(k, L, ds) * (k == 0 ? 1.0L : 2.0L);
    std::vector<long double> A((size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int jp = 0; jp < n; ++jp) {
            long double acc = 0.0L;
            for (int k = 0; k < n; ++k)
                acc += g[k] * ctab[((long)k * (2 * j + 1)) % period] * ctab[((long)k * (2 * jp + 1)) % period];
            A[(size_t)j * n + jp] = acc / (long double)n;
        }
    return A;
}

static std::vector<long double> circulant_kernel_dL(int N, long double L, long double ds) {
    std::vector<long double> ctab(N);
    for (int m = 0; m < N; ++m) ctab[m] = cosl(2.0L * kPi * (long double)m / (long double)N);
    std::vector<long double> g(N);
    for (int k = 0; k < N; ++k) g[k] = dgauss_dL(k < N - k ? k : N - k, L, ds);
    std::vector<long double> c(N);
    for (int d = 0; d < N; ++d) {
        long double acc = 0.0L;
        for (int k = 0; k < N; ++k) acc += g[k] * ctab[((long)k * d) % N];
        c[d] = acc / (long double)N;
    }
    return c;
}

std::vector<long double> p1_axis_operator_dL(int N, long double L, long double ds) {
    std::vector<long double> c = circulant_kernel_dL(N, L, ds);
    std::vector<long double> A((size_t)N * N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) A[(size_t)i * N + j] = c[((i - j) % N + N) % N];
    return A;
}

std::vector<long double> m3_axis_operator_dL(int N, long double L, long double ds) {
    const int n = N / 2;
    std::vector<long double> c = circulant_kernel_dL(N, L, ds);
    std::vector<long double> A((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int ip = 0; ip < n; ++ip) {
            long d1 = ((2L * i - 2L * ip) % N + N) % N;
            long d2 = ((2L * i + 2L * ip + 1 - N) % N + N) % N;
            A[(size_t)i * n + ip] = c[d1] + c[d2];
        }
    return A;
}

}  // namespace crysscft
