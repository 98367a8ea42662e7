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
#include <cstdio>

namespace crysscft {

static const long double kPi = 3.141592653589793238462643383279502884L;

// g_k = exp(-ds (2 pi k / L)^2): the per-axis factor of K (src/solver_Pmmm.h:166-179,
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

std::vector<long double> circulant_kernel_dL(int N, long double L, long double ds) {
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

// ---------------------------------------------------------------------------
// CrysPSSolver3m with mirror translations.
//
// The reference builds, from g, seven twiddled copies of K (generate_m3_operation,
// src/solver_utilities.h:56-66; R_mat_generator_full / K_mat_generator,
// src/solver_3m.h:172-255) and recombines four sources per frequency
// (src/solver_3m.h:281-324).  In real space this is the 2x2y2z decomposition: the
// mirror normal to axis b maps the point p to  m_b(p) = p - 2 p_b e_b - e_b + t_b
// (grid units; -1 because the mirror sits between grid points), and the eight group
// elements m_x^cx m_y^cy m_z^cz (z applied first) carry the even sub-lattice onto the
// eight parity classes c of the full grid.  The triplet on the even sub-lattice is
// then the full-grid periodic operator T = T_x (x) T_y (x) T_z applied to that
// symmetric extension and restricted back:
//   out = sum_c (x)_a  S_a^{H_a(c)} B_a(c_a),
//   B_a(0)[i][i'] = c_a[(2i - 2i') mod N],  B_a(1)[i][i'] = c_a[(2i + 2i' + 1 - par_a) mod N],
// where H_a(c) = XOR over the other set mirrors b of half[a][b] and S_a is the cyclic
// shift by N/4 of the n = N/2 sub-lattice points (a half-cell translation).  S_a is an
// involution, S = P+ - P- with the projectors P(+/-) = (I +/- S)/2, and expanding every
// S^H over these projectors factorises the sum over c into one term per sector
// e = (e_x, e_y, e_z) in {+,-}^3:
//   out = sum_e (x)_a P_a^{e_a} (B_a(0) + sigma_a(e) B_a(1)),
//   sigma_a(e) = prod over b != a with e_b = - and half[b][a] = 1 of (-1).
// Sectors whose factors agree on two axes and differ on the third only in the
// projector are merged (P+ + P- = I), so g = 0 gives the single term
// B(0) + B(1) of m3_axis_operator.
// ---------------------------------------------------------------------------
namespace crysscft {

bool m3_symmetry_from_g(const double g[9], const size_t N[3], M3Symmetry* out, std::string* why) {
    M3Symmetry s;
    // translation of the mirror normal to axis b: g[0..2] for z, g[3..5] for y, g[6..8] for x
    for (int b = 0; b < 3; ++b) {
        const double* t = g + 3 * (2 - b);
        for (int a = 0; a < 3; ++a) {
            const double v = t[a] * (double)N[a];
            const double r = std::nearbyint(v);
            char buf[160];
            if (!std::isfinite(v) || std::fabs(v - r) > 1e-9 * (1.0 + std::fabs(v))) {
                std::snprintf(buf, sizeof(buf), "mirror %c translation along %c is not a whole number of grid points",
                              "xyz"[b], "xyz"[a]);
                *why = buf;
                return false;
            }
            long k = (long)r % (long)N[a];
            if (k < 0) k += (long)N[a];
            if (a == b) {
                if (k % 2) {
                    std::snprintf(buf, sizeof(buf),
                                  "mirror %c: its plane offset must be an even number of grid points", "xyz"[b]);
                    *why = buf;
                    return false;
                }
                s.par[a] = k;
            } else if (k != 0) {
                if (2 * k != (long)N[a] || N[a] % 4) {
                    std::snprintf(buf, sizeof(buf),
                                  "mirror %c translation along %c must be 0 or half a cell (with N %% 4 == 0)",
                                  "xyz"[b], "xyz"[a]);
                    *why = buf;
                    return false;
                }
                s.half[a][b] = 1;
            }
        }
    }
    *out = s;
    return true;
}

std::vector<M3Term> m3_terms(const M3Symmetry& sym) {
    std::vector<M3Term> terms;
    for (int e = 0; e < 8; ++e) {
        const int eps[3] = {(e >> 2) & 1, (e >> 1) & 1, e & 1};  // 1: the - eigenspace
        M3Term t;
        for (int a = 0; a < 3; ++a) {
            int sigma = 1;
            for (int b = 0; b < 3; ++b)
                if (b != a && eps[b] && sym.half[b][a]) sigma = -sigma;
            t[a].mask = 1 << eps[a];
            t[a].sigma = sigma;
        }
        terms.push_back(t);
    }
    auto same = [](const M3Factor& x, const M3Factor& y) { return x.mask == y.mask && x.sigma == y.sigma; };
    for (bool merged = true; merged;) {
        merged = false;
        for (size_t i = 0; i < terms.size() && !merged; ++i)
            for (size_t j = i + 1; j < terms.size() && !merged; ++j)
                for (int a = 0; a < 3 && !merged; ++a) {
                    const int b = (a + 1) % 3, c = (a + 2) % 3;
                    if (same(terms[i][b], terms[j][b]) && same(terms[i][c], terms[j][c]) &&
                        terms[i][a].sigma == terms[j][a].sigma && !(terms[i][a].mask & terms[j][a].mask)) {
                        terms[i][a].mask |= terms[j][a].mask;
                        terms.erase(terms.begin() + (long)j);
                        merged = true;
                    }
                }
    }
    return terms;
}

std::vector<long double> m3_axis_factor(const std::vector<long double>& c, int N, long par, M3Factor f) {
    const int n = N / 2;
    std::vector<long double> K((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int ip = 0; ip < n; ++ip) {
            const long d1 = ((2L * i - 2L * ip) % N + N) % N;
            const long d2 = ((2L * i + 2L * ip + 1 - N - par) % N + N) % N;
            K[(size_t)i * n + ip] = f.sigma > 0 ? c[d1] + c[d2] : c[d1] - c[d2];
        }
    if (f.mask == 3) return K;
    const long double sgn = f.mask == 1 ? 1.0L : -1.0L;
    std::vector<long double> P((size_t)n * n);
    for (int i = 0; i < n; ++i) {
        const int i2 = (i + n / 2) % n;
        for (int ip = 0; ip < n; ++ip)
            P[(size_t)i * n + ip] = (K[(size_t)i * n + ip] + sgn * K[(size_t)i2 * n + ip]) * 0.5L;
    }
    return P;
}

}  // namespace crysscft
