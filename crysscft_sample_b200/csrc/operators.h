// Per-axis diffusion operators of the three solvers (row-major n x n, long double).
#pragma once
#include <array>
#include <string>
#include <vector>

namespace crysscft {

// CrysPSSolverPmmm, one axis of n = N/2 points, cell length L
std::vector<long double> pmmm_axis_operator(int n, long double L, long double ds);
// c[d] of the full-grid periodic operator along an axis of N points
std::vector<long double> circulant_kernel(int N, long double L, long double ds);
// CrysPSSolverP1, one axis of N points
std::vector<long double> p1_axis_operator(int N, long double L, long double ds);
// CrysPSSolver3m (zero translations), one axis of n = N/2 even-sub-lattice points
std::vector<long double> m3_axis_operator(int N, long double L, long double ds);

// d/dL of the same operators (the cell-length derivative used by the stress)
std::vector<long double> pmmm_axis_operator_dL(int n, long double L, long double ds);
std::vector<long double> p1_axis_operator_dL(int N, long double L, long double ds);
std::vector<long double> m3_axis_operator_dL(int N, long double L, long double ds);
std::vector<long double> circulant_kernel_dL(int N, long double L, long double ds);

// ---------------------------------------------------------------------------
// CrysPSSolver3m with mirror translations (src/solver_3m.h:17, :172-182,
// src/solver_utilities.h:56-66).  g[0..2], g[3..5], g[6..8] are the translations
// (x, y, z components, in cell fractions) of the mirrors normal to z, y and x.
// ---------------------------------------------------------------------------
struct M3Symmetry {
    // half[a][b] = 1: the mirror normal to axis b translates by half a cell along axis a
    int half[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    // par[a]: translation of the mirror normal to axis a along that axis, in grid points
    long par[3] = {0, 0, 0};
};
// One Kronecker factor: P_s (B0 + sigma B1), where B0/B1 are the even->even and
// mirrored even->odd blocks of the full-grid circulant and P_s projects the output onto
// the +1 (mask 1), -1 (mask 2) or both (mask 3) eigenspaces of the half-cell shift.
struct M3Factor {
    int mask = 3;
    int sigma = 1;
};
using M3Term = std::array<M3Factor, 3>;

// Decode g for logical grid N; false (reason in *why) unless every mirror maps the even
// sub-lattice onto another parity class: perpendicular components 0 or 1/2 (with
// N % 4 == 0 on that axis for 1/2), parallel components an even number of grid points.
bool m3_symmetry_from_g(const double g[9], const size_t N[3], M3Symmetry* out, std::string* why);
// The operator as a sum of Kronecker products (one term when g = 0).
std::vector<M3Term> m3_terms(const M3Symmetry& sym);
// The factor matrix (n = N/2) on one axis, from the circulant kernel c of that axis.
std::vector<long double> m3_axis_factor(const std::vector<long double>& c, int N, long par, M3Factor f);

}  // namespace crysscft
