// Per-axis diffusion operators of the three solvers (row-major n x n, long double).
#pragma once
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

}  // namespace crysscft
