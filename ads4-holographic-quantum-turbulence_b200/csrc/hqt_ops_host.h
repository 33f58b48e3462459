// hqt_ops_host.h -- host-side operator construction (FP64).
#pragma once
#include <vector>

#include "hqt_common.cuh"

namespace hqt {

// Chebyshev points x (x[0] = +1) and D1 on N points, restating
// third_party/dmsuite/chebdif.m:25-53 (M = 1): trigonometric differences
// with the flipping trick, diagonal = -(row sum of the off-diagonals).
void chebdif_host(int N, std::vector<double> &x, std::vector<double> &D);

// Row i of the same D1 (N doubles), without allocating.
void chebdif_row(int N, int i, double *row);

// Inverse of an n x n row-major matrix by Gauss-Jordan elimination with
// partial pivoting in long double.  Returns false if singular.
bool invert_host(int n, const std::vector<double> &A, std::vector<double> &inv);

// Stockham plan of a line of length n.
FFTPlan make_plan(int n);

// roots[q] = exp(-2 pi i q / n), q < n, correctly rounded from long double.
std::vector<double2> make_roots(int n);

// cos/sin tables of the radix butterflies, in the order of kTabRadices.
void make_radix_tables(std::vector<double> &c, std::vector<double> &s);

// cos/sin tables of the large odd primes of the compile-time transforms.
void make_big_tables(std::vector<double> &c, std::vector<double> &s);

// MATLAB round of the filter band edges: 1-based indices lo..hi of the
// zeroed modes (tevol_driven_cluster.m:27-30).
void filter_band(int n, int &lo, int &hi);

}  // namespace hqt
