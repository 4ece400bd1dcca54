// Reference-element tables for P1/P2/P3 triangles, computed on the host from
// the quadrature rules the reference carries and the barycentric Lagrange
// bases of backend/src/fe_interpolator.cpp:474-613.
//   Mr[i][j]   = sum_q w_q phi_i phi_j
//   Sxx/Sxy/Syy = sum_q w_q (dxi_i dxi_j), (dxi_i deta_j + deta_i dxi_j), (deta_i deta_j)
//   T[l][i][j] = sum_q w_q phi_l phi_i phi_j
// with weights normalised to sum to one (element integrals = area * table).
#pragma once
#include <vector>

namespace qd {

struct RefTables {
  int order = 0, k = 0;
  std::vector<double> Mr, Sxx, Sxy, Syy, T;  // k*k, k*k, k*k, k*k, k*k*k
};

// barycentric quadrature points (lambda0, lambda1, lambda2) and weights
void quadrature_rule(int order, std::vector<double> &lam, std::vector<double> &w);
// shape values phi[k] and barycentric partials d[3][k] at lambda
void shape_functions(int order, const double lam[3], double *phi, double *d /*3*k*/);
RefTables make_tables(int order);

// offsets of each order's tables inside the packed constant-memory block
struct TableOffsets {
  int Mr, Sxx, Sxy, Syy, T;
};
constexpr int kTableDoubles = 63 + 360 + 1400;
void pack_tables(double *dst /*kTableDoubles*/, TableOffsets off[4]);

}  // namespace qd
