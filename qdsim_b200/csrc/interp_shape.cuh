// Lagrange shape functions of the P1/P2/P3 triangle in barycentric form and
// the reference's signed-area barycentric coordinates, shared by the
// structured-lattice and the refined-mesh interpolation kernels (the
// functions of backend/src/fe_interpolator.cpp:433-613).
#pragma once
#include <cuda_runtime.h>

namespace {

// integer barycentric multi-indices of the local nodes (x order)
template <int P> struct Local;
template <> struct Local<1> {
  static constexpr int K = 3;
  __host__ __device__ static int b(int a, int m) {
    constexpr int t[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    return t[a][m];
  }
};
template <> struct Local<2> {
  static constexpr int K = 6;
  __host__ __device__ static int b(int a, int m) {
    constexpr int t[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};
    return t[a][m];
  }
};
template <> struct Local<3> {
  static constexpr int K = 10;
  __host__ __device__ static int b(int a, int m) {
    constexpr int t[10][3] = {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {1, 2, 0},
                              {0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {2, 0, 1}, {1, 1, 1}};
    return t[a][m];
  }
};

// Barycentric coordinates by the signed-area formula of
// fe_interpolator.cpp:433-457 (same association of terms); returns the
// triangle's signed area.
__host__ __device__ __forceinline__ double bary(const double vx[3], const double vy[3], double x, double y,
                                       double l[3]) {
  const double area =
      0.5 * ((vx[1] - vx[0]) * (vy[2] - vy[0]) - (vx[2] - vx[0]) * (vy[1] - vy[0]));
  l[0] = 0.5 * ((vx[1] * vy[2] - vx[2] * vy[1]) + (vy[1] - vy[2]) * x + (vx[2] - vx[1]) * y) / area;
  l[1] = 0.5 * ((vx[2] * vy[0] - vx[0] * vy[2]) + (vy[2] - vy[0]) * x + (vx[0] - vx[2]) * y) / area;
  l[2] = 0.5 * ((vx[0] * vy[1] - vx[1] * vy[0]) + (vy[0] - vy[1]) * x + (vx[1] - vx[0]) * y) / area;
  return area;
}

// Shape values phi_a and derivatives d phi_a / d lambda_m of the Lagrange
// basis at the local nodes (the functions of fe_interpolator.cpp:474-613).
template <int P>
__host__ __device__ __forceinline__ void shape(const double l[3], double phi[], double dphi[][3]);

template <>
__host__ __device__ __forceinline__ void shape<1>(const double l[3], double phi[], double dphi[][3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    phi[a] = l[a];
#pragma unroll
    for (int m = 0; m < 3; ++m) dphi[a][m] = a == m ? 1.0 : 0.0;
  }
}

template <>
__host__ __device__ __forceinline__ void shape<2>(const double l[3], double phi[], double dphi[][3]) {
#pragma unroll
  for (int a = 0; a < 6; ++a)
#pragma unroll
    for (int m = 0; m < 3; ++m) dphi[a][m] = 0.0;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    phi[m] = l[m] * (2.0 * l[m] - 1.0);
    dphi[m][m] = 4.0 * l[m] - 1.0;
  }
  // edge nodes 3, 4, 5 on edges (0, 1), (1, 2), (2, 0)
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int i = e, j = (e + 1) % 3;
    phi[3 + e] = 4.0 * l[i] * l[j];
    dphi[3 + e][i] = 4.0 * l[j];
    dphi[3 + e][j] = 4.0 * l[i];
  }
}

template <>
__host__ __device__ __forceinline__ void shape<3>(const double l[3], double phi[], double dphi[][3]) {
#pragma unroll
  for (int a = 0; a < 10; ++a)
#pragma unroll
    for (int m = 0; m < 3; ++m) dphi[a][m] = 0.0;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    phi[m] = 0.5 * l[m] * (3.0 * l[m] - 1.0) * (3.0 * l[m] - 2.0);
    dphi[m][m] = 0.5 * (27.0 * l[m] * l[m] - 18.0 * l[m] + 2.0);
  }
  // edge (i, j) carries node 3 + 2e next to vertex i and 4 + 2e next to j
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int i = e, j = (e + 1) % 3;
    const int ni = 3 + 2 * e, nj = 4 + 2 * e;
    phi[ni] = 4.5 * l[i] * l[j] * (3.0 * l[i] - 1.0);
    phi[nj] = 4.5 * l[i] * l[j] * (3.0 * l[j] - 1.0);
    dphi[ni][i] = 4.5 * l[j] * (6.0 * l[i] - 1.0);
    dphi[ni][j] = 4.5 * l[i] * (3.0 * l[i] - 1.0);
    dphi[nj][i] = 4.5 * l[j] * (3.0 * l[j] - 1.0);
    dphi[nj][j] = 4.5 * l[i] * (6.0 * l[j] - 1.0);
  }
  phi[9] = 27.0 * l[0] * l[1] * l[2];
  dphi[9][0] = 27.0 * l[1] * l[2];
  dphi[9][1] = 27.0 * l[0] * l[2];
  dphi[9][2] = 27.0 * l[0] * l[1];
}

}  // namespace
