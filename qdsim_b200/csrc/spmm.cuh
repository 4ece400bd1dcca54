// Fused dual SpMM over the shared H/M CSR pattern for a block of B vectors
// stored row-major (X[row*B + j]).  G = B/4 threads cooperate on one row, each
// owning 4 consecutive columns (one float4 or two double2 per gathered row of
// X), so a warp reads 32/G consecutive CSR rows -- contiguous col/value
// streams -- and 16- or 32-byte vector loads of X.  Accumulation is FP64 in
// both storage precisions: the products are then accurate relative to the
// result itself, which avoids the cancellation floor that FP32 accumulation
// hits when |H||x| >> |Hx| (the low eigenvalues of a 1 nm P2 mesh sit
// ~1e3-1e4 below |H|).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace qd {

template <typename TV> struct V4;
template <> struct V4<float> {
  __device__ static inline void load(const float *p, double (&v)[4]) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
  __device__ static inline void store(float *p, const double (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(float(v[0]), float(v[1]), float(v[2]), float(v[3]));
  }
};
template <> struct V4<double> {
  __device__ static inline void load(const double *p, double (&v)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  __device__ static inline void store(double *p, const double (&v)[4]) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
  }
};

// Values of the two matrices at a nonzero: the caller's FP64 arrays.
struct MatF64 {
  const double *H, *M;
  __device__ void get(int p, double &h, double &m) const {
    h = __ldg(H + p);
    m = __ldg(M + p);
  }
};

// One row r, columns [4g, 4g+4): HX = H X, MX = M X.
template <typename TV, int B, typename MAT>
__device__ inline void spmm_row(int r, int g, const int32_t *__restrict__ rowptr,
                                const int32_t *__restrict__ col, const MAT &A,
                                const TV *__restrict__ X, TV *__restrict__ HX,
                                TV *__restrict__ MX) {
  double h[4] = {0.0, 0.0, 0.0, 0.0}, m[4] = {0.0, 0.0, 0.0, 0.0};
  const int p0 = __ldg(rowptr + r), p1 = __ldg(rowptr + r + 1);
#pragma unroll 4
  for (int p = p0; p < p1; ++p) {
    const int j = __ldg(col + p);
    double hv, mv;
    A.get(p, hv, mv);
    double x[4];
    V4<TV>::load(X + size_t(j) * B + 4 * g, x);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      h[c] = fma(hv, x[c], h[c]);
      m[c] = fma(mv, x[c], m[c]);
    }
  }
  V4<TV>::store(HX + size_t(r) * B + 4 * g, h);
  V4<TV>::store(MX + size_t(r) * B + 4 * g, m);
}

// Single-matrix variant (qd_spmm_dual with only H).
template <typename TV, int B>
__device__ inline void spmv_row(int r, int g, const int32_t *__restrict__ rowptr,
                                const int32_t *__restrict__ col, const double *__restrict__ H,
                                const TV *__restrict__ X, TV *__restrict__ HX) {
  double h[4] = {0.0, 0.0, 0.0, 0.0};
  const int p0 = __ldg(rowptr + r), p1 = __ldg(rowptr + r + 1);
#pragma unroll 4
  for (int p = p0; p < p1; ++p) {
    const int j = __ldg(col + p);
    const double hv = __ldg(H + p);
    double x[4];
    V4<TV>::load(X + size_t(j) * B + 4 * g, x);
#pragma unroll
    for (int c = 0; c < 4; ++c) h[c] = fma(hv, x[c], h[c]);
  }
  V4<TV>::store(HX + size_t(r) * B + 4 * g, h);
}

}  // namespace qd
