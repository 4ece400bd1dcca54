// Products of the complex-symmetric open-system pencil (config with a complex
// absorbing potential): AX = (H + i Himag) X and MX = M X for a block of b
// complex vectors, in one pass over the CSR arrays.
//
// H, Himag and M share one CSR pattern (qd_assemble writes all three), so a
// row's column indices are read once for the three matrices.  Blocks are
// row-major complex (re, im interleaved), X[row * ldx + c], with a leading
// dimension so that column slices of a wider basis can be read and written in
// place.
//
// Replaces the complex SpMV of the shift-invert Arnoldi that scipy's eigs
// runs for the reference's complex eigenvalue path (a12:
// backend/src/schrodinger.cpp:699-818 solves the same pencil densely with
// ComplexEigenSolver; fused_gpu_kernels.cu:97-125 is its never-launched
// scalar complex CSR SpMV).
#include <cuda_runtime.h>
#include <cstdint>
#include "common.h"

namespace {

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

constexpr int kLanes = 16;          // lanes per row: two rows per warp
constexpr int kRowsPerBlock = 16;   // 256 threads

// kLanes lanes per row; lane l owns columns l, l + 16, ... (C of them, so a
// 48-column block keeps every lane busy).  The row's CSR entries are loaded 16
// at a time, one per lane, and broadcast by shuffles within the half-warp,
// so each half-warp's vector loads are 16 consecutive complex values.
template <typename T, int C>
__global__ void __launch_bounds__(kRowsPerBlock * kLanes, 4)
cap_spmm_kernel(int32_t n, int b, int ldx, int ldy, const int32_t *__restrict__ rowptr,
                const int32_t *__restrict__ col, const T *__restrict__ H,
                const T *__restrict__ G, const T *__restrict__ M,
                const typename Vec2<T>::type *__restrict__ X, typename Vec2<T>::type *AX,
                typename Vec2<T>::type *MX) {
  using V = typename Vec2<T>::type;
  const int row = blockIdx.x * kRowsPerBlock + (threadIdx.x / kLanes);
  const int lane = threadIdx.x % kLanes;
  // the two rows of a warp are independent: shuffles stay inside each half
  const unsigned mask = 0xffffu << (threadIdx.x & 16);
  const bool live = row < n;
  T ar[C], ai[C], mr[C], mi[C];
#pragma unroll
  for (int c = 0; c < C; ++c) ar[c] = ai[c] = mr[c] = mi[c] = T(0);
  const int p0 = live ? rowptr[row] : 0, p1 = live ? rowptr[row + 1] : 0;
  for (int base = p0; base < p1; base += kLanes) {
    const int p = base + lane;
    int cj = 0;
    T h = T(0), g = T(0), m = T(0);
    if (p < p1) {
      cj = col[p];
      h = H[p];
      g = G ? G[p] : T(0);
      m = M[p];
    }
    const int cnt = min(kLanes, p1 - base);
    for (int q = 0; q < cnt; ++q) {
      const int j = __shfl_sync(mask, cj, q, kLanes);
      const T hq = __shfl_sync(mask, h, q, kLanes);
      const T gq = __shfl_sync(mask, g, q, kLanes);
      const T mq = __shfl_sync(mask, m, q, kLanes);
      const V *xr = X + size_t(j) * ldx;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int cc = c * kLanes + lane;
        if (cc < b) {
          const V x = xr[cc];
          // (h + i g)(xr + i xi) = (h xr - g xi) + i (h xi + g xr)
          ar[c] = fma(hq, x.x, fma(-gq, x.y, ar[c]));
          ai[c] = fma(hq, x.y, fma(gq, x.x, ai[c]));
          mr[c] = fma(mq, x.x, mr[c]);
          mi[c] = fma(mq, x.y, mi[c]);
        }
      }
    }
  }
  if (!live) return;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int cc = c * kLanes + lane;
    if (cc < b) {
      V a, mm;
      a.x = ar[c];
      a.y = ai[c];
      mm.x = mr[c];
      mm.y = mi[c];
      AX[size_t(row) * ldy + cc] = a;
      MX[size_t(row) * ldy + cc] = mm;
    }
  }
}

template <typename T>
int launch(int32_t n, int b, int ldx, int ldy, const int32_t *rowptr, const int32_t *col,
           const void *H, const void *G, const void *M, const void *X, void *AX, void *MX,
           cudaStream_t s) {
  using V = typename Vec2<T>::type;
  const unsigned blocks = unsigned((int64_t(n) + kRowsPerBlock - 1) / kRowsPerBlock);
  const T *h = static_cast<const T *>(H), *g = static_cast<const T *>(G),
          *m = static_cast<const T *>(M);
  const V *x = static_cast<const V *>(X);
  V *ax = static_cast<V *>(AX), *mx = static_cast<V *>(MX);
  const dim3 grid(blocks), block(kRowsPerBlock * kLanes);
  switch ((b + kLanes - 1) / kLanes) {
    case 1: cap_spmm_kernel<T, 1><<<grid, block, 0, s>>>(n, b, ldx, ldy, rowptr, col, h, g, m, x, ax, mx); break;
    case 2: cap_spmm_kernel<T, 2><<<grid, block, 0, s>>>(n, b, ldx, ldy, rowptr, col, h, g, m, x, ax, mx); break;
    case 3: cap_spmm_kernel<T, 3><<<grid, block, 0, s>>>(n, b, ldx, ldy, rowptr, col, h, g, m, x, ax, mx); break;
    default: cap_spmm_kernel<T, 4><<<grid, block, 0, s>>>(n, b, ldx, ldy, rowptr, col, h, g, m, x, ax, mx); break;
  }
  QD_CHECK_LAUNCH();
  return QD_OK;
}

}  // namespace

extern "C" int qd_cap_spmm(int32_t n, int b, int vec_fp32, const int32_t *d_rowptr,
                           const int32_t *d_col, const void *d_H, const void *d_Himag,
                           const void *d_M, const void *d_X, int ldx, void *d_AX, void *d_MX,
                           int ldy, void *stream) {
  if (n < 0 || b < 1 || b > 64 || ldx < b || ldy < b || !d_rowptr || !d_col || !d_H || !d_M ||
      !d_X || !d_AX || !d_MX)
    return QD_ERR_INVALID;
  if (n == 0) return QD_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (vec_fp32)
    return launch<float>(n, b, ldx, ldy, d_rowptr, d_col, d_H, d_Himag, d_M, d_X, d_AX, d_MX, s);
  return launch<double>(n, b, ldx, ldy, d_rowptr, d_col, d_H, d_Himag, d_M, d_X, d_AX, d_MX, s);
}
