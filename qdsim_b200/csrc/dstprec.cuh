// Fast-sine-transform preconditioner for LOBPCG on structured rectangular
// meshes (no reference counterpart; the reference's eigensolves are
// unpreconditioned ARPACK / dense solves).
//
// For a dot whose reduced DOFs are the interior points of an nx x ny lattice
// (row-major), T = (cx Kx + cy Ky + shift I)^-1 where Kx, Ky are the 1-D
// second-difference matrices: the P1 stiffness of the lattice, spectrally
// equivalent to the P1/P2/P3 stiffness of the finite-element mesh, plus a
// shift that makes it positive definite.  DST-I diagonalises Kx and Ky, so
//   T R = Sx Sy (Lambda^-1 o (Sy Sx R)),   S symmetric orthonormal, S = S^-1,
// i.e. two transform-GEMMs along x and two along y per application, run for
// all dots and all B columns at once.  The transforms run in the precision of
// the vector storage: near convergence T r is dominated by a component along
// x itself and the useful correction is ~1e-6 of it, below FP32 resolution,
// so the FP64 finishing phase transforms in FP64.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "common.h"

namespace qd {

struct GemmTile {
  int dot, m0, n0, pad;
};

constexpr int kGemmTile = 64;     // rows (M) per tile
constexpr int kGemmTileN = 64;    // columns (N) per tile
constexpr int kGemmK = 16;

// out(r, n) = sum_k S[r][k] in(k, n)  (then / lambda when SCALE)
// x pass: r = ix, n = iy*B + b,  addr = base + (n / B) * nx*B + r*B + n % B
// y pass: r = iy, n = ix*B + b,  addr = base + r * nx*B + n
// 256 threads, each owns a 4 (rows) x 4 (columns) block of the 64 x 64 tile
// (small tiles keep the GPU busy when only a few large dots are still iterating).
// S is symmetric, so the A tile is read as S[k][r]: coalesced loads and
// conflict-free shared stores.  The next k-slice is prefetched into registers
// while the current one is multiplied.
template <typename TC, typename TI, typename TO, bool YPASS, bool SCALE>
__global__ void __launch_bounds__(256)
dst_gemm_kernel(const GemmTile *__restrict__ tiles, const int *__restrict__ active,
                int active_stride, const qd_dst_prec *__restrict__ desc,
                const int32_t *__restrict__ row_off, const double *__restrict__ mats, int B,
                const TI *__restrict__ in, TO *__restrict__ out) {
  const GemmTile t = tiles[blockIdx.x];
  if (active && !active[size_t(t.dot) * active_stride]) return;
  const qd_dst_prec d = desc[t.dot];
  const int nx = d.nx, ny = d.ny;
  const int dim = YPASS ? ny : nx;
  const int ncols = YPASS ? nx * B : ny * B;
  const double *S = mats + (YPASS ? d.sy_off : d.sx_off);
  const size_t base = size_t(row_off[t.dot]) * B;
  auto addr = [&](int r, int n) -> size_t {
    if (YPASS) return base + size_t(r) * (size_t(nx) * B) + n;
    return base + size_t(n / B) * (size_t(nx) * B) + size_t(r) * B + (n % B);
  };
  __shared__ __align__(16) TC As[kGemmK][kGemmTile + 4];
  __shared__ __align__(16) TC Bs[kGemmK][kGemmTileN + 4];
  const int tid = threadIdx.x;
  const int ty = tid / 16, tx = tid % 16;
  TC acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = TC(0);
  // per-thread load slots: A 4 elements (1024 / 256), B 4 elements (1024 / 256)
  TC ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      const int kk = e / kGemmTile, mm = e % kGemmTile;
      const int gk = k0 + kk, gm = t.m0 + mm;
      ra[q] = (gk < dim && gm < dim) ? TC(__ldg(S + size_t(gk) * dim + gm)) : TC(0);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      const int kk = e / kGemmTileN, nn = e % kGemmTileN;
      const int gk = k0 + kk, gn = t.n0 + nn;
      rb[q] = (gk < dim && gn < ncols) ? TC(in[addr(gk, gn)]) : TC(0);
    }
  };
  fetch(0);
  for (int k0 = 0; k0 < dim; k0 += kGemmK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      As[e / kGemmTile][e % kGemmTile] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      Bs[e / kGemmTileN][e % kGemmTileN] = rb[q];
    }
    __syncthreads();
    if (k0 + kGemmK < dim) fetch(k0 + kGemmK);
#pragma unroll
    for (int kk = 0; kk < kGemmK; ++kk) {
      TC a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  if (SCALE) {
    // eigenvalue tables for this tile: rows ky = m0.., columns kx = n0/B..
    __shared__ double s_sy[kGemmTile];
    __shared__ double s_sx[kGemmTileN / 4 + 2];
    const int kx0 = t.n0 / B;
    const int nkx = (t.n0 + kGemmTileN - 1) / B - kx0 + 1;
    if (tid < kGemmTile) {
      const double v = sinpi(double(t.m0 + tid + 1) / double(2 * (ny + 1)));
      s_sy[tid] = double(d.cy) * 4.0 * v * v;
    } else if (tid - kGemmTile < nkx) {
      const double v = sinpi(double(kx0 + tid - kGemmTile + 1) / double(2 * (nx + 1)));
      s_sx[tid - kGemmTile] = double(d.cx) * 4.0 * v * v;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = t.m0 + ty * 4 + i;
      if (r >= dim) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = t.n0 + tx * 4 + j;
        if (n >= ncols) continue;
        const double lam = s_sy[ty * 4 + i] + s_sx[n / B - kx0] + double(d.shift);
        out[addr(r, n)] = TO(double(acc[i][j]) / lam);
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = t.m0 + ty * 4 + i;
      if (r >= dim) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = t.n0 + tx * 4 + j;
        if (n < ncols) out[addr(r, n)] = TO(acc[i][j]);
      }
    }
  }
}

// Tile tables of the x and y passes for every dot with a preconditioner.
inline void dst_tiles(int n_dots, const qd_dst_prec *h, int B, GemmTile *tx, int64_t *ntx,
                      GemmTile *ty, int64_t *nty) {
  int64_t a = 0, b = 0;
  for (int d = 0; d < n_dots; ++d) {
    const int nx = h[d].nx, ny = h[d].ny;
    if (nx <= 0 || ny <= 0) continue;
    for (int m0 = 0; m0 < nx; m0 += kGemmTile)
      for (int n0 = 0; n0 < ny * B; n0 += kGemmTileN) {
        if (tx) tx[a] = GemmTile{d, m0, n0, 0};
        ++a;
      }
    for (int m0 = 0; m0 < ny; m0 += kGemmTile)
      for (int n0 = 0; n0 < nx * B; n0 += kGemmTileN) {
        if (ty) ty[b] = GemmTile{d, m0, n0, 0};
        ++b;
      }
  }
  *ntx = a;
  *nty = b;
}

// W <- T W using tmp1/tmp2 (TV, n x B each); compute precision = TV.
template <typename TV>
inline cudaError_t dst_apply(const GemmTile *tx, int64_t ntx, const GemmTile *ty, int64_t nty,
                             const int *active, int active_stride, const qd_dst_prec *desc,
                             const int32_t *row_off, const double *mats, int B, const TV *in,
                             TV *out, TV *tmp1, TV *tmp2, cudaStream_t s) {
  if (ntx == 0 || nty == 0) return cudaSuccess;
  dst_gemm_kernel<TV, TV, TV, false, false><<<unsigned(ntx), 256, 0, s>>>(
      tx, active, active_stride, desc, row_off, mats, B, in, tmp1);
  dst_gemm_kernel<TV, TV, TV, true, true><<<unsigned(nty), 256, 0, s>>>(
      ty, active, active_stride, desc, row_off, mats, B, tmp1, tmp2);
  dst_gemm_kernel<TV, TV, TV, true, false><<<unsigned(nty), 256, 0, s>>>(
      ty, active, active_stride, desc, row_off, mats, B, tmp2, tmp1);
  dst_gemm_kernel<TV, TV, TV, false, false><<<unsigned(ntx), 256, 0, s>>>(
      tx, active, active_stride, desc, row_off, mats, B, tmp1, out);
  g_launches.fetch_add(4, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace qd
